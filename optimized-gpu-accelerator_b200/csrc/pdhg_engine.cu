// PDHG engine for one B200: device state, the iteration loop, and the C ABI
// declared in include/b2p_pdhg.h.
//
// The loop restates runPdhg (src/pdhg/pdhg.cpp:483-687).  What changes is
// how it drives the GPU:
//   - one check interval (check_every iterations, ending with the check) is
//     enqueued as 2 fused kernels per iteration plus 4 check kernels and one
//     small device->host copy, and captured once into a CUDA graph that is
//     replayed for every interval (the reference issues ~8 launches per
//     iteration and 2-4 blocking copies per check, pdhg.cpp:286-370);
//   - the check reductions finish on the device: the host reads 10 doubles
//     per case per check;
//   - the host keeps exactly the reference's decisions (termination, restart,
//     primal weight; pdhg.cpp:604-659) in FP64 with the C library's sqrt/exp/log.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/b2p_pdhg.h"
#include "pdhg_host_common.h"
#include "pdhg_kernels.cuh"
#include "pdhg_prepare.h"
#include "pdhg_restart.h"
#include "pdhg_scale.cuh"
#include "pdhg_batch32.cuh"
#include "pdhg_resident.cuh"
#include "pdhg_sched.h"
#include "pdhg_spmv.cuh"

namespace b2p {

namespace {

// Device vector slots (the reference's enum V, src/pdhg/pdhg.cpp:45, minus
// ATY/ATYP which the fused kernels never store, plus the initial point).
enum Slot : int { X, XP, X0, C, LO, UP, XINIT, ATYP, NCOLVEC, Y = NCOLVEC, YP, Y0, AX, AXP, AX0, RL, RU, AXINIT,
                  YINIT, NSLOT };
inline bool row_slot(int s) { return s >= Y; }

template <class T>
using ResidentFn = void (*)(ResidentArgs<T>);

template <class T, int GC>
ResidentFn<T> resident_fn_rows(int gr) {
  switch (gr) {
    case 1: return k_resident<GC, 1, T>;
    case 2: return k_resident<GC, 2, T>;
    case 4: return k_resident<GC, 4, T>;
    default: return k_resident<GC, 8, T>;
  }
}

template <class T>
ResidentFn<T> resident_fn(int gc, int gr) {
  switch (gc) {
    case 1: return resident_fn_rows<T, 1>(gr);
    case 2: return resident_fn_rows<T, 2>(gr);
    case 4: return resident_fn_rows<T, 4>(gr);
    default: return resident_fn_rows<T, 8>(gr);
  }
}

// Contiguous split of M's rows into nb parts of near-equal (nnz + 4 rows).
std::vector<int32_t> balanced_split(const HostCsr& M, int nb) {
  std::vector<int32_t> b(nb + 1, M.rows);
  b[0] = 0;
  const double total = static_cast<double>(M.ptr[M.rows]) + 4.0 * M.rows;
  int part = 1;
  double acc = 0;
  for (int32_t i = 0; i < M.rows && part < nb; ++i) {
    acc += (M.ptr[i + 1] - M.ptr[i]) + 4.0;
    while (part < nb && acc >= total * part / nb) b[part++] = i + 1;
  }
  for (; part < nb; ++part) b[part] = M.rows;
  return b;
}

// Lanes per short row in the resident kernel: at most 1024/G groups must
// cover the block's rows in one pass; no more lanes than 90% of rows need.
int resident_lanes(const HostCsr& M, const std::vector<int32_t>& bounds) {
  int max_rows = 1;
  for (size_t b = 0; b + 1 < bounds.size(); ++b) max_rows = std::max(max_rows, bounds[b + 1] - bounds[b]);
  int cap = 1;
  while (cap < 8 && (kResidentThreads / (cap * 2)) >= max_rows) cap *= 2;
  std::vector<int32_t> len(M.rows);
  for (int32_t i = 0; i < M.rows; ++i) len[i] = M.ptr[i + 1] - M.ptr[i];
  int p90 = 0;
  if (!len.empty()) {
    const size_t q = static_cast<size_t>(0.9 * (len.size() - 1));
    std::nth_element(len.begin(), len.begin() + q, len.end());
    p90 = len[q];
  }
  int need = 1;
  while (need < 8 && need * kResUnroll < p90) need *= 2;
  return std::min(cap, need);
}

}  // namespace

// dst[r * k2 + q] = src[r * k + map[q]]: the k-interleaved rows of a vector
// with only the cases map[0..k2) kept (case compaction of a batch).
__global__ void __launch_bounds__(kBlock) k_pack_cases(int64_t rows, int32_t k, int32_t k2,
                                                       const int32_t* __restrict__ map, const double* __restrict__ src,
                                                       double* __restrict__ dst) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= rows * k2) return;
  const int64_t r = t / k2;
  dst[t] = src[r * k + map[t - r * k2]];
}

struct Engine {
  // ---- problem ----
  int device = 0;
  int n = 0, m = 0, k = 1;
  bool batch = false;
  b2p_options opt{};
  Prepared P;
  std::vector<double> cNorm, rhsNorm, omega0;
  std::vector<double> omega_cold, x_cold;  // the reference's starting weights and x (scaled, interleaved)
  bool warm = false;                       // a caller-given start replaces x0 = proj(0), y0 = 0
  double eta = 0;

  // ---- device ----
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  int32_t *dA_ptr = nullptr, *dA_idx = nullptr, *dT_ptr = nullptr, *dT_idx = nullptr;
  double *dA_val = nullptr, *dT_val = nullptr, *d_rfac = nullptr, *d_cfac = nullptr;
  double* v[NSLOT] = {};
  // Case compaction of a batch (FP64 phase): when half the live cases have
  // terminated, the rest are packed into a narrower interleave, so that the
  // kernels stop streaming the finished cases' vectors.  k is the current
  // width, case_of maps a packed case to the engine's case; v_full and k_full
  // are the engine's own buffers and width, restored when the solve ends.
  int k_full = 1;
  double* v_full[NSLOT] = {};
  std::vector<int32_t> case_of;
  int32_t* d_case_map = nullptr;
  int compactions = 0;
  double *d_tau = nullptr, *d_sigma = nullptr, *d_prow = nullptr, *d_pcol = nullptr, *d_sums = nullptr;
  int64_t *d_it_base = nullptr, *d_restart_at = nullptr;
  int32_t* d_mask = nullptr;
  int g_rows = 1, g_cols = 1;
  RowBins binsA{}, binsT{};  // k == 1 schedules of A and A^T
  // resident form
  bool resident = false;
  int res_blocks = 0, res_gc = 1, res_gr = 1;
  size_t res_smem = 0;
  int32_t *d_cb = nullptr, *d_rb = nullptr;
  unsigned* d_sync = nullptr;  // arrive, generation, error flag
  double* d_rpartial = nullptr;
  int32_t* h_error = nullptr;
  ResidentFn<double> res_fn = nullptr;
  // mixed form: FP32 operator values and iterates for the resident kernel
  bool mixed = false;    // precision MIXED requested and the FP32 resident form fits
  bool phase32 = false;  // the current interval runs in FP32
  size_t res_smem32 = 0;
  ResidentFn<float> res_fn32 = nullptr;
  float *a_val32 = nullptr, *t_val32 = nullptr;
  enum Slot32 : int { X32, XP32, X032, Y32, YP32, Y032, AX32, AX032, AXP32, C32, LO32, UP32, RL32, RU32, NSLOT32 };
  float* v32[NSLOT32] = {};

  // ---- pinned host ----
  double* h_sums = nullptr;   // k * kNumSums
  double* h_steps = nullptr;  // tau[k], sigma[k]
  int32_t* h_mask = nullptr;

  // ---- graphs and profiling ----
  std::map<int, cudaGraphExec_t> graphs, graphs32;  // per interval length; FP32 phase of a batch
  std::map<int, cudaGraph_t> graph_defs, graph_defs32;
  bool mixed_batch = false;  // mixed form of a batch (k > 1): FP32 k-interleaved kernels
  bool batch_stream_p = false, batch_stream_d = false;  // evict-first streamed vectors (tuned per kernel)
  int batch_cpt_p = 1, batch_cpt_d = 1;  // cases per thread of the primal / dual batch kernels (tuned)
  bool batch_wr_p = false, batch_wr_d = false;  // whole warps per row, entries passed by shuffle (tuned)
  bool batch_wr_p_full = false, batch_wr_d_full = false;  // the tuned choice, restored after a compaction
  int batch_tr_p = 0, batch_tr_d = 0;  // rows per block of the row-tiled layout (0 = one row's cases per block; tuned)
  bool profiling = false;
  std::vector<cudaEvent_t> prof_ev;  // 4 per iteration of the longest interval
  int64_t prof_launches[5] = {0, 0, 0, 0, 0};
  double prof_ms[5] = {0, 0, 0, 0, 0};
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;

  // ---- last solve ----
  std::vector<double> x_out, y_out;  // num_cases x n / x m, original space
  std::vector<b2p_result> results;
  b2p_stats stats{};
  int64_t launches = 0;
  int64_t bytes_up = 0, bytes_down = 0;
  double transfer_seconds = 0;

  template <class T>
  T* dalloc(size_t count) {
    void* p = nullptr;
    B2P_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(count, 1) * sizeof(T), device_pool(device), stream));
    allocs.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const std::vector<T>& h) {
    T* d = dalloc<T>(h.size());
    if (!h.empty()) B2P_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    bytes_up += static_cast<int64_t>(h.size() * sizeof(T));
    return d;
  }

  ~Engine() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    for (auto& g : graph_defs) cudaGraphDestroy(g.second);
    for (auto& g : graphs32) cudaGraphExecDestroy(g.second);
    for (auto& g : graph_defs32) cudaGraphDestroy(g.second);
    for (auto e : prof_ev) cudaEventDestroy(e);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    cudaSetDevice(device);
    if (stream) {
      for (void* p : allocs) cudaFreeAsync(p, stream);
      cudaStreamSynchronize(stream);
    }
    PinnedCache::put(h_sums, sizeof(double) * k * kNumSums);
    PinnedCache::put(h_steps, sizeof(double) * 2 * k);
    PinnedCache::put(h_mask, sizeof(int32_t) * k);
    PinnedCache::put(h_error, sizeof(int32_t));
    if (stream) cudaStreamDestroy(stream);
  }

  CsrView viewA() const { return CsrView{dA_ptr, dA_idx, dA_val, m}; }
  CsrView viewAT() const { return CsrView{dT_ptr, dT_idx, dT_val, n}; }
  static unsigned blocks(int64_t len) { return static_cast<unsigned>(std::max<int64_t>(1, (len + kBlock - 1) / kBlock)); }
  static int red_blocks(int64_t len) {
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(4 * 148, (len + kBlock - 1) / kBlock)));
  }

  void create(const b2p_lp* lp, const b2p_case* cases, int num_cases, const b2p_options* o) {
    check_lp(lp);
    if (o) opt = *o; else b2p_default_options(&opt);
    if (opt.check_every <= 0) throw Error(B2P_ERR_INVALID, "check_every must be positive");
    if (opt.precision != B2P_PRECISION_FP64 && opt.precision != B2P_PRECISION_MIXED)
      throw Error(B2P_ERR_INVALID, "unsupported precision");
    device = pick_device(opt.device);
    B2P_CUDA(cudaSetDevice(device));
    B2P_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    B2P_CUDA(cudaEventCreate(&ev_start));
    B2P_CUDA(cudaEventCreate(&ev_stop));
    batch = num_cases > 0;
    k = batch ? num_cases : 1;
    n = lp->num_cols;
    m = lp->num_rows;
    const auto t0 = Clock::now();

    // Structure (the CSR of A) on host threads; the scaling (Ruiz,
    // Pock-Chambolle, the scaled operators) and ||A|| on the device, the
    // power-of-two rounding and beta / gamma on the host -- bit-identical to
    // the host's prepare() (pdhg_scale.cuh).
    P = prepare_structure(m, n, lp->start, lp->index, lp->value, lp->obj_offset, true);
    const auto tx = Clock::now();
    dA_ptr = upload(P.A.ptr);
    dA_idx = upload(P.A.idx);
    dA_val = upload(P.A.val);
    dT_ptr = upload(P.AT.ptr);
    dT_idx = upload(P.AT.idx);
    dT_val = upload(P.AT.val);
    {
      std::vector<double> rs(m, 1.0), cs(n, 1.0);
      if (opt.ruiz_iterations > 0 && !P.A.val.empty())
        device_ruiz_factors(stream, device, viewA(), viewAT(), opt.ruiz_iterations, opt.pock_chambolle != 0, rs, cs);
      finish_scaling(P, rs.data(), cs.data(), lp->col_cost, lp->row_lower, lp->row_upper,
                     opt.rescale_objective_and_bounds != 0);
      device_scale_operators(stream, device, viewA(), viewAT(), dA_val, dT_val, P.R, P.Cs);
    }
    stats.prepare_seconds = seconds_since(t0);

    // Case data in scaled space, k-interleaved (src/pdhg/pdhg.cpp:466-481, 506-530).
    const size_t nk = static_cast<size_t>(n) * k, mk = static_cast<size_t>(m) * k;
    std::vector<double> c(nk), lo(nk), up(nk), rl(mk), ru(mk), x(nk);
    cNorm.assign(k, 0.0);
    rhsNorm.assign(k, 0.0);
    omega0.assign(k, 1.0);
    for (int b = 0; b < k; ++b) {
      const b2p_case* cs = batch ? &cases[b] : nullptr;
      const double* cc = (cs && cs->cost) ? cs->cost : lp->col_cost;
      const double* cl = (cs && cs->col_lower) ? cs->col_lower : lp->col_lower;
      const double* cu = (cs && cs->col_upper) ? cs->col_upper : lp->col_upper;
      const double* rlo = (cs && cs->row_lower) ? cs->row_lower : lp->row_lower;
      const double* rup = (cs && cs->row_upper) ? cs->row_upper : lp->row_upper;
      double s = 0;
      for (int j = 0; j < n; ++j) s += cc[j] * cc[j];
      cNorm[b] = std::sqrt(s);
      s = 0;
      for (int i = 0; i < m; ++i) {
        if (finite_bound(rlo[i])) s += rlo[i] * rlo[i];
        if (finite_bound(rup[i]) && rup[i] != rlo[i]) s += rup[i] * rup[i];
      }
      rhsNorm[b] = std::sqrt(s);
      double cn = 0, bn = 0;
      for (int j = 0; j < n; ++j) {
        const size_t t = static_cast<size_t>(j) * k + b;
        c[t] = cc[j] * P.Cs[j] / P.gamma;
        lo[t] = finite_bound(cl[j]) ? cl[j] / P.Cs[j] / P.beta : -HUGE_VAL;
        up[t] = finite_bound(cu[j]) ? cu[j] / P.Cs[j] / P.beta : HUGE_VAL;
        x[t] = smin(smax(0.0, lo[t]), up[t]);
        cn += c[t] * c[t];
      }
      for (int i = 0; i < m; ++i) {
        const size_t t = static_cast<size_t>(i) * k + b;
        rl[t] = finite_bound(rlo[i]) ? rlo[i] * P.R[i] / P.beta : -HUGE_VAL;
        ru[t] = finite_bound(rup[i]) ? rup[i] * P.R[i] / P.beta : HUGE_VAL;
        if (finite_bound(rl[t])) bn += rl[t] * rl[t];
        if (finite_bound(ru[t]) && ru[t] != rl[t]) bn += ru[t] * ru[t];
      }
      if (cn > 1e-20 && bn > 1e-20) omega0[b] = std::sqrt(cn) / std::sqrt(bn);
    }

    // ---- device state (GpuBackend::init, src/pdhg/pdhg.cpp:238-277) ----
    const auto tn = Clock::now();
    P.normA = device_power_iteration(40) * 1.01;
    stats.prepare_seconds += seconds_since(tn);
    eta = 0.998 / P.normA;
    d_rfac = upload(P.rfac);
    d_cfac = upload(P.cfac);
    if (k == 1) {
      const auto tk = Clock::now();
      int per_sm = 0;
      B2P_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dual_binned<4, true>, kBlock, 0));
      int sms = 0;
      B2P_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
      const int64_t wave = static_cast<int64_t>(std::max(1, per_sm)) * sms * kBlock;
      const int rounds = opt.short_row_rounds > 0 ? opt.short_row_rounds : 2;
      binsA = device_bins(P.A, wave, opt.lanes_per_row_a, rounds);
      binsT = device_bins(P.AT, wave, opt.lanes_per_row_at, rounds);
      stats.lanes_per_row_a = binsA.g;
      stats.lanes_per_row_at = binsT.g;
      setup_resident(sms);
      stats.graph_seconds += seconds_since(tk);
    }
    mixed_batch = k > 1 && opt.precision == B2P_PRECISION_MIXED;
    stats.kernel_mode = (resident || mixed) ? B2P_KERNELS_RESIDENT : B2P_KERNELS_FUSED;
    stats.precision_used = (mixed || mixed_batch) ? B2P_PRECISION_MIXED : B2P_PRECISION_FP64;
    for (int s = 0; s < NSLOT; ++s) v[s] = dalloc<double>(row_slot(s) ? mk : nk);
    k_full = k;
    for (int s = 0; s < NSLOT; ++s) v_full[s] = v[s];
    case_of.resize(k);
    for (int b = 0; b < k; ++b) case_of[b] = b;
    d_case_map = dalloc<int32_t>(k);
    auto put = [&](int s, const std::vector<double>& h) {
      if (!h.empty())
        B2P_CUDA(cudaMemcpyAsync(v[s], h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
      bytes_up += static_cast<int64_t>(h.size() * sizeof(double));
    };
    put(C, c);
    put(LO, lo);
    put(UP, up);
    put(RL, rl);
    put(RU, ru);
    put(XINIT, x);
    x_cold = x;
    omega_cold = omega0;
    if (mk) B2P_CUDA(cudaMemsetAsync(v[YINIT], 0, mk * sizeof(double), stream));
    d_tau = dalloc<double>(k);
    d_sigma = dalloc<double>(k);
    d_it_base = dalloc<int64_t>(1);
    d_restart_at = dalloc<int64_t>(k);
    d_mask = dalloc<int32_t>(k);
    g_rows = red_blocks(m);
    g_cols = red_blocks(n);
    d_prow = dalloc<double>(static_cast<size_t>(k) * g_rows * kRowSums);
    d_pcol = dalloc<double>(static_cast<size_t>(k) * g_cols * kRowSums);
    d_sums = dalloc<double>(static_cast<size_t>(k) * kNumSums);
    h_sums = static_cast<double*>(PinnedCache::get(sizeof(double) * k * kNumSums));
    h_steps = static_cast<double*>(PinnedCache::get(sizeof(double) * 2 * k));
    h_mask = static_cast<int32_t*>(PinnedCache::get(sizeof(int32_t) * k));
    if (mixed || mixed_batch) setup_mixed();
    // AX = A x0 on the device (pdhg.cpp:540-545), kept as the restart point of every solve.
    if (m > 0) {
      k_spmv<<<blocks(static_cast<int64_t>(m) * k), kBlock, 0, stream>>>(m, k, viewA(), v[XINIT], v[AXINIT]);
      B2P_CUDA(cudaGetLastError());
    }
    tune_batch();
    B2P_CUDA(cudaStreamSynchronize(stream));
    transfer_seconds = seconds_since(tx);
    stats.upload_seconds = transfer_seconds;
    stats.setup_seconds = seconds_since(t0);
    stats.spectral_norm = P.normA;
  }

  // ||A||_2 estimate of powerIteration (src/pdhg/pdhg.cpp:404-422) with the
  // products on the device: A x and A^T y by CSR row sums in increasing column
  // order, which is exactly the addition order of SparseMatrix::multiply /
  // multiplyTranspose (src/core/sparse.cpp:67-82); the norm of z is summed on
  // the host in index order.  The result is bit-identical to the reference's.
  double device_power_iteration(int iters) {
    if (P.A.val.empty() || n == 0 || m == 0) return 1.0;
    double* dx = dalloc<double>(n);
    double* dy = dalloc<double>(m);
    double* dz = dalloc<double>(n);
    std::vector<double> hx(n, 1.0 / std::sqrt(static_cast<double>(n > 1 ? n : 1)));
    B2P_CUDA(cudaMemcpyAsync(dx, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream));
    double* hz = nullptr;
    hz = static_cast<double*>(PinnedCache::get(sizeof(double) * n));
    struct PinnedGuard {
      double* p;
      size_t bytes;
      ~PinnedGuard() { PinnedCache::put(p, bytes); }
    } guard{hz, sizeof(double) * n};
    double s = 1;
    for (int it = 0; it < iters; ++it) {
      k_spmv<<<blocks(m), kBlock, 0, stream>>>(m, 1, viewA(), dx, dy);
      k_spmv<<<blocks(n), kBlock, 0, stream>>>(n, 1, viewAT(), dy, dz);
      B2P_CUDA(cudaGetLastError());
      B2P_CUDA(cudaMemcpyAsync(hz, dz, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
      B2P_CUDA(cudaStreamSynchronize(stream));
      double nz = 0;
      for (int j = 0; j < n; ++j) nz += hz[j] * hz[j];
      nz = std::sqrt(nz);
      if (nz == 0) return 1.0;
      s = std::sqrt(nz);
      k_div_scalar<<<blocks(n), kBlock, 0, stream>>>(n, dz, nz, dx);
      B2P_CUDA(cudaGetLastError());
    }
    B2P_CUDA(cudaStreamSynchronize(stream));
    return s;
  }

  // Resident form if the LP's slices fit in shared memory, one block per SM
  // (FP64 for the plain form; FP32 too when the mixed form is requested).
  void setup_resident(int sms) {
    if (opt.kernel_mode == B2P_KERNELS_FUSED || n == 0 || m == 0) return;
    int optin = 0;
    B2P_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    const int nb = sms;
    std::vector<int32_t> cb = balanced_split(P.AT, nb), rb = balanced_split(P.A, nb);
    size_t need64 = 0, need32 = 0;
    for (int b = 0; b < nb; ++b) {
      const int nc = cb[b + 1] - cb[b], nr = rb[b + 1] - rb[b];
      const int tn = P.AT.ptr[cb[b + 1]] - P.AT.ptr[cb[b]], an = P.A.ptr[rb[b + 1]] - P.A.ptr[rb[b]];
      need64 = std::max(need64, resident_smem_bytes<double>(nc, nr, tn, an));
      need32 = std::max(need32, resident_smem_bytes<float>(nc, nr, tn, an));
    }
    const size_t reserve = 1024;  // static shared memory of the kernel
    res_gc = resident_lanes(P.AT, cb);
    res_gr = resident_lanes(P.A, rb);
    bool ok64 = need64 + reserve <= static_cast<size_t>(optin);
    bool ok32 = opt.precision == B2P_PRECISION_MIXED && need32 + reserve <= static_cast<size_t>(optin);
    if (ok64) {
      res_fn = resident_fn<double>(res_gc, res_gr);
      B2P_CUDA(cudaFuncSetAttribute(res_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(need64)));
      int per_sm = 0;
      B2P_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, res_fn, kResidentThreads, need64));
      ok64 = per_sm >= 1;
    }
    if (ok32) {
      res_fn32 = resident_fn<float>(res_gc, res_gr);
      B2P_CUDA(cudaFuncSetAttribute(res_fn32, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(need32)));
      int per_sm = 0;
      B2P_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, res_fn32, kResidentThreads, need32));
      ok32 = per_sm >= 1;
    }
    if (!ok64 && opt.kernel_mode == B2P_KERNELS_RESIDENT && !ok32)
      throw Error(B2P_ERR_TOO_LARGE, "LP does not fit the resident form (shared memory)");
    if (!ok64 && !ok32) return;
    d_cb = upload(cb);
    d_rb = upload(rb);
    d_sync = dalloc<unsigned>(4);
    d_rpartial = dalloc<double>(static_cast<size_t>(nb) * kNumSums);
    h_error = static_cast<int32_t*>(PinnedCache::get(sizeof(int32_t)));
    *h_error = 0;
    res_blocks = nb;
    res_smem = ok64 ? need64 : 0;
    res_smem32 = ok32 ? need32 : 0;
    resident = ok64;
    mixed = ok32;
    stats.resident_blocks = nb;
    stats.resident_smem_bytes = static_cast<int64_t>(ok64 ? need64 : need32);
  }

  // FP32 copies of the operators and case vectors for the mixed form.
  void setup_mixed() {
    // FP32 copies of the scaled operators, rounded to nearest on the device
    const int64_t nnz = static_cast<int64_t>(P.A.val.size());
    a_val32 = dalloc<float>(static_cast<size_t>(nnz));
    t_val32 = dalloc<float>(static_cast<size_t>(nnz));
    if (nnz) {
      k_convert<double, float><<<blocks(nnz), kBlock, 0, stream>>>(nnz, dA_val, a_val32);
      k_convert<double, float><<<blocks(nnz), kBlock, 0, stream>>>(nnz, dT_val, t_val32);
    }
    for (int q = 0; q < NSLOT32; ++q)
      v32[q] = dalloc<float>(static_cast<size_t>(q >= Y32 && q != C32 && q != LO32 && q != UP32 ? m : n) * k);
    const int src[5] = {C, LO, UP, RL, RU}, dst[5] = {C32, LO32, UP32, RL32, RU32};
    for (int q = 0; q < 5; ++q) {
      const int64_t len = static_cast<int64_t>(row_slot(src[q]) ? m : n) * k;
      if (len) k_convert<double, float><<<blocks(len), kBlock, 0, stream>>>(len, v[src[q]], v32[dst[q]]);
    }
    B2P_CUDA(cudaGetLastError());
  }

  template <class T>
  void launch_resident(int L, ResidentFn<T> fn, size_t smem, const T* a_val, const T* t_val, T* const* vs) {
    B2P_CUDA(cudaMemsetAsync(d_sync, 0, 4 * sizeof(unsigned), stream));
    ResidentArgs<T> ra{};
    ra.cb = d_cb;
    ra.rb = d_rb;
    ra.a_ptr = dA_ptr;
    ra.a_idx = dA_idx;
    ra.a_val = a_val;
    ra.t_ptr = dT_ptr;
    ra.t_idx = dT_idx;
    ra.t_val = t_val;
    ra.x = vs[0];
    ra.xp = vs[1];
    ra.x0 = vs[2];
    ra.y = vs[3];
    ra.yp = vs[4];
    ra.y0 = vs[5];
    ra.ax = vs[6];
    ra.ax0 = vs[7];
    ra.axp = vs[8];
    ra.c = vs[9];
    ra.lo = vs[10];
    ra.up = vs[11];
    ra.rl = vs[12];
    ra.ru = vs[13];
    ra.c64 = v[C];
    ra.lo64 = v[LO];
    ra.up64 = v[UP];
    ra.rl64 = v[RL];
    ra.ru64 = v[RU];
    ra.rfac = d_rfac;
    ra.cfac = d_cfac;
    ra.tau = d_tau;
    ra.sigma = d_sigma;
    ra.ck = IterClock{d_it_base, d_restart_at, 0};
    ra.rho = opt.reflection;
    ra.L = L;
    ra.g_cols = res_gc;
    ra.g_rows = res_gr;
    ra.lt_cols = 2 * kResUnroll * res_gc;
    ra.lt_rows = 2 * kResUnroll * res_gr;
    ra.arrive = d_sync;
    ra.gen = d_sync + 1;
    ra.error = reinterpret_cast<int32_t*>(d_sync + 2);
    ra.partial = d_rpartial;
    ra.sums = d_sums;
    ra.it_base = d_it_base;
    void* args[] = {&ra};
    if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[0], stream));
    B2P_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(fn), dim3(res_blocks), dim3(kResidentThreads), args,
                                         smem, stream));
    if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[1], stream));
    B2P_CUDA(cudaMemcpyAsync(h_sums, d_sums, sizeof(double) * kNumSums, cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaMemcpyAsync(h_error, ra.error, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
  }

  void launch_resident64(int L) {
    double* const vs[14] = {v[X], v[XP], v[X0], v[Y], v[YP], v[Y0], v[AX], v[AX0], v[AXP],
                            v[C], v[LO], v[UP], v[RL], v[RU]};
    launch_resident<double>(L, res_fn, res_smem, dA_val, dT_val, vs);
  }

  void launch_resident32(int L) {
    float* const vs[14] = {v32[X32], v32[XP32], v32[X032], v32[Y32], v32[YP32], v32[Y032], v32[AX32],
                           v32[AX032], v32[AXP32], v32[C32], v32[LO32], v32[UP32], v32[RL32], v32[RU32]};
    launch_resident<float>(L, res_fn32, res_smem32, a_val32, t_val32, vs);
  }

  // FP32 state from the FP64 state (start of the mixed form's FP32 phase).
  void state_to_fp32() {
    const int pairs[6][2] = {{X, X32}, {X0, X032}, {Y, Y32}, {Y0, Y032}, {AX, AX32}, {AX0, AX032}};
    for (auto& pr : pairs) {
      const int64_t len = static_cast<int64_t>(row_slot(pr[0]) ? m : n) * k;
      if (len) k_convert<double, float><<<blocks(len), kBlock, 0, stream>>>(len, v[pr[0]], v32[pr[1]]);
    }
    B2P_CUDA(cudaGetLastError());
  }

  // x+, y+ of the FP32 phase in FP64, and A x+ recomputed in FP64.
  void fp32_point_to_fp64() {
    const int64_t nk = static_cast<int64_t>(n) * k, mk = static_cast<int64_t>(m) * k;
    if (nk) k_convert<float, double><<<blocks(nk), kBlock, 0, stream>>>(nk, v32[XP32], v[XP]);
    if (mk) k_convert<float, double><<<blocks(mk), kBlock, 0, stream>>>(mk, v32[YP32], v[YP]);
    if (mk) k_spmv<<<blocks(mk), kBlock, 0, stream>>>(m, k, viewA(), v[XP], v[AXP]);
    B2P_CUDA(cudaGetLastError());
    launches += 3;
  }

  // FP64 check sums of the FP64 point (XP, YP, AXP) into h_sums (the movement
  // norms of this call are not meaningful).
  void verify_fp64() {
    if (n) k_spmv<<<blocks(static_cast<int64_t>(n) * k), kBlock, 0, stream>>>(n, k, viewAT(), v[YP], v[ATYP]);
    k_check_rows<<<dim3(g_rows, k), kBlock, 0, stream>>>(m, k, v[AXP], v[RL], v[RU], v[YP], v[Y], v[Y0], d_rfac,
                                                         d_prow);
    k_check_cols<<<dim3(g_cols, k), kBlock, 0, stream>>>(n, k, viewAT(), v[YP], v[ATYP], v[XP], v[X], v[X0], v[C],
                                                         v[LO], v[UP], d_cfac, d_pcol);
    k_check_finalize<<<k, kBlock, 0, stream>>>(k, g_rows, g_cols, d_prow, d_pcol, d_sums, d_it_base, 0);
    B2P_CUDA(cudaGetLastError());
    B2P_CUDA(cudaMemcpyAsync(h_sums, d_sums, sizeof(double) * k * kNumSums, cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaStreamSynchronize(stream));
    launches += 5;
  }

  // Continue in FP64 from the FP32 phase's x+, y+ as from a restart.
  void switch_to_fp64() {
    fp32_point_to_fp64();
    const int64_t nn = static_cast<int64_t>(n) * k, mm = static_cast<int64_t>(m) * k;
    if (nn) {
      B2P_CUDA(cudaMemcpyAsync(v[X], v[XP], sizeof(double) * nn, cudaMemcpyDeviceToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(v[X0], v[XP], sizeof(double) * nn, cudaMemcpyDeviceToDevice, stream));
    }
    if (mm) {
      B2P_CUDA(cudaMemcpyAsync(v[Y], v[YP], sizeof(double) * mm, cudaMemcpyDeviceToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(v[Y0], v[YP], sizeof(double) * mm, cudaMemcpyDeviceToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(v[AX], v[AXP], sizeof(double) * mm, cudaMemcpyDeviceToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(v[AX0], v[AXP], sizeof(double) * mm, cudaMemcpyDeviceToDevice, stream));
    }
    k_restart_clock<<<(k + 127) / 128, 128, 0, stream>>>(k, d_it_base, d_restart_at);
    B2P_CUDA(cudaGetLastError());
    ++launches;
    phase32 = false;
  }

  RowBins device_bins(const HostCsr& M, int64_t wave, int g_override, int rounds) {
    HostBins hb = make_bins(M, wave, g_override, rounds);
    RowBins b{};
    b.long_rows = upload(hb.long_rows);
    b.vlong_rows = upload(hb.vlong_rows);
    b.short_rows = nullptr;
    b.n_short = 0;
    b.n_long = static_cast<int32_t>(hb.long_rows.size());
    b.n_vlong = static_cast<int32_t>(hb.vlong_rows.size());
    b.long_thr = hb.long_thr;
    b.vlong_blocks = b.n_vlong;
    b.long_blocks = (b.n_long + kBlock / 32 - 1) / (kBlock / 32);
    b.short_blocks = static_cast<int32_t>((static_cast<int64_t>(M.rows) * hb.g + kBlock - 1) / kBlock);
    b.g = hb.g;
    return b;
  }
  static unsigned bin_grid(const RowBins& b) {
    return static_cast<unsigned>(std::max(1, b.vlong_blocks + b.long_blocks + b.short_blocks));
  }

  void reset_state(std::vector<double>& omega) {
    const size_t nk = static_cast<size_t>(n) * k, mk = static_cast<size_t>(m) * k;
    auto cp = [&](int dst, int src, size_t len) {
      if (len) B2P_CUDA(cudaMemcpyAsync(v[dst], v[src], len * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    };
    cp(X, XINIT, nk);
    cp(X0, XINIT, nk);
    cp(AX, AXINIT, mk);
    cp(AX0, AXINIT, mk);
    cp(Y, YINIT, mk);
    cp(Y0, YINIT, mk);
    if (mk) {
      B2P_CUDA(cudaMemsetAsync(v[YP], 0, mk * sizeof(double), stream));
      B2P_CUDA(cudaMemsetAsync(v[AXP], 0, mk * sizeof(double), stream));
    }
    if (nk) B2P_CUDA(cudaMemsetAsync(v[XP], 0, nk * sizeof(double), stream));
    B2P_CUDA(cudaMemsetAsync(d_it_base, 0, sizeof(int64_t), stream));
    B2P_CUDA(cudaMemsetAsync(d_restart_at, 0, sizeof(int64_t) * k, stream));
    omega = omega0;
    upload_steps(omega);
  }

  // Starting point of the next solves, in the original space (case-major
  // k x n, k x m): x is scaled and projected onto the bounds, y scaled, A x
  // recomputed; NULL x and y restore the reference's cold start.
  void set_start(const double* x, const double* y, double primal_weight) {
    B2P_CUDA(cudaSetDevice(device));
    const size_t nk = static_cast<size_t>(n) * k, mk = static_cast<size_t>(m) * k;
    std::vector<double> lo(nk), up(nk);
    if (nk) {
      B2P_CUDA(cudaMemcpyAsync(lo.data(), v[LO], nk * sizeof(double), cudaMemcpyDeviceToHost, stream));
      B2P_CUDA(cudaMemcpyAsync(up.data(), v[UP], nk * sizeof(double), cudaMemcpyDeviceToHost, stream));
      B2P_CUDA(cudaStreamSynchronize(stream));
    }
    std::vector<double> xs(x_cold), ys(mk, 0.0);
    warm = x || y;
    if (x)
      for (int b = 0; b < k; ++b)
        for (int j = 0; j < n; ++j) {
          const size_t t = static_cast<size_t>(j) * k + b;
          xs[t] = smin(smax(x[static_cast<size_t>(b) * n + j] / P.Cs[j] / P.beta, lo[t]), up[t]);
        }
    if (y)
      for (int b = 0; b < k; ++b)
        for (int i = 0; i < m; ++i)
          ys[static_cast<size_t>(i) * k + b] = y[static_cast<size_t>(b) * m + i] / P.R[i] / P.gamma;
    if (nk) B2P_CUDA(cudaMemcpyAsync(v[XINIT], xs.data(), nk * sizeof(double), cudaMemcpyHostToDevice, stream));
    if (mk) {
      B2P_CUDA(cudaMemcpyAsync(v[YINIT], ys.data(), mk * sizeof(double), cudaMemcpyHostToDevice, stream));
      k_spmv<<<blocks(static_cast<int64_t>(m) * k), kBlock, 0, stream>>>(m, k, viewA(), v[XINIT], v[AXINIT]);
      B2P_CUDA(cudaGetLastError());
    }
    B2P_CUDA(cudaStreamSynchronize(stream));
    bytes_up += static_cast<int64_t>((nk + mk) * sizeof(double));
    omega0 = omega_cold;
    if (primal_weight > 0) omega0.assign(k, primal_weight);
  }

  void upload_steps(const std::vector<double>& omega) {
    for (int b = 0; b < k; ++b) {
      h_steps[b] = eta / omega[b];
      h_steps[k + b] = eta * omega[b];
    }
    B2P_CUDA(cudaMemcpyAsync(d_tau, h_steps, sizeof(double) * k, cudaMemcpyHostToDevice, stream));
    B2P_CUDA(cudaMemcpyAsync(d_sigma, h_steps + k, sizeof(double) * k, cudaMemcpyHostToDevice, stream));
    bytes_up += static_cast<int64_t>(2 * k * sizeof(double));
  }

  void ensure_prof_events(int L) {
    const size_t need = static_cast<size_t>(4) * L;
    while (prof_ev.size() < need) {
      cudaEvent_t e;
      B2P_CUDA(cudaEventCreate(&e));
      prof_ev.push_back(e);
    }
  }

  // One LP: binned fused kernels with programmatic dependent launch.
  void enqueue_interval_single(int L) {
    const double rho = opt.reflection;
    const CsrView A = viewA(), AT = viewAT();
    const unsigned gp = bin_grid(binsT), gd = bin_grid(binsA);
    for (int l = 0; l < L; ++l) {
      const bool last = l == L - 1;
      const IterClock ck{d_it_base, d_restart_at, l};
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 0], stream));
      if (n) {
#define B2P_PRIMAL(G)                                                                                     \
  if (last)                                                                                               \
    launch(k_primal_binned<G, false>, gp, stream, true, AT, binsT, v[Y], v[C], v[LO], v[UP], v[X], v[XP], v[X0], \
           d_tau, ck, rho, InstanceMap{nullptr, nullptr});                                                \
  else                                                                                                    \
    launch(k_primal_binned<G, true>, gp, stream, true, AT, binsT, v[Y], v[C], v[LO], v[UP], v[X], v[XP], v[X0],  \
           d_tau, ck, rho, InstanceMap{nullptr, nullptr});
        B2P_G_SWITCH(binsT.g, B2P_PRIMAL)
#undef B2P_PRIMAL
      }
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 1], stream));
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 2], stream));
      if (m) {
#define B2P_DUAL(G)                                                                                        \
  if (last)                                                                                                \
    launch(k_dual_binned<G, false>, gd, stream, true, A, binsA, v[XP], v[RL], v[RU], v[Y], v[YP], v[Y0], v[AX], \
           v[AXP], v[AX0], d_sigma, ck, rho, InstanceMap{nullptr, nullptr});                               \
  else                                                                                                     \
    launch(k_dual_binned<G, true>, gd, stream, true, A, binsA, v[XP], v[RL], v[RU], v[Y], v[YP], v[Y0], v[AX],  \
           v[AXP], v[AX0], d_sigma, ck, rho, InstanceMap{nullptr, nullptr});
        B2P_G_SWITCH(binsA.g, B2P_DUAL)
#undef B2P_DUAL
      }
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 3], stream));
    }
    // A^T y+ for the dual residual, then the check reductions.
    if (n) {
#define B2P_ATY(G) launch(k_spmv_binned<G>, gp, stream, false, AT, binsT, v[YP], v[ATYP], InstanceMap{nullptr, nullptr});
      B2P_G_SWITCH(binsT.g, B2P_ATY)
#undef B2P_ATY
    }
    enqueue_check_tail(L, v[ATYP]);
  }

  void enqueue_check_tail(int L, const double* atyp) {
    const double rho = opt.reflection;
    const int64_t nk = static_cast<int64_t>(n) * k, mk = static_cast<int64_t>(m) * k;
    const IterClock ck{d_it_base, d_restart_at, L - 1};
    k_check_rows<<<dim3(g_rows, k), kBlock, 0, stream>>>(m, k, v[AXP], v[RL], v[RU], v[YP], v[Y], v[Y0], d_rfac,
                                                         d_prow);
    k_check_cols<<<dim3(g_cols, k), kBlock, 0, stream>>>(n, k, viewAT(), v[YP], atyp, v[XP], v[X], v[X0], v[C],
                                                         v[LO], v[UP], d_cfac, d_pcol);
    k_halpern_all<<<blocks(nk + mk), kBlock, 0, stream>>>(n, m, k, v[X], v[XP], v[X0], v[Y], v[YP], v[Y0], v[AX],
                                                         v[AXP], v[AX0], ck, rho);
    k_check_finalize<<<k, kBlock, 0, stream>>>(k, g_rows, g_cols, d_prow, d_pcol, d_sums, d_it_base, L);
    B2P_CUDA(cudaGetLastError());
    B2P_CUDA(cudaMemcpyAsync(h_sums, d_sums, sizeof(double) * k * kNumSums, cudaMemcpyDeviceToHost, stream));
  }

  // Calls f with the compile-time form of a batch kernel variant: Halpern
  // step, streamed vectors, cases per thread, whole warps per row, tile rows.
  template <class F>
  static void batch_dispatch(bool h, bool st, int cpt, bool wr, int tr, F&& f) {
    using std::false_type;
    using std::integral_constant;
    using std::true_type;
    auto d4 = [&](auto H, auto ST, auto CP, auto WR) {
      if (tr == 16) f(H, ST, CP, WR, integral_constant<int, 16>{});
      else if (tr == 8) f(H, ST, CP, WR, integral_constant<int, 8>{});
      else if (tr == 4) f(H, ST, CP, WR, integral_constant<int, 4>{});
      else f(H, ST, CP, WR, integral_constant<int, 0>{});
    };
    auto d3 = [&](auto H, auto ST, auto CP) {
      if (wr) d4(H, ST, CP, true_type{});
      else d4(H, ST, CP, false_type{});
    };
    auto d2 = [&](auto H, auto ST) {
      if (cpt == 2) d3(H, ST, integral_constant<int, 2>{});
      else d3(H, ST, integral_constant<int, 1>{});
    };
    auto d1 = [&](auto H) {
      if (st) d2(H, true_type{});
      else d2(H, false_type{});
    };
    if (h) d1(true_type{});
    else d1(false_type{});
  }

  // Grid of a batch kernel over `rows` rows (layouts in pdhg_kernels.cuh).
  unsigned batch_grid(int64_t rows, int cpt, int tr) const {
    const int64_t kh = (k + cpt - 1) / cpt;
    if (tr == 0) return blocks(rows * kh);
    return static_cast<unsigned>(std::max<int64_t>(1, ((rows + tr - 1) / tr) * ((kh + 31) / 32)));
  }

  // FP64 batch kernels (k > 1) of one iteration.
  void enqueue_batch_primal(bool halpern, bool streamed, const IterClock& ck, int cpt, bool wr, int tr) {
    const double rho = opt.reflection;
    const unsigned grid = batch_grid(n, cpt, tr), block = batch_block(tr);
    const CsrView AT = viewAT();
    batch_dispatch(halpern, streamed, cpt, wr, tr, [&](auto H, auto ST, auto CP, auto WR, auto TR) {
      launch_nt(k_primal<decltype(H)::value, decltype(ST)::value, decltype(CP)::value, decltype(WR)::value,
                         decltype(TR)::value>,
                grid, block, stream, true, n, k, AT, v[Y], v[C], v[LO], v[UP], v[X], v[XP], v[X0], d_tau, ck, rho);
    });
  }
  void enqueue_batch_dual(bool halpern, bool streamed, const IterClock& ck, int cpt, bool wr, int tr) {
    const double rho = opt.reflection;
    const unsigned grid = batch_grid(m, cpt, tr), block = batch_block(tr);
    const CsrView A = viewA();
    batch_dispatch(halpern, streamed, cpt, wr, tr, [&](auto H, auto ST, auto CP, auto WR, auto TR) {
      launch_nt(k_dual<decltype(H)::value, decltype(ST)::value, decltype(CP)::value, decltype(WR)::value,
                       decltype(TR)::value>,
                grid, block, stream, true, m, k, A, v[XP], v[RL], v[RU], v[Y], v[YP], v[Y0], v[AX], v[AXP], v[AX0],
                d_sigma, ck, rho);
    });
  }

  // Row tiles of the batch kernels' layouts (0 = one row's cases per block).
  static constexpr int kTileRows[4] = {0, 4, 8, 16};

  // FP64 batch kernel variants: forced by the options, or, for batches whose
  // vectors far exceed L2 (k (m + n) >= 2^22 elements), each kernel is timed
  // with one and with two cases per thread, with and (when k / cases per
  // thread is a multiple of 32) without per-lane index loads, with cached and
  // with evict-first streamed vectors, in the row-per-block layout and the
  // row-tiled ones of 4, 8 and 16 rows (one warm-up, three timed launches
  // each, from the starting state), and the fastest is kept per kernel.
  void tune_batch() {
    if (opt.batch_variant < 0 || opt.batch_variant > 32) throw Error(B2P_ERR_INVALID, "batch_variant must be 0..32");
    if (k <= 1 || mixed_batch) return;
    if (opt.batch_variant > 0) {
      const int w = (opt.batch_variant - 1) % 8 + 1;  // the layout-free part, 1..8
      const int v0 = (w - 1) % 4 + 1;
      batch_cpt_p = batch_cpt_d = (v0 == 2 || v0 == 4) ? 2 : 1;
      batch_stream_p = batch_stream_d = v0 >= 3;
      batch_wr_p = batch_wr_d = w > 4 && warp_rows(batch_cpt_p);
      batch_tr_p = batch_tr_d = kTileRows[(opt.batch_variant - 1) / 8];
    } else if (static_cast<int64_t>(n + m) * k >= (int64_t(1) << 22)) {
      time_batch_variants();
    }
    stats.streaming_at = batch_stream_p;
    stats.streaming_a = batch_stream_d;
    stats.cases_per_thread_at = batch_cpt_p;
    stats.cases_per_thread_a = batch_cpt_d;
    stats.warp_rows_at = batch_wr_p;
    stats.warp_rows_a = batch_wr_d;
    stats.tile_rows_at = batch_tr_p;
    stats.tile_rows_a = batch_tr_d;
  }

  // Whole warps per row: k / cpt (rounded up) a multiple of 32.
  bool warp_rows(int cpt) const { return ((k + cpt - 1) / cpt) % 32 == 0; }

  void time_batch_variants() {
    const auto t0 = Clock::now();
    std::vector<double> omega;
    reset_state(omega);
    cudaEvent_t e0, e1;
    B2P_CUDA(cudaEventCreate(&e0));
    B2P_CUDA(cudaEventCreate(&e1));
    const IterClock ck{d_it_base, d_restart_at, 0};
    auto timed = [&](auto&& enq) {
      enq();
      B2P_CUDA(cudaEventRecord(e0, stream));
      for (int r = 0; r < 3; ++r) enq();
      B2P_CUDA(cudaEventRecord(e1, stream));
      B2P_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      B2P_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      return static_cast<double>(ms);
    };
    double best_p = INFINITY, best_d = INFINITY;
    for (const int tr : kTileRows)
      for (const int cpt : {1, 2})
        for (int wr = 0; wr < 2; ++wr) {
          if (wr && !warp_rows(cpt)) continue;
          for (int st = 0; st < 2; ++st) {
            if (n) {
              const double t = timed([&] { enqueue_batch_primal(true, st != 0, ck, cpt, wr != 0, tr); });
              if (t < best_p)
                best_p = t, batch_stream_p = st != 0, batch_cpt_p = cpt, batch_wr_p = wr != 0, batch_tr_p = tr;
            }
            if (m) {
              const double t = timed([&] { enqueue_batch_dual(true, st != 0, ck, cpt, wr != 0, tr); });
              if (t < best_d)
                best_d = t, batch_stream_d = st != 0, batch_cpt_d = cpt, batch_wr_d = wr != 0, batch_tr_d = tr;
            }
          }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    stats.autotune_seconds = seconds_since(t0);
  }

  // Enqueues one check interval of L iterations on the stream (captured or not).
  void enqueue_interval(int L) {
    if (k == 1) {
      enqueue_interval_single(L);
      return;
    }
    const int64_t nk = static_cast<int64_t>(n) * k, mk = static_cast<int64_t>(m) * k;
    for (int l = 0; l < L; ++l) {
      const bool last = l == L - 1;
      const IterClock ck{d_it_base, d_restart_at, l};
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 0], stream));
      if (nk) enqueue_batch_primal(!last, batch_stream_p, ck, batch_cpt_p, batch_wr_p, batch_tr_p);
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 1], stream));
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 2], stream));
      if (mk) enqueue_batch_dual(!last, batch_stream_d, ck, batch_cpt_d, batch_wr_d, batch_tr_d);
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 3], stream));
      B2P_CUDA(cudaGetLastError());
    }
    enqueue_check_tail(L, nullptr);
  }

  CsrView32 viewA32() const { return CsrView32{dA_ptr, dA_idx, a_val32, m}; }
  CsrView32 viewAT32() const { return CsrView32{dT_ptr, dT_idx, t_val32, n}; }

  // One check interval of the FP32 phase of a batch (mixed form, k > 1).
  void enqueue_interval32(int L) {
    const double rho = opt.reflection;
    const int64_t nk = static_cast<int64_t>(n) * k, mk = static_cast<int64_t>(m) * k;
    const unsigned gp = blocks(nk), gd = blocks(mk);
    const CsrView32 A = viewA32(), AT = viewAT32();
    float* const* w = v32;
    for (int l = 0; l < L; ++l) {
      const bool last = l == L - 1;
      const IterClock ck{d_it_base, d_restart_at, l};
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 0], stream));
      if (nk) {
        if (last)
          launch(k_primal32<false>, gp, stream, true, n, k, AT, w[Y32], w[C32], w[LO32], w[UP32], w[X32], w[XP32],
                 w[X032], d_tau, ck, rho);
        else
          launch(k_primal32<true>, gp, stream, true, n, k, AT, w[Y32], w[C32], w[LO32], w[UP32], w[X32], w[XP32],
                 w[X032], d_tau, ck, rho);
      }
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 1], stream));
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 2], stream));
      if (mk) {
        if (last)
          launch(k_dual32<false>, gd, stream, true, m, k, A, w[XP32], w[RL32], w[RU32], w[Y32], w[YP32], w[Y032],
                 w[AX32], w[AXP32], w[AX032], d_sigma, ck, rho);
        else
          launch(k_dual32<true>, gd, stream, true, m, k, A, w[XP32], w[RL32], w[RU32], w[Y32], w[YP32], w[Y032],
                 w[AX32], w[AXP32], w[AX032], d_sigma, ck, rho);
      }
      if (profiling) B2P_CUDA(cudaEventRecord(prof_ev[4 * l + 3], stream));
      B2P_CUDA(cudaGetLastError());
    }
    const IterClock ck{d_it_base, d_restart_at, L - 1};
    k_check_rows32<<<dim3(g_rows, k), kBlock, 0, stream>>>(m, k, w[AXP32], v[RL], v[RU], w[YP32], w[Y32], w[Y032],
                                                           d_rfac, d_prow);
    k_check_cols32<<<dim3(g_cols, k), kBlock, 0, stream>>>(n, k, AT, w[YP32], w[XP32], w[X32], w[X032], v[C], v[LO],
                                                           v[UP], d_cfac, d_pcol);
    k_halpern_all32<<<blocks(nk + mk), kBlock, 0, stream>>>(n, m, k, w[X32], w[XP32], w[X032], w[Y32], w[YP32],
                                                           w[Y032], w[AX32], w[AXP32], w[AX032], ck, rho);
    k_check_finalize<<<k, kBlock, 0, stream>>>(k, g_rows, g_cols, d_prow, d_pcol, d_sums, d_it_base, L);
    B2P_CUDA(cudaGetLastError());
    B2P_CUDA(cudaMemcpyAsync(h_sums, d_sums, sizeof(double) * k * kNumSums, cudaMemcpyDeviceToHost, stream));
  }

  int64_t launches_per_interval(int L) const {
    return static_cast<int64_t>(L) * ((n ? 1 : 0) + (m ? 1 : 0)) + 4 + (k == 1 && n ? 1 : 0);
  }

  void run_interval(int L) {
    if (profiling) ensure_prof_events(L);
    if ((phase32 && !mixed_batch) || resident) {
      if (phase32)
        launch_resident32(L);
      else
        launch_resident64(L);
      launches += 1;
      bytes_down += static_cast<int64_t>(sizeof(double) * kNumSums + sizeof(int32_t));
      return;
    }
    const bool fp32 = phase32 && mixed_batch;
    auto& gexec = fp32 ? graphs32 : graphs;
    auto& gdefs = fp32 ? graph_defs32 : graph_defs;
    if (opt.use_graphs && !profiling) {
      auto it = gexec.find(L);
      if (it == gexec.end()) {
        const auto tg = Clock::now();
        cudaGraph_t g;
        B2P_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
          if (fp32) enqueue_interval32(L);
          else enqueue_interval(L);
        } catch (...) {
          cudaStreamEndCapture(stream, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        B2P_CUDA(cudaStreamEndCapture(stream, &g));
        cudaGraphExec_t ge;
        B2P_CUDA(cudaGraphInstantiate(&ge, g, 0));
        gdefs[L] = g;
        it = gexec.emplace(L, ge).first;
        stats.graph_seconds += seconds_since(tg);
      }
      B2P_CUDA(cudaGraphLaunch(it->second, stream));
    } else if (fp32) {
      enqueue_interval32(L);
    } else {
      enqueue_interval(L);
    }
    launches += launches_per_interval(L);
    bytes_down += static_cast<int64_t>(sizeof(double) * k * kNumSums);
  }

  void collect_profile(int L) {
    if (!profiling) return;
    if (phase32 && mixed_batch) {  // the FP32 batch kernels: classes 3 and 4
      for (int l = 0; l < L; ++l) {
        float ms = 0;
        if (n) {
          B2P_CUDA(cudaEventElapsedTime(&ms, prof_ev[4 * l], prof_ev[4 * l + 1]));
          prof_ms[3] += ms;
          prof_launches[3]++;
        }
        if (m) {
          B2P_CUDA(cudaEventElapsedTime(&ms, prof_ev[4 * l + 2], prof_ev[4 * l + 3]));
          prof_ms[4] += ms;
          prof_launches[4]++;
        }
      }
      return;
    }
    if (phase32 || resident) {
      float ms = 0;
      B2P_CUDA(cudaEventElapsedTime(&ms, prof_ev[0], prof_ev[1]));
      prof_ms[2] += ms;
      prof_launches[2] += L;
      return;
    }
    for (int l = 0; l < L; ++l) {
      float ms = 0;
      if (n) {
        B2P_CUDA(cudaEventElapsedTime(&ms, prof_ev[4 * l], prof_ev[4 * l + 1]));
        prof_ms[0] += ms;
        prof_launches[0]++;
      }
      if (m) {
        B2P_CUDA(cudaEventElapsedTime(&ms, prof_ev[4 * l + 2], prof_ev[4 * l + 3]));
        prof_ms[1] += ms;
        prof_launches[1]++;
      }
    }
  }

  void download_iterates(std::vector<double>& xs, std::vector<double>& ys) {
    const auto t0 = Clock::now();
    xs.resize(static_cast<size_t>(n) * k);
    ys.resize(static_cast<size_t>(m) * k);
    if (!xs.empty())
      B2P_CUDA(cudaMemcpyAsync(xs.data(), v[XP], xs.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (!ys.empty())
      B2P_CUDA(cudaMemcpyAsync(ys.data(), v[YP], ys.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaStreamSynchronize(stream));
    bytes_down += static_cast<int64_t>((xs.size() + ys.size()) * sizeof(double));
    transfer_seconds += seconds_since(t0);
  }

  void drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    for (auto& g : graph_defs) cudaGraphDestroy(g.second);
    graphs.clear();
    graph_defs.clear();
  }

  // Keeps the packed cases keep[0..k2) (ascending, k2 >= 2): every vector slot
  // re-interleaved k -> k2 into new buffers, the restart clocks re-indexed;
  // each kept case's state is moved unchanged, so its iterates are those it
  // would have had.  Graphs are recaptured for the new width.
  void compact_cases(const std::vector<int32_t>& keep) {
    const int k2 = static_cast<int>(keep.size());
    B2P_CUDA(cudaMemcpyAsync(d_case_map, keep.data(), sizeof(int32_t) * k2, cudaMemcpyHostToDevice, stream));
    double* nv[NSLOT];
    for (int q = 0; q < NSLOT; ++q) {
      const int64_t rows = row_slot(q) ? m : n;
      void* p = nullptr;
      B2P_CUDA(cudaMallocFromPoolAsync(&p, std::max<int64_t>(rows * k2, 1) * sizeof(double), device_pool(device),
                                       stream));
      nv[q] = static_cast<double*>(p);
      if (rows) k_pack_cases<<<blocks(rows * k2), kBlock, 0, stream>>>(rows, k, k2, d_case_map, v[q], nv[q]);
    }
    B2P_CUDA(cudaGetLastError());
    std::vector<int64_t> ra(k), rb(k2);
    B2P_CUDA(cudaMemcpyAsync(ra.data(), d_restart_at, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaStreamSynchronize(stream));
    for (int q = 0; q < k2; ++q) rb[q] = ra[keep[q]];
    B2P_CUDA(cudaMemcpyAsync(d_restart_at, rb.data(), sizeof(int64_t) * k2, cudaMemcpyHostToDevice, stream));
    if (v[0] != v_full[0])
      for (int q = 0; q < NSLOT; ++q) B2P_CUDA(cudaFreeAsync(v[q], stream));
    for (int q = 0; q < NSLOT; ++q) v[q] = nv[q];
    std::vector<int32_t> co(k2);
    for (int q = 0; q < k2; ++q) co[q] = case_of[keep[q]];
    case_of = co;
    k = k2;
    // whole-warp rows need k / (cases per thread) to be a multiple of 32
    if (batch_wr_p && ((k + batch_cpt_p - 1) / batch_cpt_p) % 32 != 0) batch_wr_p = false;
    if (batch_wr_d && ((k + batch_cpt_d - 1) / batch_cpt_d) % 32 != 0) batch_wr_d = false;
    drop_graphs();
    ++compactions;
    B2P_CUDA(cudaStreamSynchronize(stream));
  }

  // Back to the engine's own buffers and width (after a solve that compacted).
  void restore_cases() {
    if (k == k_full && v[0] == v_full[0]) return;
    B2P_CUDA(cudaStreamSynchronize(stream));
    for (int q = 0; q < NSLOT; ++q) {
      if (v[q] != v_full[q]) B2P_CUDA(cudaFreeAsync(v[q], stream));
      v[q] = v_full[q];
    }
    k = k_full;
    case_of.resize(k);
    for (int b = 0; b < k; ++b) case_of[b] = b;
    batch_wr_p = batch_wr_p_full;
    batch_wr_d = batch_wr_d_full;
    drop_graphs();
    B2P_CUDA(cudaStreamSynchronize(stream));
  }

  // runPdhg's loop (src/pdhg/pdhg.cpp:560-687).
  void solve(Clock::time_point deadline_start) {
    B2P_CUDA(cudaSetDevice(device));
    restore_cases();
    batch_wr_p_full = batch_wr_p;
    batch_wr_d_full = batch_wr_d;
    compactions = 0;
    std::vector<double> cn(cNorm), rn(rhsNorm);  // per packed case
    const auto t_solve = Clock::now();
    std::vector<double> omega;
    launches = 0;
    for (int c = 0; c < 5; ++c) {
      prof_launches[c] = 0;
      prof_ms[c] = 0;
    }
    reset_state(omega);
    phase32 = mixed || mixed_batch;
    if (phase32) state_to_fp32();
    // mixed batch: per case, reached the tolerance in FP32 / stalled there
    std::vector<char> conv32(k, 0), stall32(k, 0);
    std::vector<double> best32v(k, INFINITY);
    std::vector<int> stale32v(k, 0);
    stats.fp32_iterations = 0;
    double best32 = INFINITY;  // mixed form: best FP32-phase KKT and checks since it improved
    int stale32 = 0;
    constexpr int kStallChecks = 20;
    results.assign(k, b2p_result{});
    x_out.assign(static_cast<size_t>(n) * k, 0.0);
    y_out.assign(static_cast<size_t>(m) * k, 0.0);
    stats.restarts = 0;
    std::vector<char> done(k, 0);
    std::vector<RestartTracker> restarts(k);
    std::vector<double> xs, ys;
    int remaining = k;
    int checks = 0;
    const double scaleObj = P.beta * P.gamma;
    const int cE = opt.check_every;
    auto expired = [&]() {
      if (opt.cancel_flag && *opt.cancel_flag) return true;
      return opt.time_limit > 0 && seconds_since(deadline_start) >= opt.time_limit;
    };
    auto extract = [&](int b, int status, double relKkt, double pobj, double dobj, int64_t it) {
      const size_t cb = static_cast<size_t>(case_of[b]);
      for (int j = 0; j < n; ++j) x_out[cb * n + j] = xs[static_cast<size_t>(j) * k + b] * P.Cs[j] * P.beta;
      for (int i = 0; i < m; ++i) y_out[cb * m + i] = ys[static_cast<size_t>(i) * k + b] * P.R[i] * P.gamma;
      b2p_result& r = results[cb];
      r.status = status;
      r.iterations = it;
      r.relative_kkt = relKkt;
      r.objective = pobj + P.offset;
      r.dual_objective = dobj + P.offset;
    };

    B2P_CUDA(cudaEventRecord(ev_start, stream));
    int64_t it = 0;
    bool expiredStop = false;
    while (it < opt.max_iterations) {
      const int L = static_cast<int>(std::min<int64_t>(cE, opt.max_iterations - it));
      run_interval(L);
      B2P_CUDA(cudaStreamSynchronize(stream));
      if ((resident || (phase32 && !mixed_batch)) && *h_error)
        throw Error(B2P_ERR_CUDA, "resident kernel: grid barrier timed out (kernel left the interval)");
      collect_profile(L);
      if (phase32) stats.fp32_iterations += L;
      it += L - 1;  // index of the check iteration
      ++checks;
      bool anyRestart = false, fetched = false;
      for (int b = 0; b < k; ++b) h_mask[b] = 0;
      if (phase32 && mixed_batch) {
        // Mixed form of a batch: each case's FP32 point is measured in FP64
        // arithmetic against the FP64 data; when every live case has met the
        // tolerance there or stalled (no 10% gain in kStallChecks checks),
        // the whole batch is re-measured from its FP64 point: cases that
        // pass terminate, the others continue in FP64 from that point as
        // from a restart.
        bool ready = true;
        for (int b = 0; b < k; ++b) {
          if (done[b]) continue;
          const double* s = h_sums + static_cast<size_t>(b) * kNumSums;
          const double pobj = s[CS_POBJ] * scaleObj, dobj = (s[CS_ROW_DOBJ] + s[CS_COL_DOBJ]) * scaleObj;
          const double relP = std::sqrt(s[CS_ROW_RES2]) / (1.0 + rn[b]);
          const double relD = std::sqrt(s[CS_COL_RES2]) / (1.0 + cn[b]);
          const double gap = std::fabs(pobj - dobj) / (1.0 + std::fabs(pobj) + std::fabs(dobj));
          const double kkt32 = smax(relP, smax(relD, gap));
          if (relP <= opt.tolerance && relD <= opt.tolerance && gap <= opt.tolerance) {
            conv32[b] = 1;
          } else if (kkt32 < 0.9 * best32v[b]) {
            best32v[b] = kkt32;
            stale32v[b] = 0;
          } else if (++stale32v[b] >= kStallChecks) {
            stall32[b] = 1;
          }
          if (!conv32[b] && !stall32[b]) ready = false;
        }
        if (ready) {
          fp32_point_to_fp64();
          verify_fp64();
          bool fetched64 = false;
          for (int b = 0; b < k; ++b) {
            if (done[b]) continue;
            const double* s = h_sums + static_cast<size_t>(b) * kNumSums;
            const double pobj = s[CS_POBJ] * scaleObj, dobj = (s[CS_ROW_DOBJ] + s[CS_COL_DOBJ]) * scaleObj;
            const double relP = std::sqrt(s[CS_ROW_RES2]) / (1.0 + rn[b]);
            const double relD = std::sqrt(s[CS_COL_RES2]) / (1.0 + cn[b]);
            const double gap = std::fabs(pobj - dobj) / (1.0 + std::fabs(pobj) + std::fabs(dobj));
            if (relP <= opt.tolerance && relD <= opt.tolerance && gap <= opt.tolerance) {
              if (!fetched64) {
                download_iterates(xs, ys);
                fetched64 = true;
              }
              extract(b, B2P_STATUS_OPTIMAL, smax(relP, smax(relD, gap)), pobj, dobj, it);
              done[b] = 1;
              --remaining;
            }
          }
          if (remaining == 0) break;
          switch_to_fp64();
          for (auto& r : restarts) r.reset();
          stats.restarts++;
          if (expired()) {
            expiredStop = true;
            break;
          }
          ++it;
          continue;
        }
      }
      if (phase32 && !mixed_batch) {
        // Mixed form (k == 1): an FP32 point that meets the tolerance is
        // re-measured in FP64; failing that, or after kStallChecks checks
        // without a 10% gain, the solve continues in FP64 from this point.
        const double* s = h_sums;
        const double pobj = s[CS_POBJ] * scaleObj, dobj = (s[CS_ROW_DOBJ] + s[CS_COL_DOBJ]) * scaleObj;
        const double relP = std::sqrt(s[CS_ROW_RES2]) / (1.0 + rn[0]);
        const double relD = std::sqrt(s[CS_COL_RES2]) / (1.0 + cn[0]);
        const double gap = std::fabs(pobj - dobj) / (1.0 + std::fabs(pobj) + std::fabs(dobj));
        const double kkt32 = smax(relP, smax(relD, gap));
        bool to_fp64 = false;
        if (relP <= opt.tolerance && relD <= opt.tolerance && gap <= opt.tolerance) {
          fp32_point_to_fp64();
          verify_fp64();
          const double vpobj = h_sums[CS_POBJ] * scaleObj;
          const double vdobj = (h_sums[CS_ROW_DOBJ] + h_sums[CS_COL_DOBJ]) * scaleObj;
          const double vrelP = std::sqrt(h_sums[CS_ROW_RES2]) / (1.0 + rn[0]);
          const double vrelD = std::sqrt(h_sums[CS_COL_RES2]) / (1.0 + cn[0]);
          const double vgap = std::fabs(vpobj - vdobj) / (1.0 + std::fabs(vpobj) + std::fabs(vdobj));
          stats.primal_residual = vrelP;
          stats.dual_residual = vrelD;
          stats.gap = vgap;
          if (vrelP <= opt.tolerance && vrelD <= opt.tolerance && vgap <= opt.tolerance) {
            download_iterates(xs, ys);
            extract(0, B2P_STATUS_OPTIMAL, smax(vrelP, smax(vrelD, vgap)), vpobj, vdobj, it);
            done[0] = 1;
            remaining = 0;
            break;
          }
          to_fp64 = true;
        } else if (kkt32 < 0.9 * best32) {
          best32 = kkt32;
          stale32 = 0;
        } else if (++stale32 >= kStallChecks) {
          to_fp64 = true;
        }
        if (to_fp64) {
          switch_to_fp64();
          restarts[0].reset();
          stats.restarts++;
          if (expired()) {
            expiredStop = true;
            break;
          }
          ++it;
          continue;
        }
      }
      for (int b = 0; b < k; ++b) {
        if (done[b]) continue;
        const double* s = h_sums + static_cast<size_t>(b) * kNumSums;
        const double pobj = s[CS_POBJ] * scaleObj;
        const double dobj = (s[CS_ROW_DOBJ] + s[CS_COL_DOBJ]) * scaleObj;
        const double relP = std::sqrt(s[CS_ROW_RES2]) / (1.0 + rn[b]);
        const double relD = std::sqrt(s[CS_COL_RES2]) / (1.0 + cn[b]);
        const double gap = std::fabs(pobj - dobj) / (1.0 + std::fabs(pobj) + std::fabs(dobj));
        const double kktErr = smax(relP, smax(relD, gap));
        if (k == 1) {
          stats.primal_residual = relP;
          stats.dual_residual = relD;
          stats.gap = gap;
        }
        if (opt.log_interval > 0 && k == 1 && checks % opt.log_interval == 0)
          std::fprintf(stderr,
                       "  pdhg %8lld  pobj % .8e  dobj % .8e  relP %.2e  relD %.2e  gap %.2e  w %.2e  restarts %d  %.2fs\n",
                       static_cast<long long>(it + 1), pobj + P.offset, dobj + P.offset, relP, relD, gap, omega[b],
                       stats.restarts, seconds_since(t_solve));
        if (!phase32 && relP <= opt.tolerance && relD <= opt.tolerance && gap <= opt.tolerance) {
          if (!fetched) {
            download_iterates(xs, ys);
            fetched = true;
          }
          extract(b, B2P_STATUS_OPTIMAL, kktErr, pobj, dobj, it);
          done[b] = 1;
          --remaining;
          continue;
        }
        if (restarts[b].due(omega[b], s, it, cE)) {
          h_mask[b] = 1;
          anyRestart = true;
        }
      }
      if (anyRestart) {
        for (int b = 0; b < k; ++b) {
          if (!h_mask[b]) continue;
          restarts[b].restart(omega[b], h_sums + static_cast<size_t>(b) * kNumSums);
          stats.restarts++;
        }
        upload_steps(omega);
      }
      if (remaining == 0) break;
      if (expired()) {
        expiredStop = true;
        break;
      }
      if (anyRestart) {
        const int64_t nk = static_cast<int64_t>(n) * k, mk = static_cast<int64_t>(m) * k;
        B2P_CUDA(cudaMemcpyAsync(d_mask, h_mask, sizeof(int32_t) * k, cudaMemcpyHostToDevice, stream));
        bytes_up += static_cast<int64_t>(sizeof(int32_t) * k);
        if (phase32)
          k_restart<float><<<blocks(std::max<int64_t>(nk + mk, k)), kBlock, 0, stream>>>(
              n, m, k, d_mask, v32[X32], v32[X032], v32[XP32], v32[Y32], v32[Y032], v32[YP32], v32[AX32],
              v32[AX032], v32[AXP32], d_it_base, d_restart_at);
        else
          k_restart<double><<<blocks(std::max<int64_t>(nk + mk, k)), kBlock, 0, stream>>>(
              n, m, k, d_mask, v[X], v[X0], v[XP], v[Y], v[Y0], v[YP], v[AX], v[AX0], v[AXP], d_it_base,
              d_restart_at);
        B2P_CUDA(cudaGetLastError());
        ++launches;
      }
      if (!phase32 && !opt.batch_no_compaction && k > 2 && remaining * 2 <= k) {
        // half the packed cases have terminated: keep the live ones (and, if
        // only one is live, one finished case beside it, so that the width
        // stays >= 2 for the batch kernels)
        std::vector<int32_t> keep;
        for (int b = 0; b < k; ++b)
          if (!done[b] || (remaining == 1 && b == (done[0] ? 0 : 1))) keep.push_back(b);
        compact_cases(keep);
        auto remap = [&](auto& vec) {
          auto old = vec;
          vec.resize(keep.size());
          for (size_t q = 0; q < keep.size(); ++q) vec[q] = old[keep[q]];
        };
        remap(done);
        remap(restarts);
        remap(omega);
        remap(rn);
        remap(cn);
        remap(conv32);
        remap(stall32);
        remap(best32v);
        remap(stale32v);
        upload_steps(omega);
      }
      ++it;
    }
    B2P_CUDA(cudaEventRecord(ev_stop, stream));
    B2P_CUDA(cudaEventSynchronize(ev_stop));
    float ms = 0;
    B2P_CUDA(cudaEventElapsedTime(&ms, ev_start, ev_stop));
    stats.kernel_seconds = ms / 1000.0;
    stats.solve_seconds = seconds_since(t_solve);
    stats.iterations = it + (remaining == 0 ? 1 : 0);
    stats.primal_weight = omega.empty() ? 1 : omega[0];
    if (remaining > 0) {
      // Unconverged cases: the last check's sums are the KKT of (x+, y+)
      // (the reference recomputes the same quantities, pdhg.cpp:668-680);
      // an FP32 point is re-measured in FP64 first.
      if (phase32) {
        fp32_point_to_fp64();
        verify_fp64();
      }
      download_iterates(xs, ys);
      for (int b = 0; b < k; ++b) {
        if (done[b]) continue;
        const double* s = h_sums + static_cast<size_t>(b) * kNumSums;
        const double pobj = s[CS_POBJ] * scaleObj, dobj = (s[CS_ROW_DOBJ] + s[CS_COL_DOBJ]) * scaleObj;
        const double relP = std::sqrt(s[CS_ROW_RES2]) / (1 + rn[b]);
        const double relD = std::sqrt(s[CS_COL_RES2]) / (1 + cn[b]);
        const double gap = std::fabs(pobj - dobj) / (1 + std::fabs(pobj) + std::fabs(dobj));
        extract(b, (expiredStop || expired()) ? B2P_STATUS_TIME_LIMIT : B2P_STATUS_ITERATION_LIMIT,
                smax(relP, smax(relD, gap)), pobj, dobj, it);
      }
    }
    stats.kernel_launches = launches;
    stats.bytes_uploaded = bytes_up;
    stats.bytes_downloaded = bytes_down;
    stats.transfer_seconds = transfer_seconds;
    stats.batch_compactions = compactions;
    restore_cases();
  }

  double kernel_bytes(int cls) const {
    if (cls == 2) return kernel_bytes(0) + kernel_bytes(1);
    // Algorithmic bytes of one launch per case-batch: the CSR operator
    // (12 nnz + 4 (rows+1)), the gathered vector once (8 cols k), and the
    // streamed vectors (primal: x, c, lo, up, x0 read + x, x+ written = 7;
    // dual: y, ax, rl, ru, y0, ax0 read + y, y+, ax, ax+ written = 10).
    const double nnz = static_cast<double>(P.A.val.size());
    if (cls == 0) return 12.0 * nnz + 4.0 * (n + 1) + 8.0 * m * k + 8.0 * 7 * n * k;
    if (cls == 1) return 12.0 * nnz + 4.0 * (m + 1) + 8.0 * n * k + 8.0 * 10 * m * k;
    // FP32 batch kernels: 4-byte values and vectors (the streamed costs and
    // bounds are FP32 copies too)
    if (cls == 3) return 8.0 * nnz + 4.0 * (n + 1) + 4.0 * m * k + 4.0 * 7 * n * k;
    return 8.0 * nnz + 4.0 * (m + 1) + 4.0 * n * k + 4.0 * 10 * m * k;
  }
};

}  // namespace b2p

using b2p::Engine;
using b2p::Error;
using b2p::guarded;

namespace {

void copy_results(Engine& e, double* x, double* y, b2p_result* results, b2p_stats* stats) {
  if (x && !e.x_out.empty()) std::memcpy(x, e.x_out.data(), e.x_out.size() * sizeof(double));
  if (y && !e.y_out.empty()) std::memcpy(y, e.y_out.data(), e.y_out.size() * sizeof(double));
  if (results) std::memcpy(results, e.results.data(), e.results.size() * sizeof(b2p_result));
  if (stats) *stats = e.stats;
}

}  // namespace

extern "C" {

void b2p_default_options(b2p_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->tolerance = 1e-6;
  o->max_iterations = 1000000;
  o->check_every = 64;
  o->ruiz_iterations = 10;
  o->pock_chambolle = 1;
  o->rescale_objective_and_bounds = 1;
  o->reflection = 1.0;
  o->log_interval = 0;
  o->device = -1;
  o->time_limit = 0;
  o->cancel_flag = nullptr;
  o->precision = B2P_PRECISION_FP64;
  o->use_graphs = 1;
  o->kernel_mode = B2P_KERNELS_AUTO;
  o->spmv_schedule = B2P_SCHEDULE_AUTO;
}

const char* b2p_last_error(void) { return b2p::last_error().c_str(); }

int b2p_engine_create(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const b2p_options* opts,
                      b2p_engine** out) {
  return guarded([&] {
    if (!out) throw Error(B2P_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (num_cases > 0 && !cases) throw Error(B2P_ERR_INVALID, "cases is NULL");
    auto e = std::make_unique<Engine>();
    e->create(lp, cases, num_cases, opts);
    *out = reinterpret_cast<b2p_engine*>(e.release());
  });
}

int b2p_engine_solve(b2p_engine* h, b2p_result* results, b2p_stats* stats) {
  return guarded([&] {
    if (!h) throw Error(B2P_ERR_INVALID, "engine is NULL");
    Engine& e = *reinterpret_cast<Engine*>(h);
    e.solve(b2p::Clock::now());
    copy_results(e, nullptr, nullptr, results, stats);
  });
}

int b2p_engine_fetch(b2p_engine* h, double* x, double* y) {
  return guarded([&] {
    if (!h) throw Error(B2P_ERR_INVALID, "engine is NULL");
    copy_results(*reinterpret_cast<Engine*>(h), x, y, nullptr, nullptr);
  });
}

int b2p_engine_destroy(b2p_engine* h) {
  return guarded([&] { delete reinterpret_cast<Engine*>(h); });
}

int b2p_engine_set_start(b2p_engine* h, const double* x, const double* row_dual, double primal_weight) {
  return guarded([&] {
    if (!h) throw Error(B2P_ERR_INVALID, "engine is NULL");
    reinterpret_cast<Engine*>(h)->set_start(x, row_dual, primal_weight);
  });
}

int b2p_engine_set_profiling(b2p_engine* h, int32_t on) {
  return guarded([&] {
    if (!h) throw Error(B2P_ERR_INVALID, "engine is NULL");
    reinterpret_cast<Engine*>(h)->profiling = on != 0;
  });
}

int b2p_engine_kernel_times(b2p_engine* h, int32_t cls, int64_t* launches, double* total_ms) {
  return guarded([&] {
    if (!h || cls < 0 || cls > 4) throw Error(B2P_ERR_INVALID, "bad engine or kernel class");
    Engine& e = *reinterpret_cast<Engine*>(h);
    if (launches) *launches = e.prof_launches[cls];
    if (total_ms) *total_ms = e.prof_ms[cls];
  });
}

int b2p_engine_kernel_bytes(b2p_engine* h, int32_t cls, double* bytes) {
  return guarded([&] {
    if (!h || cls < 0 || cls > 4 || !bytes) throw Error(B2P_ERR_INVALID, "bad engine, class or output");
    *bytes = reinterpret_cast<Engine*>(h)->kernel_bytes(cls);
  });
}

int b2p_solve_pdhg(const b2p_lp* lp, const b2p_options* opts, double* x, double* row_dual, b2p_result* result,
                   b2p_stats* stats) {
  return guarded([&] {
    const auto t0 = b2p::Clock::now();
    Engine e;
    e.create(lp, nullptr, 0, opts);
    e.solve(t0);
    copy_results(e, x, row_dual, result, stats);
  });
}

int b2p_solve_pdhg_batch(const b2p_lp* base, const b2p_case* cases, int32_t num_cases, const b2p_options* opts,
                         double* x, double* row_dual, b2p_result* results, b2p_stats* batch_stats) {
  return guarded([&] {
    if (num_cases <= 0) return;  // solvePdhgBatch returns {} for no cases
    if (!cases) throw Error(B2P_ERR_INVALID, "cases is NULL");
    const auto t0 = b2p::Clock::now();
    Engine e;
    e.create(base, cases, num_cases, opts);
    e.solve(t0);
    copy_results(e, x, row_dual, results, batch_stats);
  });
}

int b2p_gpu_available(void) {
  try {
    const int dev = b2p::pick_device(-1);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, b2p::k_spmv) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    (void)dev;
    return 1;
  } catch (...) {
    return 0;
  }
}

int b2p_gpu_info_json(char* buf, size_t cap) {
  std::string name, reason;
  bool avail = false;
  int major = 0, minor = 0, sms = 0, drv = 0, rt = 0, binver = 0;
  double mem = 0, bw = 0;
  try {
    const int dev = b2p::pick_device(-1);
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) == cudaSuccess) {
      name = p.name;
      major = p.major;
      minor = p.minor;
      sms = p.multiProcessorCount;
      mem = static_cast<double>(p.totalGlobalMem);
      int clk = 0, bus = 0;
      cudaDeviceGetAttribute(&clk, cudaDevAttrMemoryClockRate, dev);
      cudaDeviceGetAttribute(&bus, cudaDevAttrGlobalMemoryBusWidth, dev);
      bw = 2.0 * clk * 1e3 * (bus / 8.0) / 1e9;
    }
    cudaDriverGetVersion(&drv);
    cudaRuntimeGetVersion(&rt);
    avail = b2p_gpu_available() != 0;
    if (!avail) reason = "kernels not loadable on this device";
    cudaFuncAttributes fa;
    if (avail && cudaFuncGetAttributes(&fa, b2p::k_spmv) == cudaSuccess) binver = fa.binaryVersion;
  } catch (std::exception& e) {
    reason = e.what();
  }
  char tmp[1024];
  int len = std::snprintf(tmp, sizeof(tmp),
                          "{\"available\": %s, \"name\": \"%s\", \"reason\": \"%s\", \"compute_capability\": \"%d.%d\", "
                          "\"multiprocessors\": %d, \"memory_bytes\": %.0f, \"peak_bandwidth_GBs\": %.1f, "
                          "\"driver_version\": %d, \"runtime_version\": %d, \"kernel_binary_version\": %d, "
                          "\"kernels\": \"ahead-of-time sm_100a\"}",
                          avail ? "true" : "false", name.c_str(), reason.c_str(), major, minor, sms, mem, bw, drv, rt,
                          binver);
  if (buf && cap > 0) {
    std::strncpy(buf, tmp, cap - 1);
    buf[cap - 1] = '\0';
  }
  return len;
}

int b2p_csr_spmv(int32_t rows, int32_t cols, int32_t k, const int32_t* ptr, const int32_t* idx, const double* val,
                 const double* x, double* y) {
  return guarded([&] {
    if (rows < 0 || cols < 0 || k <= 0 || !ptr || (rows > 0 && !y)) throw Error(B2P_ERR_INVALID, "bad arguments");
    const int32_t nnz = ptr[rows];
    for (int32_t i = 0; i < rows; ++i)
      if (ptr[i + 1] < ptr[i]) throw Error(B2P_ERR_INVALID, "ptr must be non-decreasing");
    for (int32_t q = 0; q < nnz; ++q)
      if (idx[q] < 0 || idx[q] >= cols) throw Error(B2P_ERR_INVALID, "column index out of range");
    const int dev = b2p::pick_device(-1);
    B2P_CUDA(cudaSetDevice(dev));
    Engine tmp;  // owns the allocations and the stream
    B2P_CUDA(cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking));
    int32_t* dp = tmp.upload(std::vector<int32_t>(ptr, ptr + rows + 1));
    int32_t* di = tmp.upload(std::vector<int32_t>(idx, idx + nnz));
    double* dv = tmp.upload(std::vector<double>(val, val + nnz));
    double* dx = tmp.upload(std::vector<double>(x, x + static_cast<size_t>(cols) * k));
    double* dy = tmp.dalloc<double>(static_cast<size_t>(rows) * k);
    if (rows > 0) {
      b2p::k_spmv<<<Engine::blocks(static_cast<int64_t>(rows) * k), b2p::kBlock, 0, tmp.stream>>>(
          rows, k, b2p::CsrView{dp, di, dv, rows}, dx, dy);
      B2P_CUDA(cudaGetLastError());
      B2P_CUDA(cudaMemcpyAsync(y, dy, sizeof(double) * rows * k, cudaMemcpyDeviceToHost, tmp.stream));
    }
    B2P_CUDA(cudaStreamSynchronize(tmp.stream));
  });
}

}  // extern "C"
