// Many LPs of different sizes, each with its own A, solved together.
//
// The reference batches only cases that share one A (solvePdhgBatch,
// src/pdhg/pdhg.cpp:719-728, k-interleaved vectors).  Uneven families -- many
// independent LPs -- are solved here as ONE block-diagonal LP: the instances'
// A (and A^T) are concatenated with row and column offsets, so every
// iteration is a single pair of fused, row-binned SpMV kernels over all
// instances (the same kernels as the single-LP fused form, with a per-row
// instance id that selects the instance's tau, sigma and Halpern counter).
// Each instance keeps its own scaling, step sizes, primal weight, restart
// state and termination: the host takes the reference's decisions per
// instance at every check, and a terminated instance's rows are skipped by
// every kernel from then on.  Check reductions are segmented by instance with
// a fixed block table, so results are deterministic; one check interval is
// one CUDA graph.  Instance b's iterates are those of its own single solve up
// to the rounding order of the sums.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "pdhg_host_common.h"
#include "pdhg_kernels.cuh"
#include "pdhg_prepare.h"
#include "pdhg_restart.h"
#include "pdhg_scale.cuh"
#include "pdhg_cta.cuh"
#include "pdhg_sched.h"
#include "pdhg_spmv.cuh"
#include "pdhg_tiled.cuh"

namespace b2p {

// Instantiated owner-kernel variants: (threads per block, elements per thread).
#define B2P_OWNER_VARIANTS(X) X(128, 1) X(256, 1) X(512, 1) X(128, 2) X(256, 2) X(512, 2)

constexpr int kSegRows = 2048;  // rows (or columns) per check-reduction block

// Per check block: its instance and its [beg, end) range of global rows.
struct SegTable {
  const int32_t* __restrict__ inst;
  const int32_t* __restrict__ beg;
  const int32_t* __restrict__ end;
};

// x_out = the projection of x onto [lo, up] (the FP64 run's starting point
// from an FP32 run's x+, whose FP32 rounding may sit just outside a bound).
__global__ void __launch_bounds__(kBlock) k_clamp_to_bounds(int32_t n, const double* __restrict__ x,
                                                            const double* __restrict__ lo,
                                                            const double* __restrict__ up, double* __restrict__ out) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double v = x[j];
  v = (v < lo[j]) ? lo[j] : v;
  v = (up[j] < v) ? up[j] : v;
  out[j] = v;
}

// Row part of the check for every live instance (see k_check_rows).
__global__ void __launch_bounds__(kBlock) k_check_rows_multi(SegTable t, const int32_t* __restrict__ done,
                                                             const double* __restrict__ axp,
                                                             const double* __restrict__ rl,
                                                             const double* __restrict__ ru,
                                                             const double* __restrict__ yp,
                                                             const double* __restrict__ y,
                                                             const double* __restrict__ y0,
                                                             const double* __restrict__ rfac,
                                                             double* __restrict__ partial) {
  __shared__ double sh[kRowSums * (kBlock / 32)];
  double s[kRowSums] = {0, 0, 0, 0, 0};
  const int blk = blockIdx.x;
  if (!done[t.inst[blk]]) {
    for (int i = t.beg[blk] + threadIdx.x; i < t.end[blk]; i += blockDim.x) {
      const double a = axp[i], l = rl[i], u = ru[i];
      double e1 = l - a, e2 = a - u;
      e1 = (e1 < 0.0) ? 0.0 : e1;
      e2 = (e2 < 0.0) ? 0.0 : e2;
      const double res = (e1 + e2) * rfac[i];
      s[0] += res * res;
      const double yv = yp[i];
      if (yv > 0.0 && l > -1e300)
        s[1] += yv * l;
      else if (yv < 0.0 && u < 1e300)
        s[1] += yv * u;
      s[2] += yv * yv;
      const double d1 = y[i] - yv, d2 = yv - y0[i];
      s[3] += d1 * d1;
      s[4] += d2 * d2;
    }
  }
  block_reduce<kRowSums>(s, sh);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < kRowSums; ++q) partial[blk * kRowSums + q] = s[q];
}

// Column part (A^T y+ precomputed by the binned SpMV).
__global__ void __launch_bounds__(kBlock) k_check_cols_multi(SegTable t, const int32_t* __restrict__ done,
                                                             const double* __restrict__ atyp,
                                                             const double* __restrict__ xp,
                                                             const double* __restrict__ x,
                                                             const double* __restrict__ x0,
                                                             const double* __restrict__ c,
                                                             const double* __restrict__ lo,
                                                             const double* __restrict__ up,
                                                             const double* __restrict__ cfac,
                                                             double* __restrict__ partial) {
  __shared__ double sh[kRowSums * (kBlock / 32)];
  double s[kRowSums] = {0, 0, 0, 0, 0};
  const int blk = blockIdx.x;
  if (!done[t.inst[blk]]) {
    for (int j = t.beg[blk] + threadIdx.x; j < t.end[blk]; j += blockDim.x) {
      const double cv = c[j], l = lo[j], u = up[j], xpv = xp[j];
      const double d = cv - atyp[j];
      const bool hl = l > -1e300, hu = u < 1e300;
      double res = 0.0;
      if (!hl && !hu)
        res = fabs(d);
      else if (!hl)
        res = (d < 0.0) ? 0.0 : d;
      else if (!hu)
        res = (-d < 0.0) ? 0.0 : -d;
      res *= cfac[j];
      s[0] += res * res;
      s[1] += cv * xpv;
      if (d > 0.0 && hl)
        s[2] += d * l;
      else if (d < 0.0 && hu)
        s[2] += d * u;
      const double d1 = x[j] - xpv, d2 = xpv - x0[j];
      s[3] += d1 * d1;
      s[4] += d2 * d2;
    }
  }
  block_reduce<kRowSums>(s, sh);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < kRowSums; ++q) partial[blk * kRowSums + q] = s[q];
}

// grid = instances: sums of the instance's blocks, in block order.
__global__ void __launch_bounds__(kBlock) k_check_finalize_multi(const int32_t* __restrict__ rblk_off,
                                                                 const int32_t* __restrict__ cblk_off,
                                                                 const int32_t* __restrict__ done,
                                                                 const double* __restrict__ prow,
                                                                 const double* __restrict__ pcol,
                                                                 double* __restrict__ out,
                                                                 int64_t* __restrict__ it_base, int32_t L) {
  __shared__ double sh[kNumSums * (kBlock / 32)];
  const int b = blockIdx.x;
  double s[kNumSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (!done[b]) {
    for (int g = rblk_off[b] + threadIdx.x; g < rblk_off[b + 1]; g += blockDim.x)
#pragma unroll
      for (int q = 0; q < kRowSums; ++q) s[q] += prow[g * kRowSums + q];
    for (int g = cblk_off[b] + threadIdx.x; g < cblk_off[b + 1]; g += blockDim.x)
#pragma unroll
      for (int q = 0; q < kRowSums; ++q) s[kRowSums + q] += pcol[g * kRowSums + q];
  }
  block_reduce<kNumSums>(s, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < kNumSums; ++q) out[static_cast<int64_t>(b) * kNumSums + q] = s[q];
    if (b == 0) *it_base += L;
  }
}

// Deferred Halpern steps at a check iteration, per element's instance.
__global__ void __launch_bounds__(kBlock) k_halpern_all_multi(int32_t n, int32_t m, const int32_t* __restrict__ cinst,
                                                              const int32_t* __restrict__ rinst,
                                                              const int32_t* __restrict__ done,
                                                              double* __restrict__ x, const double* __restrict__ xp,
                                                              const double* __restrict__ x0, double* __restrict__ y,
                                                              const double* __restrict__ yp,
                                                              const double* __restrict__ y0, double* __restrict__ ax,
                                                              const double* __restrict__ axp,
                                                              const double* __restrict__ ax0, IterClock ck,
                                                              double rho) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < n) {
    const int b = cinst[t];
    if (!done[b]) x[t] = halpern_step(x[t], xp[t], x0[t], halpern_lambda(ck, b), rho);
  } else if (t < static_cast<int64_t>(n) + m) {
    const int64_t u = t - n;
    const int b = rinst[u];
    if (!done[b]) {
      const double lam = halpern_lambda(ck, b);
      y[u] = halpern_step(y[u], yp[u], y0[u], lam, rho);
      ax[u] = halpern_step(ax[u], axp[u], ax0[u], lam, rho);
    }
  }
}

// Masked restart per instance (src/pdhg/pdhg.cpp:153-165).
__global__ void __launch_bounds__(kBlock) k_restart_multi(int32_t n, int32_t m, int32_t k,
                                                          const int32_t* __restrict__ cinst,
                                                          const int32_t* __restrict__ rinst,
                                                          const int32_t* __restrict__ mask, double* __restrict__ x,
                                                          double* __restrict__ x0, const double* __restrict__ xp,
                                                          double* __restrict__ y, double* __restrict__ y0,
                                                          const double* __restrict__ yp, double* __restrict__ ax,
                                                          double* __restrict__ ax0, const double* __restrict__ axp,
                                                          const int64_t* __restrict__ it_base,
                                                          int64_t* __restrict__ restart_at) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < k && mask[t]) restart_at[t] = *it_base;
  if (t < n) {
    if (mask[cinst[t]]) x[t] = x0[t] = xp[t];
  } else if (t < static_cast<int64_t>(n) + m) {
    const int64_t u = t - n;
    if (mask[rinst[u]]) {
      y[u] = y0[u] = yp[u];
      ax[u] = ax0[u] = axp[u];
    }
  }
}

// idx[q] += off[b] for the entries q of LP b (block b): LP-local indices of
// the concatenated operator become global ones.
// Sliced-ELL copy of CSR rows: row r's entries to base[r] + 32 q.
__global__ void __launch_bounds__(kBlock) k_to_sliced(int32_t rows, const int32_t* __restrict__ ptr,
                                                      const int32_t* __restrict__ idx, const double* __restrict__ val,
                                                      const int32_t* __restrict__ base, int32_t* __restrict__ sidx,
                                                      double* __restrict__ sval) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  int64_t b = base[r];
  for (int32_t p = ptr[r]; p < ptr[r + 1]; ++p, b += 32) {
    sidx[b] = idx[p];
    sval[b] = val[p];
  }
}

__global__ void k_offset_segments(const int64_t* __restrict__ seg, const int32_t* __restrict__ off,
                                  int32_t* __restrict__ idx) {
  const int b = blockIdx.x;
  const int32_t o = off[b];
  for (int64_t q = seg[b] + threadIdx.x; q < seg[b + 1]; q += blockDim.x) idx[q] += o;
}

// ---- ||A|| of every LP at once (powerIteration, src/pdhg/pdhg.cpp:404-422) ----
// The block-diagonal A x and A^T y are CSR row sums in increasing column
// order -- the addition order of the reference's scatter products -- and each
// LP's ||z|| is summed by one thread in index order, so every LP's estimate is
// bit-identical to its own sequential power iteration.

// x_j = 1 / sqrt(n_b) for the columns of LP b; LPs without entries are done
// from the start with ||A|| = 1.
__global__ void k_pi_init(int32_t N, int32_t K, const int32_t* __restrict__ cinst, const int32_t* __restrict__ coff,
                          const int64_t* __restrict__ lp_nnz, double* __restrict__ x, int32_t* __restrict__ done,
                          double* __restrict__ s) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < N) {
    const int b = cinst[t];
    const int32_t nb = coff[b + 1] - coff[b];
    x[t] = __ddiv_rn(1.0, __dsqrt_rn(static_cast<double>(nb > 1 ? nb : 1)));
  }
  if (t < K) {
    done[t] = lp_nnz[t] == 0 ? 1 : 0;
    s[t] = 1.0;
  }
}

// One thread per LP: nz = sqrt(sum z_j^2) in index order; nz == 0 ends the
// LP's iteration with ||A|| = 1, else s = sqrt(nz).
__global__ void k_pi_norm(int32_t K, const int32_t* __restrict__ coff, const double* __restrict__ z,
                          int32_t* __restrict__ done, double* __restrict__ nz_out, double* __restrict__ s) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= K || done[b]) return;
  double acc = 0.0;
  for (int32_t j = coff[b]; j < coff[b + 1]; ++j) acc = __dadd_rn(acc, __dmul_rn(z[j], z[j]));
  const double nz = __dsqrt_rn(acc);
  nz_out[b] = nz;
  if (nz == 0.0) {
    done[b] = 1;
    s[b] = 1.0;
  } else {
    s[b] = __dsqrt_rn(nz);
  }
}

// x = z / nz of the column's LP (LPs that are done keep their x).
__global__ void k_pi_scale(int32_t N, const int32_t* __restrict__ cinst, const int32_t* __restrict__ done,
                           const double* __restrict__ nz, const double* __restrict__ z, double* __restrict__ x) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= N) return;
  const int b = cinst[t];
  if (!done[b]) x[t] = __ddiv_rn(z[t], nz[b]);
}

namespace {

enum MSlot : int { MX, MXP, MX0, MC, MLO, MUP, MXINIT, MATYP, MNCOL, MY = MNCOL, MYP, MY0, MAX, MAXP, MAX0, MRL, MRU,
                   MAXINIT, MYINIT, MNSLOT };

struct MultiEngine {
  int device = 0;
  int K = 0;
  b2p_options opt{};
  std::vector<Prepared> P;
  std::vector<int64_t> roff, coff;  // row / column offsets of instance b
  int32_t M = 0, N = 0;
  std::vector<double> cNorm, rhsNorm, omega0, eta;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  int32_t *dA_ptr = nullptr, *dA_idx = nullptr, *dT_ptr = nullptr, *dT_idx = nullptr;
  // CTA form: sliced-ELL copies of the operators (see CtaArgs), NULL when not built
  int32_t *d_sa_base = nullptr, *d_sa_idx = nullptr, *d_st_base = nullptr, *d_st_idx = nullptr;
  double *d_sa_val = nullptr, *d_st_val = nullptr;
  float *d_sa_val32 = nullptr, *d_st_val32 = nullptr;
  int64_t sa_len = 0, st_len = 0;
  double *dA_val = nullptr, *dT_val = nullptr, *d_rfac = nullptr, *d_cfac = nullptr;
  double* v[MNSLOT] = {};
  int32_t *d_rinst = nullptr, *d_cinst = nullptr, *d_done = nullptr, *d_mask = nullptr;
  double *d_tau = nullptr, *d_sigma = nullptr, *d_prow = nullptr, *d_pcol = nullptr, *d_sums = nullptr;
  int64_t *d_it_base = nullptr, *d_restart_at = nullptr;
  SegTable rtab{}, ctab{};
  int32_t *d_rblk_off = nullptr, *d_cblk_off = nullptr;
  int g_rows = 0, g_cols = 0;
  RowBins binsA{}, binsT{};
  // host copies for compaction: row pointers of the concatenated operators,
  // nonzeros of each instance, and the nonzeros the current schedule covers
  std::vector<int32_t> hA_ptr, hT_ptr;
  std::vector<int64_t> inst_nnz;
  int64_t sched_nnz = 0;
  int ltA = 0, ltT = 0;
  int64_t wave = 0;
  int rounds = 2;
  // Per operator, when chosen: the warp-tile schedule of the short rows plus a
  // binned schedule of the long rows only (pdhg_tiled.cuh).
  struct TileSched {
    bool on = false;
    bool capped = false;  // kernels compiled for 4 resident blocks per SM (64 registers)
    TileSet ts{};
    RowBins longb{};
  };
  TileSched tilesA, tilesT;
  bool streamA = false, streamT = false;  // binned schedules: evict-first streaming loads
  double* h_sums = nullptr;
  double* h_steps = nullptr;
  int32_t *h_mask = nullptr, *h_done = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  std::map<int, cudaGraph_t> graph_defs;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  b2p_stats stats{};
  std::vector<b2p_result> results;
  std::vector<double> weights;  // per LP: final primal weight, original-space units (omega gamma / beta)
  std::vector<std::vector<double>> xs, ys;  // per instance, original space
  int64_t launches = 0, bytes_up = 0, bytes_down = 0;
  int compactions = 0;
  // CTA form (pdhg_cta.cuh): one block per LP
  bool cta = false;
  // kernel variant: threads per block and elements owned per thread (0: the
  // general kernel, run_lp; -1: the general kernel compiled for 1,024 threads
  // per SM (64 registers); 1 or 2: the owner kernel, run_owner)
  int cta_nt = 256, cta_r = 0;
  int64_t cta_smem = 0;        // general kernel: largest LP's tier bytes
  int64_t cta_owner_smem = 0;  // owner kernel: largest LP's bytes (0: not every LP fits)
  int32_t cta_max_dim = 0;     // largest max(m, n)
  std::vector<CtaLp> cta_lps;
  CtaLp* d_lps = nullptr;
  int32_t* d_order = nullptr;
  CtaOut* d_out = nullptr;
  int32_t* h_stop = nullptr;  // host-mapped stop flag
  // Mixed precision in the CTA form: an FP32 run of every LP (operators and
  // state in FP32), then an FP64 run from each LP's FP32 point.
  bool mixed = false;
  // every LP has the same A (members of one family): the CTA form reads the
  // first LP's copy of the (identically scaled) operators for all of them
  bool shared_operator = false;
  float *dA_val32 = nullptr, *dT_val32 = nullptr;
  float* v32[9] = {};           // global-tier FP32 state: x, x+, x0 (N); y, y+, y0, Ax, Ax+, Ax0 (M)
  int64_t cta_smem32 = 0;       // FP32 run: largest LP's tier bytes
  int cta_nt32 = 256, cta_r32 = 0;  // FP32 run: general-kernel variant (threads, 0 or -1 as cta_r)
  double *d_x2 = nullptr, *d_y2 = nullptr, *d_ax2 = nullptr;  // the FP64 run's starting point
  CtaLp* d_lps2 = nullptr;
  int32_t* d_order2 = nullptr;
  std::vector<int32_t> host_order;  // largest LPs first
  static constexpr int kStallChecks = 20;  // FP32 run: checks without a 10% KKT gain before it ends

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
  static unsigned blocks(int64_t len) { return static_cast<unsigned>(std::max<int64_t>(1, (len + kBlock - 1) / kBlock)); }
  CsrView viewA() const { return CsrView{dA_ptr, dA_idx, dA_val, M}; }
  CsrView viewAT() const { return CsrView{dT_ptr, dT_idx, dT_val, N}; }

  ~MultiEngine() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    for (auto& g : graph_defs) cudaGraphDestroy(g.second);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    cudaSetDevice(device);
    if (stream) {
      for (void* p : allocs) cudaFreeAsync(p, stream);
      cudaStreamSynchronize(stream);
    }
    PinnedCache::put(h_sums, sizeof(double) * K * kNumSums);
    PinnedCache::put(h_steps, sizeof(double) * 2 * K);
    PinnedCache::put(h_mask, sizeof(int32_t) * K);
    PinnedCache::put(h_done, sizeof(int32_t) * K);
    if (h_stop) cudaFreeHost(h_stop);
    if (stream) cudaStreamDestroy(stream);
  }

  void create(const b2p_lp* lps, int num, const b2p_options* o) {
    if (!lps || num <= 0) throw Error(B2P_ERR_INVALID, "no LPs");
    for (int b = 0; b < num; ++b) check_lp(&lps[b]);
    if (o) opt = *o; else b2p_default_options(&opt);
    if (opt.check_every <= 0) throw Error(B2P_ERR_INVALID, "check_every must be positive");
    device = pick_device(opt.device);
    B2P_CUDA(cudaSetDevice(device));
    B2P_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    B2P_CUDA(cudaEventCreate(&ev_start));
    B2P_CUDA(cudaEventCreate(&ev_stop));
    K = num;
    shared_operator = same_operator(lps, num);
    const auto t0 = Clock::now();
    // ---- host preparation of every instance (structure only), on all host threads ----
    P.resize(K);
    std::atomic<int> next{0};
    const int nth = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), static_cast<unsigned>(K)));
    std::vector<std::thread> pool;
    std::vector<std::string> errs(nth);
    for (int t = 0; t < nth; ++t)
      pool.emplace_back([&, t] {
        try {
          for (int b; (b = next.fetch_add(1)) < K;) {
            const b2p_lp& l = lps[b];
            // structure and raw values; the scaling runs on the device below
            P[b] = prepare_structure(l.num_rows, l.num_cols, l.start, l.index, l.value, l.obj_offset, false);
          }
        } catch (std::exception& e) {
          errs[t] = e.what();
        }
      });
    for (auto& th : pool) th.join();
    for (auto& e : errs)
      if (!e.empty()) throw Error(B2P_ERR_INVALID, e);
    stats.prepare_seconds = seconds_since(t0);
    // ---- block-diagonal concatenation ----
    roff.assign(K + 1, 0);
    coff.assign(K + 1, 0);
    int64_t annz = 0;
    for (int b = 0; b < K; ++b) {
      roff[b + 1] = roff[b] + P[b].m;
      coff[b + 1] = coff[b] + P[b].n;
      annz += static_cast<int64_t>(P[b].A.val.size());
    }
    if (roff[K] >= INT32_MAX || coff[K] >= INT32_MAX || annz >= INT32_MAX)
      throw Error(B2P_ERR_TOO_LARGE, "family exceeds 2^31 rows, columns or nonzeros");
    M = static_cast<int32_t>(roff[K]);
    N = static_cast<int32_t>(coff[K]);
    HostCsr A, AT;
    A.rows = M;
    A.cols = N;
    AT.rows = N;
    AT.cols = M;
    std::vector<int64_t> aoff(K + 1, 0);  // first entry of LP b in the concatenated operators
    for (int b = 0; b < K; ++b) aoff[b + 1] = aoff[b] + static_cast<int64_t>(P[b].A.val.size());
    A.ptr.resize(static_cast<size_t>(M) + 1);
    AT.ptr.resize(static_cast<size_t>(N) + 1);
    A.ptr[0] = 0;
    AT.ptr[0] = 0;
    std::vector<int32_t> rinst(M), cinst(N);
    std::vector<double> rfac(M), cfac(N), c(N), lo(N), up(N), rl(M), ru(M), x0(N);
    cNorm.assign(K, 0);
    rhsNorm.assign(K, 0);
    omega0.assign(K, 1.0);
    eta.assign(K, 0);
    // every LP fills its own ranges: on all host threads, with the same values
    // as one pass in LP order
    auto parallel_lps = [&](auto&& f) {
      std::atomic<int> nextb{0};
      std::vector<std::thread> workers;
      for (int t = 0; t < nth; ++t)
        workers.emplace_back([&] {
          for (int b; (b = nextb.fetch_add(1)) < K;) f(b);
        });
      for (auto& th : workers) th.join();
    };
    parallel_lps([&](int b) {
      const Prepared& p = P[b];
      const int32_t base = static_cast<int32_t>(aoff[b]);
      for (int32_t i = 0; i < p.m; ++i) A.ptr[roff[b] + i + 1] = base + p.A.ptr[i + 1];
      for (int32_t j = 0; j < p.n; ++j) AT.ptr[coff[b] + j + 1] = base + p.AT.ptr[j + 1];
    });
    auto fill = [&](int b) {
      const Prepared& p = P[b];
      const b2p_lp& l = lps[b];
      // scaled case vectors (src/pdhg/pdhg.cpp:466-481, 506-530), k = 1 per instance
      double s = 0;
      for (int32_t j = 0; j < p.n; ++j) s += l.col_cost[j] * l.col_cost[j];
      cNorm[b] = std::sqrt(s);
      s = 0;
      for (int32_t i = 0; i < p.m; ++i) {
        if (finite_bound(l.row_lower[i])) s += l.row_lower[i] * l.row_lower[i];
        if (finite_bound(l.row_upper[i]) && l.row_upper[i] != l.row_lower[i]) s += l.row_upper[i] * l.row_upper[i];
      }
      rhsNorm[b] = std::sqrt(s);
      double cn = 0, bn = 0;
      for (int32_t j = 0; j < p.n; ++j) {
        const size_t t = static_cast<size_t>(coff[b] + j);
        cinst[t] = b;
        cfac[t] = p.cfac[j];
        c[t] = l.col_cost[j] * p.Cs[j] / p.gamma;
        lo[t] = finite_bound(l.col_lower[j]) ? l.col_lower[j] / p.Cs[j] / p.beta : -HUGE_VAL;
        up[t] = finite_bound(l.col_upper[j]) ? l.col_upper[j] / p.Cs[j] / p.beta : HUGE_VAL;
        x0[t] = smin(smax(0.0, lo[t]), up[t]);
        cn += c[t] * c[t];
      }
      for (int32_t i = 0; i < p.m; ++i) {
        const size_t t = static_cast<size_t>(roff[b] + i);
        rinst[t] = b;
        rfac[t] = p.rfac[i];
        rl[t] = finite_bound(l.row_lower[i]) ? l.row_lower[i] * p.R[i] / p.beta : -HUGE_VAL;
        ru[t] = finite_bound(l.row_upper[i]) ? l.row_upper[i] * p.R[i] / p.beta : HUGE_VAL;
        if (finite_bound(rl[t])) bn += rl[t] * rl[t];
        if (finite_bound(ru[t]) && ru[t] != rl[t]) bn += ru[t] * ru[t];
      }
      if (cn > 1e-20 && bn > 1e-20) omega0[b] = std::sqrt(cn) / std::sqrt(bn);
    };
    // ---- device ----
    const auto tx = Clock::now();
    dA_ptr = upload(A.ptr);
    // Each LP's index and value arrays go straight to their ranges of the
    // concatenated device operators (no host copy of the whole batch); the
    // row / column offsets of the indices are added on the device.
    dA_idx = dalloc<int32_t>(static_cast<size_t>(annz) + kTilePad);
    dA_val = dalloc<double>(static_cast<size_t>(annz) + kTilePad);
    dT_idx = dalloc<int32_t>(static_cast<size_t>(annz) + kTilePad);
    dT_val = dalloc<double>(static_cast<size_t>(annz) + kTilePad);
    B2P_CUDA(cudaMemsetAsync(dA_idx + annz, 0, kTilePad * sizeof(int32_t), stream));
    B2P_CUDA(cudaMemsetAsync(dA_val + annz, 0, kTilePad * sizeof(double), stream));
    B2P_CUDA(cudaMemsetAsync(dT_idx + annz, 0, kTilePad * sizeof(int32_t), stream));
    B2P_CUDA(cudaMemsetAsync(dT_val + annz, 0, kTilePad * sizeof(double), stream));
    for (int b = 0; b < K; ++b) {
      const Prepared& p = P[b];
      const size_t e = p.A.val.size();
      if (!e) continue;
      B2P_CUDA(cudaMemcpyAsync(dA_idx + aoff[b], p.A.idx.data(), e * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(dA_val + aoff[b], p.A.val.data(), e * sizeof(double), cudaMemcpyHostToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(dT_idx + aoff[b], p.AT.idx.data(), e * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(dT_val + aoff[b], p.AT.val.data(), e * sizeof(double), cudaMemcpyHostToDevice, stream));
    }
    bytes_up += 24 * annz;
    {
      std::vector<int32_t> co(K), ro(K);
      for (int b = 0; b < K; ++b) {
        co[b] = static_cast<int32_t>(coff[b]);
        ro[b] = static_cast<int32_t>(roff[b]);
      }
      const int64_t* d_aoff = upload(aoff);
      const int32_t* d_co = upload(co);
      const int32_t* d_ro = upload(ro);
      k_offset_segments<<<K, kBlock, 0, stream>>>(d_aoff, d_co, dA_idx);
      k_offset_segments<<<K, kBlock, 0, stream>>>(d_aoff, d_ro, dT_idx);
      B2P_CUDA(cudaGetLastError());
    }
    dT_ptr = upload(AT.ptr);
    // ---- scaling on the device (Ruiz + Pock-Chambolle), rounding and the
    // rescaling constants on the host, the scaled operators on the device ----
    const auto ts = Clock::now();
    {
      std::vector<double> rs(M, 1.0), cs(N, 1.0);
      if (opt.ruiz_iterations > 0 && annz > 0)
        device_ruiz_factors(stream, device, viewA(), viewAT(), opt.ruiz_iterations, opt.pock_chambolle != 0, rs, cs);
      const bool rescale = opt.rescale_objective_and_bounds != 0;
      parallel_lps([&](int b) {
        const b2p_lp& l = lps[b];
        finish_scaling(P[b], rs.data() + roff[b], cs.data() + coff[b], l.col_cost, l.row_lower, l.row_upper,
                       rescale);
      });
      std::vector<double> R(M), Cs(N);
      for (int b = 0; b < K; ++b) {
        std::copy(P[b].R.begin(), P[b].R.end(), R.begin() + roff[b]);
        std::copy(P[b].Cs.begin(), P[b].Cs.end(), Cs.begin() + coff[b]);
      }
      device_scale_operators(stream, device, viewA(), viewAT(), dA_val, dT_val, R, Cs);
    }
    stats.prepare_seconds += seconds_since(ts);
    parallel_lps(fill);
    d_rfac = upload(rfac);
    d_cfac = upload(cfac);
    d_rinst = upload(rinst);
    d_cinst = upload(cinst);
    device_power_iterations(40);
    for (int b = 0; b < K; ++b) eta[b] = 0.998 / P[b].normA;
    for (int q = 0; q < MNSLOT; ++q) v[q] = dalloc<double>(q >= MY ? M : N);
    auto put = [&](int q, const std::vector<double>& h) {
      if (!h.empty()) B2P_CUDA(cudaMemcpyAsync(v[q], h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
      bytes_up += static_cast<int64_t>(h.size() * sizeof(double));
    };
    put(MC, c);
    put(MLO, lo);
    put(MUP, up);
    put(MRL, rl);
    put(MRU, ru);
    put(MXINIT, x0);
    if (M) B2P_CUDA(cudaMemsetAsync(v[MYINIT], 0, sizeof(double) * M, stream));
    d_tau = dalloc<double>(K);
    d_sigma = dalloc<double>(K);
    d_it_base = dalloc<int64_t>(1);
    d_restart_at = dalloc<int64_t>(K);
    d_done = dalloc<int32_t>(K);
    d_mask = dalloc<int32_t>(K);
    if (M > 0) {
      k_spmv<<<blocks(M), kBlock, 0, stream>>>(M, 1, viewA(), v[MXINIT], v[MAXINIT]);
      B2P_CUDA(cudaGetLastError());
    }
    inst_nnz.assign(K, 0);
    for (int b = 0; b < K; ++b) inst_nnz[b] = static_cast<int64_t>(P[b].A.val.size());
    cta = choose_cta();
    if (cta)
      setup_cta(A, AT);
    else
      setup_grid(A, AT, annz);
    B2P_CUDA(cudaStreamSynchronize(stream));
    stats.upload_seconds = seconds_since(tx);
    stats.setup_seconds = seconds_since(t0);
    stats.kernel_mode = B2P_KERNELS_FUSED;
    stats.precision_used = B2P_PRECISION_FP64;
  }

  // Whether all LPs have one A: equal sizes and equal column pointers, row
  // indices and values (the same arrays, or equal contents).  Scaling
  // depends on A alone, so their scaled operators are then identical too.
  static bool same_operator(const b2p_lp* lps, int num) {
    if (num < 2) return false;
    const b2p_lp& f = lps[0];
    const int32_t nnz = f.start[f.num_cols];
    for (int b = 1; b < num; ++b) {
      const b2p_lp& l = lps[b];
      if (l.num_rows != f.num_rows || l.num_cols != f.num_cols || l.start[l.num_cols] != nnz) return false;
      if (l.start != f.start && std::memcmp(l.start, f.start, sizeof(int32_t) * (f.num_cols + 1)) != 0) return false;
      if (nnz == 0) continue;
      if (l.index != f.index && std::memcmp(l.index, f.index, sizeof(int32_t) * nnz) != 0) return false;
      if (l.value != f.value && std::memcmp(l.value, f.value, sizeof(double) * nnz) != 0) return false;
    }
    return true;
  }

  // ||A|| of every LP on the device (1.01 x the power-iteration estimate, as
  // prepare() computes on the host), bit-identical to the host's.
  void device_power_iterations(int iters) {
    if (M == 0 || N == 0) {
      for (int b = 0; b < K; ++b) P[b].normA = 1.0 * 1.01;
      return;
    }
    std::vector<int32_t> co(K + 1);
    for (int b = 0; b <= K; ++b) co[b] = static_cast<int32_t>(coff[b]);
    int32_t* d_co = upload(co);
    int64_t* d_nnz = upload(inst_nnz_of_lps());
    double* dx = dalloc<double>(N);
    double* dy = dalloc<double>(M);
    double* dz = dalloc<double>(N);
    double* d_nz = dalloc<double>(K);
    double* d_s = dalloc<double>(K);
    int32_t* d_pdone = dalloc<int32_t>(K);
    const unsigned kb = static_cast<unsigned>((K + kBlock - 1) / kBlock);
    k_pi_init<<<blocks(std::max<int64_t>(N, K)), kBlock, 0, stream>>>(N, K, d_cinst, d_co, d_nnz, dx, d_pdone, d_s);
    for (int it = 0; it < iters; ++it) {
      k_spmv<<<blocks(M), kBlock, 0, stream>>>(M, 1, viewA(), dx, dy);
      k_spmv<<<blocks(N), kBlock, 0, stream>>>(N, 1, viewAT(), dy, dz);
      k_pi_norm<<<kb, kBlock, 0, stream>>>(K, d_co, dz, d_pdone, d_nz, d_s);
      k_pi_scale<<<blocks(N), kBlock, 0, stream>>>(N, d_cinst, d_pdone, d_nz, dz, dx);
    }
    B2P_CUDA(cudaGetLastError());
    std::vector<double> s(K);
    B2P_CUDA(cudaMemcpyAsync(s.data(), d_s, sizeof(double) * K, cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaStreamSynchronize(stream));
    for (int b = 0; b < K; ++b) P[b].normA = s[b] * 1.01;
  }
  std::vector<int64_t> inst_nnz_of_lps() const {
    std::vector<int64_t> v(K);
    for (int b = 0; b < K; ++b) v[b] = static_cast<int64_t>(P[b].A.val.size());
    return v;
  }

  // Block-diagonal form: check tables, fused-kernel schedules, autotuner.
  void setup_grid(const HostCsr& A, const HostCsr& AT, int64_t annz) {
    stats.multi_form = B2P_MULTI_GRID;
    // segmented check tables
    auto seg = [&](const std::vector<int64_t>& off, SegTable& tab, int32_t*& dofs, int& g) {
      std::vector<int32_t> inst, beg, end, bo(K + 1, 0);
      for (int b = 0; b < K; ++b) {
        bo[b] = static_cast<int32_t>(inst.size());
        for (int64_t s0 = off[b]; s0 < off[b + 1]; s0 += kSegRows) {
          inst.push_back(b);
          beg.push_back(static_cast<int32_t>(s0));
          end.push_back(static_cast<int32_t>(std::min<int64_t>(off[b + 1], s0 + kSegRows)));
        }
      }
      bo[K] = static_cast<int32_t>(inst.size());
      g = static_cast<int>(inst.size());
      tab = SegTable{upload(inst), upload(beg), upload(end)};
      dofs = upload(bo);
    };
    seg(roff, rtab, d_rblk_off, g_rows);
    seg(coff, ctab, d_cblk_off, g_cols);
    d_prow = dalloc<double>(static_cast<size_t>(std::max(1, g_rows)) * kRowSums);
    d_pcol = dalloc<double>(static_cast<size_t>(std::max(1, g_cols)) * kRowSums);
    d_sums = dalloc<double>(static_cast<size_t>(K) * kNumSums);
    h_sums = static_cast<double*>(PinnedCache::get(sizeof(double) * K * kNumSums));
    h_steps = static_cast<double*>(PinnedCache::get(sizeof(double) * 2 * K));
    h_mask = static_cast<int32_t*>(PinnedCache::get(sizeof(int32_t) * K));
    h_done = static_cast<int32_t*>(PinnedCache::get(sizeof(int32_t) * K));
    // fused-kernel schedules of the concatenated operators
    int per_sm = 0, sms = 0;
    B2P_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dual_binned<4, true, true>, kBlock, 0));
    B2P_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    wave = static_cast<int64_t>(std::max(1, per_sm)) * sms * kBlock;
    rounds = opt.short_row_rounds > 0 ? opt.short_row_rounds : 2;
    const HostBins hbA = make_bins(A, wave, opt.lanes_per_row_a, rounds);
    const HostBins hbT = make_bins(AT, wave, opt.lanes_per_row_at, rounds);
    binsA = device_bins(hbA, M);
    binsT = device_bins(hbT, N);
    ltA = hbA.long_thr;
    ltT = hbT.long_thr;
    hA_ptr = A.ptr;
    hT_ptr = AT.ptr;
    sched_nnz = annz;
    const bool tune = opt.spmv_schedule == B2P_SCHEDULE_TUNED ||
                      (opt.spmv_schedule == B2P_SCHEDULE_AUTO && annz >= (int64_t(1) << 20));
    if (opt.spmv_schedule == B2P_SCHEDULE_TILED) {
      tilesA = device_tiles(hA_ptr, roff, nullptr);
      tilesT = device_tiles(hT_ptr, coff, nullptr);
    } else if (tune) {
      autotune(A, AT);
    }
    stats.lanes_per_row_a = binsA.g;
    stats.lanes_per_row_at = binsT.g;
    stats.schedule_a = tilesA.on ? B2P_SCHEDULE_TILED : B2P_SCHEDULE_BINNED;
    stats.schedule_at = tilesT.on ? B2P_SCHEDULE_TILED : B2P_SCHEDULE_BINNED;
    stats.streaming_a = !tilesA.on && streamA;
    stats.streaming_at = !tilesT.on && streamT;
  }

  // ---- CTA form (pdhg_cta.cuh) ----

  // Static shared memory of k_lp_cta (reduction buffers, up to 1,024 threads) is below this.
  static constexpr int64_t kCtaStaticReserve = 4096;

  // Shared memory one block may give its LP: the device's opt-in per-block
  // maximum less the kernel's static buffers, or the caller's limit.
  int64_t cta_budget() const {
    int optin = 0;
    B2P_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    int64_t b = static_cast<int64_t>(optin) - kCtaStaticReserve;
    if (opt.cta_smem_limit > 0) b = std::min<int64_t>(b, opt.cta_smem_limit);
    return std::max<int64_t>(b, 0);
  }
  int cta_tier(int b, int64_t budget, int esize = 8) const {
    const Prepared& p = P[b];
    const int64_t nnz = static_cast<int64_t>(p.A.val.size());
    if (cta_tier_bytes(kCtaAll, p.m, p.n, nnz, esize) <= budget) return kCtaAll;
    if (cta_tier_bytes(kCtaVectorsPtr, p.m, p.n, nnz, esize) <= budget) return kCtaVectorsPtr;
    if (cta_tier_bytes(kCtaVectors, p.m, p.n, nnz, esize) <= budget) return kCtaVectors;
    return kCtaGlobal;
  }
  // AUTO: the CTA form when every LP fits wholly in one block's shared memory,
  // or when all LPs share one A.
  bool choose_cta() const {
    if (opt.multi_form == B2P_MULTI_GRID) return false;
    if (opt.multi_form == B2P_MULTI_CTA) return true;
    if (opt.multi_form != B2P_MULTI_AUTO) throw Error(B2P_ERR_INVALID, "unknown multi_form");
    if (shared_operator) return true;  // one operator in L2 for every block
    const int64_t budget = cta_budget();
    for (int b = 0; b < K; ++b)
      if (cta_tier(b, budget) != kCtaAll) return false;
    return true;
  }

  void setup_cta(const HostCsr& A, const HostCsr& AT) {
    stats.multi_form = B2P_MULTI_CTA;
    const int64_t budget = cta_budget();
    cta_lps.resize(K);
    cta_smem = 0;
    int n_all = 0, n_vec = 0;
    for (int b = 0; b < K; ++b) {
      const Prepared& p = P[b];
      CtaLp& c = cta_lps[b];
      c.roff = static_cast<int32_t>(roff[b]);
      c.coff = static_cast<int32_t>(coff[b]);
      c.m = p.m;
      c.n = p.n;
      if (shared_operator) {
        c.a_beg = c.t_beg = 0;
        c.aptr_off = c.tptr_off = c.ashift = c.tshift = 0;
      } else {
        c.a_beg = A.ptr[roff[b]];
        c.t_beg = AT.ptr[coff[b]];
        c.aptr_off = c.tshift = static_cast<int32_t>(roff[b]);
        c.tptr_off = c.ashift = static_cast<int32_t>(coff[b]);
      }
      c.nnz = static_cast<int32_t>(p.A.val.size());
      c.tier = cta_tier(b, budget);
      c.tier32 = cta_tier(b, budget, 4);
      c.pad = 0;
      c.it0 = 0;
      c.eta = eta[b];
      c.omega0 = omega0[b];
      c.cnorm = cNorm[b];
      c.rhsnorm = rhsNorm[b];
      c.scale_obj = p.beta * p.gamma;
      cta_smem = std::max(cta_smem, cta_tier_bytes(c.tier, p.m, p.n, c.nnz));
      cta_smem32 = std::max(cta_smem32, cta_tier_bytes(c.tier32, p.m, p.n, c.nnz, 4));
      cta_owner_smem = std::max(cta_owner_smem, cta_owner_bytes(p.m, p.n, c.nnz));
      cta_max_dim = std::max(cta_max_dim, std::max(p.m, p.n));
      n_all += c.tier == kCtaAll;
      n_vec += c.tier == kCtaVectors || c.tier == kCtaVectorsPtr;
    }
    if (cta_owner_smem > budget) cta_owner_smem = 0;
    // largest LPs first, so that the small ones fill in behind them
    std::vector<int32_t> order(K);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return inst_nnz[x] > inst_nnz[y]; });
    d_lps = upload(cta_lps);
    d_order = upload(order);
    host_order = order;
    d_out = dalloc<CtaOut>(K);
    B2P_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&h_stop), sizeof(int32_t), cudaHostAllocMapped));
    *h_stop = 0;
    const int smem = static_cast<int>(cta_smem), osmem = static_cast<int>(cta_owner_smem);
    set_general_attributes<double>(smem);
#define B2P_OWNER_ATTR(NT, R) \
  B2P_CUDA(cudaFuncSetAttribute(k_lp_owner<NT, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, osmem));
    B2P_OWNER_VARIANTS(B2P_OWNER_ATTR)
#undef B2P_OWNER_ATTR
    mixed = opt.precision == B2P_PRECISION_MIXED;
    bool vec_tier = false;  // an LP that reads its operators from global memory and gathers from shared
    for (const CtaLp& c : cta_lps) {
      vec_tier = vec_tier || c.tier == kCtaVectors || c.tier == kCtaVectorsPtr;
      if (mixed) vec_tier = vec_tier || c.tier32 == kCtaVectors || c.tier32 == kCtaVectorsPtr;
    }
    if (opt.cta_layout != B2P_CTA_LAYOUT_CSR && vec_tier) build_sliced(A, AT);
    if (mixed) setup_cta_fp32();
    tune_cta();
    if (mixed) tune_cta_fp32();
    stats.cta_threads = cta_nt;
    stats.cta_owned_per_thread = cta_r > 0 ? cta_r : 0;
    stats.cta_smem_bytes = cta_r > 0 ? cta_owner_smem : cta_smem;
    stats.cta_lps_smem = n_all;
    stats.cta_lps_vectors = n_vec;
    stats.cta_sliced = d_sa_base != nullptr && cta_r <= 0;
  }

  // Sliced-ELL copies of A and A^T for the CTA form: per LP (LP 0 alone when
  // all LPs share one operator), the rows in slices of 32 consecutive local
  // rows -- the rows one warp of the CTA kernel takes together -- each slice
  // as wide as its longest row, entry q of the slice's lane l at
  // slice + 32 q + l.  Not built when the padded copy would exceed 2^31
  // entries.
  void build_sliced(const HostCsr& A, const HostCsr& AT) {
    const int nlp = shared_operator ? std::min(K, 1) : K;
    auto bases = [&](const HostCsr& H, const std::vector<int64_t>& off, bool cols, std::vector<int32_t>& base,
                     int64_t& total) {
      base.assign(H.ptr.size() > 0 ? H.ptr.size() - 1 : 0, 0);
      total = 0;
      for (int b = 0; b < nlp; ++b) {
        const int64_t r0 = off[b], rows = cols ? P[b].n : P[b].m;
        for (int64_t s0 = 0; s0 < rows; s0 += 32) {
          const int64_t s1 = std::min<int64_t>(rows, s0 + 32);
          int32_t w = 0;
          for (int64_t r = s0; r < s1; ++r) w = std::max(w, H.ptr[r0 + r + 1] - H.ptr[r0 + r]);
          if (total + 32 * static_cast<int64_t>(w) >= (int64_t(1) << 31)) return false;
          for (int64_t r = s0; r < s1; ++r) base[r0 + r] = static_cast<int32_t>(total + (r - s0));
          total += 32 * static_cast<int64_t>(w);
        }
      }
      return true;
    };
    std::vector<int32_t> ba, bt;
    if (!bases(A, roff, false, ba, sa_len) || !bases(AT, coff, true, bt, st_len)) {
      sa_len = st_len = 0;
      return;
    }
    d_sa_base = upload(ba);
    d_st_base = upload(bt);
    d_sa_idx = dalloc<int32_t>(std::max<int64_t>(sa_len, 1));
    d_sa_val = dalloc<double>(std::max<int64_t>(sa_len, 1));
    d_st_idx = dalloc<int32_t>(std::max<int64_t>(st_len, 1));
    d_st_val = dalloc<double>(std::max<int64_t>(st_len, 1));
    B2P_CUDA(cudaMemsetAsync(d_sa_idx, 0, sizeof(int32_t) * std::max<int64_t>(sa_len, 1), stream));
    B2P_CUDA(cudaMemsetAsync(d_sa_val, 0, sizeof(double) * std::max<int64_t>(sa_len, 1), stream));
    B2P_CUDA(cudaMemsetAsync(d_st_idx, 0, sizeof(int32_t) * std::max<int64_t>(st_len, 1), stream));
    B2P_CUDA(cudaMemsetAsync(d_st_val, 0, sizeof(double) * std::max<int64_t>(st_len, 1), stream));
    const int32_t ra = nlp == K ? M : P[0].m, rt = nlp == K ? N : P[0].n;
    if (ra) k_to_sliced<<<blocks(ra), kBlock, 0, stream>>>(ra, dA_ptr, dA_idx, dA_val, d_sa_base, d_sa_idx, d_sa_val);
    if (rt) k_to_sliced<<<blocks(rt), kBlock, 0, stream>>>(rt, dT_ptr, dT_idx, dT_val, d_st_base, d_st_idx, d_st_val);
    B2P_CUDA(cudaGetLastError());
  }

  CtaArgs cta_args(double tol, int64_t max_it) const {
    CtaArgs a;
    a.lps = d_lps;
    a.order = d_order;
    a.out = d_out;
    a.A = viewA();
    a.AT = viewAT();
    a.c = v[MC], a.lo = v[MLO], a.up = v[MUP], a.rl = v[MRL], a.ru = v[MRU];
    a.rfac = d_rfac, a.cfac = d_cfac;
    a.xinit = v[MXINIT], a.yinit = v[MYINIT], a.axinit = v[MAXINIT];
    a.x = v[MX], a.xp = v[MXP], a.x0 = v[MX0];
    a.y = v[MY], a.yp = v[MYP], a.y0 = v[MY0];
    a.ax = v[MAX], a.axp = v[MAXP], a.ax0 = v[MAX0];
    a.A32 = dA_val32, a.AT32 = dT_val32;
    a.sa_base = d_sa_base, a.sa_idx = d_sa_idx, a.st_base = d_st_base, a.st_idx = d_st_idx;
    a.sa_val = d_sa_val, a.st_val = d_st_val, a.sa_val32 = d_sa_val32, a.st_val32 = d_st_val32;
    a.x32 = v32[0], a.xp32 = v32[1], a.x032 = v32[2];
    a.y32 = v32[3], a.yp32 = v32[4], a.y032 = v32[5];
    a.ax32 = v32[6], a.axp32 = v32[7], a.ax032 = v32[8];
    a.tol = tol;
    a.rho = opt.reflection;
    a.max_it = max_it;
    a.check_every = opt.check_every;
    a.entry_check = 0;
    a.stall_checks = 0;
    a.pad = 0;
    a.stop = h_stop;
    return a;
  }

  // FP32 run of the mixed form: FP32 copies of the scaled operators' values,
  // FP32 global-tier state, the FP64 run's starting point, kernel attributes.
  void setup_cta_fp32() {
    const size_t annz = static_cast<size_t>(inst_nnz_total());
    dA_val32 = dalloc<float>(annz);
    dT_val32 = dalloc<float>(annz);
    if (annz) {
      k_convert<double, float><<<blocks(static_cast<int64_t>(annz)), kBlock, 0, stream>>>(annz, dA_val, dA_val32);
      k_convert<double, float><<<blocks(static_cast<int64_t>(annz)), kBlock, 0, stream>>>(annz, dT_val, dT_val32);
      B2P_CUDA(cudaGetLastError());
    }
    if (d_sa_base) {
      d_sa_val32 = dalloc<float>(std::max<int64_t>(sa_len, 1));
      d_st_val32 = dalloc<float>(std::max<int64_t>(st_len, 1));
      if (sa_len) k_convert<double, float><<<blocks(sa_len), kBlock, 0, stream>>>(sa_len, d_sa_val, d_sa_val32);
      if (st_len) k_convert<double, float><<<blocks(st_len), kBlock, 0, stream>>>(st_len, d_st_val, d_st_val32);
      B2P_CUDA(cudaGetLastError());
    }
    for (int q = 0; q < 9; ++q) v32[q] = dalloc<float>(q < 3 ? N : M);
    d_x2 = dalloc<double>(N);
    d_y2 = dalloc<double>(M);
    d_ax2 = dalloc<double>(M);
    d_lps2 = dalloc<CtaLp>(K);
    d_order2 = dalloc<int32_t>(K);
    set_general_attributes<float>(static_cast<int>(cta_smem32));
  }
  int64_t inst_nnz_total() const {
    int64_t t = 0;
    for (int b = 0; b < K; ++b) t += inst_nnz[b];
    return t;
  }

// The general kernel's variants: (threads, 0) as compiled, (threads, -1)
// with 1,024 / threads blocks per SM in registers.
#define B2P_GENERAL_VARIANTS(X) X(128, 0, 1) X(256, 0, 1) X(512, 0, 1) X(1024, 0, 1) X(256, -1, 4) X(512, -1, 2)
  template <class T>
  void set_general_attributes(int smem) {
#define B2P_GEN_ATTR(NT, R, MINB) \
  B2P_CUDA(cudaFuncSetAttribute(k_lp_cta<NT, T, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    B2P_GENERAL_VARIANTS(B2P_GEN_ATTR)
#undef B2P_GEN_ATTR
  }
  template <class T>
  void launch_general(int nt, int r, const CtaArgs& a, unsigned grid, size_t smem) {
    bool launched = false;
#define B2P_GEN_LAUNCH(NT, R, MINB)                                 \
  if (!launched && nt == NT && r == R) {                            \
    k_lp_cta<NT, T, MINB><<<grid, NT, smem, stream>>>(a);           \
    launched = true;                                                \
  }
    B2P_GENERAL_VARIANTS(B2P_GEN_LAUNCH)
#undef B2P_GEN_LAUNCH
    if (!launched) throw Error(B2P_ERR_INVALID, "no such CTA kernel variant");
    B2P_CUDA(cudaGetLastError());
  }
  void launch_cta32(int nt, int r, const CtaArgs& a, unsigned grid) {
    launch_general<float>(nt, r, a, grid, static_cast<size_t>(cta_smem32));
  }

  // Threads per block of the FP32 run: each count runs every LP for five
  // check intervals, twice; the fastest is kept (remembered per batch shape).
  void tune_cta_fp32() {
    const auto t0 = Clock::now();
    const std::vector<std::pair<int, int>> cands = general_candidates();
    cta_nt32 = cands.front().first;
    cta_r32 = cands.front().second;
    const int64_t probe = std::min<int64_t>(opt.max_iterations, 5 * static_cast<int64_t>(opt.check_every));
    if (probe <= 0 || cands.size() == 1) return;
    const std::vector<int64_t> key{device, K, cta_max_dim, cta_smem32, inst_nnz_total(), opt.check_every,
                                   opt.cta_threads};
    static std::mutex mu;
    static std::map<std::vector<int64_t>, std::pair<int, int>> chosen;
    {
      std::lock_guard<std::mutex> lock(mu);
      const auto it = chosen.find(key);
      if (it != chosen.end()) {
        cta_nt32 = it->second.first;
        cta_r32 = it->second.second;
        return;
      }
    }
    cudaEvent_t e0, e1;
    B2P_CUDA(cudaEventCreate(&e0));
    B2P_CUDA(cudaEventCreate(&e1));
    double best = INFINITY;
    for (const auto& v : cands) {
      launch_cta32(v.first, v.second, cta_args(-1.0, 1), static_cast<unsigned>(K));
      for (int rep = 0; rep < 2; ++rep) {
        B2P_CUDA(cudaEventRecord(e0, stream));
        launch_cta32(v.first, v.second, cta_args(-1.0, probe), static_cast<unsigned>(K));
        B2P_CUDA(cudaEventRecord(e1, stream));
        B2P_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        B2P_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
          best = ms;
          cta_nt32 = v.first;
          cta_r32 = v.second;
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
      std::lock_guard<std::mutex> lock(mu);
      chosen[key] = {cta_nt32, cta_r32};
    }
    stats.autotune_seconds += seconds_since(t0);
  }

  void launch_cta(int nt, int r, const CtaArgs& a, int lps = -1) {
    const unsigned grid = static_cast<unsigned>(lps < 0 ? K : lps);
    if (r <= 0) {
      launch_general<double>(nt, r, a, grid, static_cast<size_t>(cta_smem));
    } else {
      const size_t smem = static_cast<size_t>(cta_owner_smem);
      bool launched = false;
#define B2P_OWNER_LAUNCH(NT, R)                                 \
  if (!launched && nt == NT && r == R) {                        \
    k_lp_owner<NT, R><<<grid, NT, smem, stream>>>(a);           \
    launched = true;                                            \
  }
      B2P_OWNER_VARIANTS(B2P_OWNER_LAUNCH)
#undef B2P_OWNER_LAUNCH
      if (!launched) throw Error(B2P_ERR_INVALID, "no such CTA kernel variant");
    }
    B2P_CUDA(cudaGetLastError());
  }

  // The general kernel's variants allowed by the options (threads, 0 / -1).
  std::vector<std::pair<int, int>> general_candidates() const {
    std::vector<std::pair<int, int>> c;
#define B2P_GEN_CAND(NT, R, MINB) \
  if (opt.cta_threads == 0 || opt.cta_threads == NT) c.emplace_back(NT, R);
    B2P_GENERAL_VARIANTS(B2P_GEN_CAND)
#undef B2P_GEN_CAND
    return c;
  }

  // Kernel variants that can run this batch: the general kernel at 128, 256,
  // 512 and 1,024 threads (256 and 512 also compiled for 1,024 threads per
  // SM), and the owner kernel where every LP's rows and columns fit R per
  // thread and its data fits in shared memory.
  std::vector<std::pair<int, int>> cta_candidates() const {
    const int want = opt.cta_kernel;  // B2P_CTA_*
    if (want < B2P_CTA_AUTO || want > B2P_CTA_OWNER2) throw Error(B2P_ERR_INVALID, "unknown cta_kernel");
    std::vector<std::pair<int, int>> c;
    if (want == B2P_CTA_AUTO || want == B2P_CTA_GENERAL) c = general_candidates();
    if (cta_owner_smem > 0 && want != B2P_CTA_GENERAL && opt.precision != B2P_PRECISION_MIXED) {
#define B2P_OWNER_CAND(NT, R)                                                                        \
  if ((opt.cta_threads == 0 || opt.cta_threads == NT) && cta_max_dim <= NT * R &&                    \
      (want == B2P_CTA_AUTO || want == B2P_CTA_OWNER1 + R - 1))                                      \
    c.emplace_back(NT, R);
      B2P_OWNER_VARIANTS(B2P_OWNER_CAND)
#undef B2P_OWNER_CAND
    }
    if (c.empty()) throw Error(B2P_ERR_INVALID, "no CTA kernel variant fits these LPs and options");
    return c;
  }

  // Variant choice: each candidate runs every LP for five check intervals
  // (tolerance -1: no LP stops early), twice, and the fastest is kept.  The
  // choice is remembered for the process per batch shape (device, LP count,
  // largest dimension, shared-memory sizes, nonzeros, options), so repeated
  // batches of one family pay for it once.
  void tune_cta() {
    const auto t0 = Clock::now();
    if (opt.cta_threads != 0 && opt.cta_threads != 128 && opt.cta_threads != 256 && opt.cta_threads != 512 &&
        opt.cta_threads != 1024)
      throw Error(B2P_ERR_INVALID, "cta_threads must be 128, 256, 512 or 1024");
    const std::vector<std::pair<int, int>> cands = cta_candidates();
    cta_nt = cands.front().first;
    cta_r = cands.front().second;
    const int64_t probe = std::min<int64_t>(opt.max_iterations, 5 * static_cast<int64_t>(opt.check_every));
    if (probe <= 0 || cands.size() == 1) return;
    int64_t total_nnz = 0;
    for (const CtaLp& c : cta_lps) total_nnz += c.nnz;
    const std::vector<int64_t> key{device, K, cta_max_dim, cta_smem, cta_owner_smem, total_nnz, opt.cta_threads,
                                   opt.cta_kernel, opt.check_every};
    static std::mutex mu;
    static std::map<std::vector<int64_t>, std::pair<int, int>> chosen;
    {
      std::lock_guard<std::mutex> lock(mu);
      const auto it = chosen.find(key);
      if (it != chosen.end()) {
        cta_nt = it->second.first;
        cta_r = it->second.second;
        return;
      }
    }
    cudaEvent_t e0, e1;
    B2P_CUDA(cudaEventCreate(&e0));
    B2P_CUDA(cudaEventCreate(&e1));
    double best = INFINITY;
    for (const auto& v : cands) {
      launch_cta(v.first, v.second, cta_args(-1.0, 1));  // first launch of this kernel: module load
      for (int rep = 0; rep < 2; ++rep) {
        B2P_CUDA(cudaEventRecord(e0, stream));
        launch_cta(v.first, v.second, cta_args(-1.0, probe));
        B2P_CUDA(cudaEventRecord(e1, stream));
        B2P_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        B2P_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
          best = ms;
          cta_nt = v.first;
          cta_r = v.second;
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
      std::lock_guard<std::mutex> lock(mu);
      chosen[key] = {cta_nt, cta_r};
    }
    stats.autotune_seconds = seconds_since(t0);
  }

  // The whole solve is one launch (mixed precision: two, the FP32 run of
  // every LP and the FP64 run from its point); the host only watches the
  // deadline and the cancel flag and raises the mapped stop flag (read at
  // every check).
  void solve_cta(Clock::time_point deadline_start) {
    const auto t_solve = Clock::now();
    results.assign(K, b2p_result{});
    weights.assign(K, 1.0);
    xs.assign(K, {});
    ys.assign(K, {});
    *reinterpret_cast<volatile int32_t*>(h_stop) = 0;
    bool raised = false;
    auto wait_for = [&](cudaEvent_t ev) {
      if (opt.time_limit <= 0 && !opt.cancel_flag) {
        B2P_CUDA(cudaEventSynchronize(ev));
        return;
      }
      for (;;) {
        const cudaError_t q = cudaEventQuery(ev);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) B2P_CUDA(q);
        const bool expired = (opt.cancel_flag && *opt.cancel_flag) ||
                             (opt.time_limit > 0 && seconds_since(deadline_start) >= opt.time_limit);
        if (expired && !raised) {
          *reinterpret_cast<volatile int32_t*>(h_stop) = 1;
          raised = true;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(100));
      }
    };
    std::vector<CtaOut> out(K), out32;
    std::vector<char> ran32(K, 0);
    B2P_CUDA(cudaEventRecord(ev_start, stream));
    if (!mixed) {
      launch_cta(cta_nt, cta_r, cta_args(opt.tolerance, opt.max_iterations));
      B2P_CUDA(cudaEventRecord(ev_stop, stream));
      launches = 1;
      wait_for(ev_stop);
    } else {
      // FP32 run of every LP
      CtaArgs a1 = cta_args(opt.tolerance, opt.max_iterations);
      a1.stall_checks = kStallChecks;
      launch_cta32(cta_nt32, cta_r32, a1, static_cast<unsigned>(K));
      B2P_CUDA(cudaEventRecord(ev_stop, stream));
      wait_for(ev_stop);
      out32.resize(K);
      B2P_CUDA(cudaMemcpyAsync(out32.data(), d_out, sizeof(CtaOut) * K, cudaMemcpyDeviceToHost, stream));
      B2P_CUDA(cudaStreamSynchronize(stream));
      bytes_down += static_cast<int64_t>(sizeof(CtaOut) * K);
      // FP64 run from each LP's FP32 point (measured first), as from a
      // restart: its primal weight, the iteration count carried on
      std::vector<CtaLp> lps2 = cta_lps;
      std::vector<int32_t> order2;
      for (int b = 0; b < K; ++b) {
        const CtaOut& o = out32[b];
        if (o.status == B2P_STATUS_TIME_LIMIT) continue;
        lps2[b].omega0 = o.omega;
        lps2[b].it0 = o.status == B2P_STATUS_ITERATION_LIMIT ? o.iterations : o.iterations + 1;
        ran32[b] = 1;
      }
      for (int b = 0; b < K; ++b) {
        const int lp = host_order[b];
        if (ran32[lp]) order2.push_back(lp);
      }
      launches = 1;
      if (!order2.empty()) {
        B2P_CUDA(cudaMemcpyAsync(d_lps2, lps2.data(), sizeof(CtaLp) * K, cudaMemcpyHostToDevice, stream));
        B2P_CUDA(cudaMemcpyAsync(d_order2, order2.data(), sizeof(int32_t) * order2.size(), cudaMemcpyHostToDevice,
                                 stream));
        bytes_up += static_cast<int64_t>(sizeof(CtaLp) * K + sizeof(int32_t) * order2.size());
        if (N) k_clamp_to_bounds<<<blocks(N), kBlock, 0, stream>>>(N, v[MXP], v[MLO], v[MUP], d_x2);
        if (M) {
          B2P_CUDA(cudaMemcpyAsync(d_y2, v[MYP], sizeof(double) * M, cudaMemcpyDeviceToDevice, stream));
          k_spmv<<<blocks(M), kBlock, 0, stream>>>(M, 1, viewA(), d_x2, d_ax2);
        }
        B2P_CUDA(cudaGetLastError());
        CtaArgs a2 = cta_args(opt.tolerance, opt.max_iterations);
        a2.lps = d_lps2;
        a2.order = d_order2;
        a2.xinit = d_x2;
        a2.yinit = d_y2;
        a2.axinit = d_ax2;
        a2.entry_check = 1;
        launch_cta(cta_nt, cta_r, a2, static_cast<int>(order2.size()));
        launches += 3;
      }
      B2P_CUDA(cudaEventRecord(ev_stop, stream));
      wait_for(ev_stop);
    }
    float ms = 0;
    B2P_CUDA(cudaEventElapsedTime(&ms, ev_start, ev_stop));
    stats.kernel_seconds = ms / 1000.0;
    std::vector<double> xp(N), yp(M);
    B2P_CUDA(cudaMemcpyAsync(out.data(), d_out, sizeof(CtaOut) * K, cudaMemcpyDeviceToHost, stream));
    if (N) B2P_CUDA(cudaMemcpyAsync(xp.data(), v[MXP], sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
    if (M) B2P_CUDA(cudaMemcpyAsync(yp.data(), v[MYP], sizeof(double) * M, cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaStreamSynchronize(stream));
    bytes_down += static_cast<int64_t>(sizeof(CtaOut) * K + sizeof(double) * (static_cast<int64_t>(N) + M));
    int64_t its = 0, its32 = 0;
    stats.restarts = 0;
    for (int b = 0; b < K; ++b) {
      CtaOut o = out[b];
      if (mixed) {
        // an LP without an FP64 run keeps its FP32 result; one with both
        // counts the switch as a restart
        if (!ran32[b]) o = out32[b];
        else o.restarts += out32[b].restarts + 1;
        its32 = std::max<int64_t>(its32, out32[b].iterations);
        if (o.status == kCtaStalled) o.status = B2P_STATUS_ITERATION_LIMIT;
      }
      store_result(b, o.status, o.rel_kkt, o.pobj, o.dobj, o.iterations, xp.data() + coff[b], yp.data() + roff[b]);
      weights[b] = o.omega * P[b].gamma / P[b].beta;
      its = std::max<int64_t>(its, o.iterations + (o.status == B2P_STATUS_OPTIMAL ? 1 : 0));
      stats.restarts += o.restarts;
    }
    stats.iterations = its;
    stats.fp32_iterations = its32;
    stats.precision_used = mixed ? B2P_PRECISION_MIXED : B2P_PRECISION_FP64;
    stats.primal_weight = K ? out[0].omega : 1.0;
    stats.solve_seconds = seconds_since(t_solve);
    stats.kernel_launches = launches;
    stats.bytes_uploaded = bytes_up;
    stats.bytes_downloaded = bytes_down;
  }

  // Warm starts of some instances (original space); others keep the cold start.
  // Warm start of the next solve: points in the original space (x projected
  // onto the bounds) and primal weights in the original space's units
  // (w = omega gamma / beta of the scaled problem); NULL arrays, NULL entries
  // and weights that are not finite and positive leave that part cold.
  void set_start(const double* const* xst, const double* const* yst, const double* wst = nullptr) {
    if (wst) {
      for (int b = 0; b < K; ++b)
        if (std::isfinite(wst[b]) && wst[b] > 0) omega0[b] = wst[b] * P[b].beta / P[b].gamma;
      if (cta) {
        for (int b = 0; b < K; ++b) cta_lps[b].omega0 = omega0[b];
        B2P_CUDA(cudaMemcpyAsync(d_lps, cta_lps.data(), sizeof(CtaLp) * K, cudaMemcpyHostToDevice, stream));
        B2P_CUDA(cudaStreamSynchronize(stream));
      }
    }
    if (M) B2P_CUDA(cudaMemsetAsync(v[MYINIT], 0, sizeof(double) * M, stream));
    if (!xst && !yst) return;
    std::vector<double> lo(N), up(N), x0(N), y0(M, 0.0);
    if (N) {
      B2P_CUDA(cudaMemcpyAsync(lo.data(), v[MLO], sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
      B2P_CUDA(cudaMemcpyAsync(up.data(), v[MUP], sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
      B2P_CUDA(cudaMemcpyAsync(x0.data(), v[MXINIT], sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
    }
    B2P_CUDA(cudaStreamSynchronize(stream));
    for (int b = 0; b < K; ++b) {
      const Prepared& p = P[b];
      if (xst && xst[b])
        for (int32_t j = 0; j < p.n; ++j) {
          const size_t t = static_cast<size_t>(coff[b] + j);
          x0[t] = smin(smax(xst[b][j] / p.Cs[j] / p.beta, lo[t]), up[t]);
        }
      if (yst && yst[b])
        for (int32_t i = 0; i < p.m; ++i) y0[static_cast<size_t>(roff[b] + i)] = yst[b][i] / p.R[i] / p.gamma;
    }
    if (N) B2P_CUDA(cudaMemcpyAsync(v[MXINIT], x0.data(), sizeof(double) * N, cudaMemcpyHostToDevice, stream));
    if (M) {
      B2P_CUDA(cudaMemcpyAsync(v[MYINIT], y0.data(), sizeof(double) * M, cudaMemcpyHostToDevice, stream));
      k_spmv<<<blocks(M), kBlock, 0, stream>>>(M, 1, viewA(), v[MXINIT], v[MAXINIT]);
      B2P_CUDA(cudaGetLastError());
    }
    B2P_CUDA(cudaStreamSynchronize(stream));
  }

  // Tile schedule of an operator over the live LPs (all when done == NULL).
  TileSched device_tiles(const std::vector<int32_t>& ptr, const std::vector<int64_t>& off,
                         const std::vector<char>* done) {
    const HostTiles h = make_tiles(ptr, off, done);
    TileSched t;
    t.on = true;
    t.ts.tiles = upload(h.tiles);
    t.ts.inst = upload(h.inst);
    t.ts.n_tiles = static_cast<int32_t>(h.tiles.size());
    t.ts.grid = 0;  // set below, after the long-row blocks are known
    RowBins& lb = t.longb;
    lb.long_rows = upload(h.long_rows);
    lb.vlong_rows = upload(h.vlong_rows);
    lb.short_rows = nullptr;
    lb.n_short = 0;
    lb.n_long = static_cast<int32_t>(h.long_rows.size());
    lb.n_vlong = static_cast<int32_t>(h.vlong_rows.size());
    lb.long_thr = kTileRowMax;
    lb.vlong_blocks = lb.n_vlong;
    lb.long_blocks = (lb.n_long + kBlock / 32 - 1) / (kBlock / 32);
    lb.short_blocks = 0;
    lb.g = 1;
    t.ts.grid = std::max(1, lb.vlong_blocks + lb.long_blocks + (t.ts.n_tiles + kBlock / 32 - 1) / (kBlock / 32));
    return t;
  }

  // The state every solve starts from (also the autotuner's playground).
  void reset_state() {
    auto cp = [&](int dst, int src, int64_t len) {
      if (len) B2P_CUDA(cudaMemcpyAsync(v[dst], v[src], len * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    };
    cp(MX, MXINIT, N);
    cp(MX0, MXINIT, N);
    cp(MAX, MAXINIT, M);
    cp(MAX0, MAXINIT, M);
    cp(MY, MYINIT, M);
    cp(MY0, MYINIT, M);
    B2P_CUDA(cudaMemsetAsync(d_it_base, 0, sizeof(int64_t), stream));
    B2P_CUDA(cudaMemsetAsync(d_restart_at, 0, sizeof(int64_t) * K, stream));
    B2P_CUDA(cudaMemsetAsync(d_done, 0, sizeof(int32_t) * K, stream));
    upload_steps(omega0);
  }

  // One primal / dual / A^T y launch set with the operator's current schedule.
  void enqueue_primal(bool halpern, const IterClock& ck) {
    if (!N) return;
    const double rho = opt.reflection;
    const CsrView AT = viewAT();
    const InstanceMap im{d_cinst, d_done};
    if (tilesT.on) {
      const RowBins& lb = tilesT.longb;
      const unsigned g = static_cast<unsigned>(tilesT.ts.grid);
#define B2P_PT(H, MB)                                                                                            \
  launch(k_primal_tiled<H, true, MB>, g, stream, true, AT, tilesT.ts, lb, v[MY], v[MC], v[MLO], v[MUP], v[MX], \
         v[MXP], v[MX0], d_tau, ck, rho, im)
      if (tilesT.capped) {
        if (halpern) B2P_PT(true, 4);
        else B2P_PT(false, 4);
      } else {
        if (halpern) B2P_PT(true, 1);
        else B2P_PT(false, 1);
      }
#undef B2P_PT
      return;
    }
    const unsigned gp = bin_grid(binsT);
#define B2P_MPRIMAL_S(G, H, S)                                                                              \
  launch(k_primal_binned<G, H, true, S>, gp, stream, true, AT, binsT, v[MY], v[MC], v[MLO], v[MUP], v[MX], v[MXP], \
         v[MX0], d_tau, ck, rho, im);
#define B2P_MPRIMAL(G)                    \
  if (streamT) {                          \
    if (halpern) B2P_MPRIMAL_S(G, true, true) \
    else B2P_MPRIMAL_S(G, false, true)    \
  } else {                                \
    if (halpern) B2P_MPRIMAL_S(G, true, false) \
    else B2P_MPRIMAL_S(G, false, false)   \
  }
    B2P_G_SWITCH(binsT.g, B2P_MPRIMAL)
#undef B2P_MPRIMAL
#undef B2P_MPRIMAL_S
  }

  void enqueue_dual(bool halpern, const IterClock& ck) {
    if (!M) return;
    const double rho = opt.reflection;
    const CsrView A = viewA();
    const InstanceMap im{d_rinst, d_done};
    if (tilesA.on) {
      const RowBins& lb = tilesA.longb;
      const unsigned g = static_cast<unsigned>(tilesA.ts.grid);
#define B2P_DT(H, MB)                                                                                             \
  launch(k_dual_tiled<H, true, MB>, g, stream, true, A, tilesA.ts, lb, v[MXP], v[MRL], v[MRU], v[MY], v[MYP],   \
         v[MY0], v[MAX], v[MAXP], v[MAX0], d_sigma, ck, rho, im)
      if (tilesA.capped) {
        if (halpern) B2P_DT(true, 4);
        else B2P_DT(false, 4);
      } else {
        if (halpern) B2P_DT(true, 1);
        else B2P_DT(false, 1);
      }
#undef B2P_DT
      return;
    }
    const unsigned gd = bin_grid(binsA);
#define B2P_MDUAL_S(G, H, S)                                                                                 \
  launch(k_dual_binned<G, H, true, S>, gd, stream, true, A, binsA, v[MXP], v[MRL], v[MRU], v[MY], v[MYP], v[MY0], \
         v[MAX], v[MAXP], v[MAX0], d_sigma, ck, rho, im);
#define B2P_MDUAL(G)                      \
  if (streamA) {                          \
    if (halpern) B2P_MDUAL_S(G, true, true) \
    else B2P_MDUAL_S(G, false, true)      \
  } else {                                \
    if (halpern) B2P_MDUAL_S(G, true, false) \
    else B2P_MDUAL_S(G, false, false)     \
  }
    B2P_G_SWITCH(binsA.g, B2P_MDUAL)
#undef B2P_MDUAL
#undef B2P_MDUAL_S
  }

  void enqueue_aty() {
    if (!N) return;
    const CsrView AT = viewAT();
    const InstanceMap im{d_cinst, d_done};
    if (tilesT.on) {
      launch(k_spmv_tiled<true>, static_cast<unsigned>(tilesT.ts.grid), stream, false, AT, tilesT.ts, tilesT.longb,
             v[MYP], v[MATYP], im);
      return;
    }
    const unsigned gp = bin_grid(binsT);
#define B2P_MATY(G) launch(k_spmv_binned<G, true>, gp, stream, false, AT, binsT, v[MYP], v[MATYP], im);
    B2P_G_SWITCH(binsT.g, B2P_MATY)
#undef B2P_MATY
  }

  // Kernel launches of one iteration / of the A^T y+ product.
  static int sched_launches(const TileSched&) { return 1; }

  // Autotuner: for A^T (primal kernel) and A (dual kernel) separately, time
  // every binned schedule (1..32 lanes per short row, with cached or
  // evict-first streaming loads) and the tile schedule on the device, from the
  // solve's starting state, and keep the fastest.
  // The choice per operator: binned (lanes per short row, streaming) or tiles
  // (capped or not).  Remembered for the process per batch shape, so repeated
  // solves of a batch (or of batches of one family) time the candidates once.
  struct SchedChoice {
    int g = 1;
    bool streaming = false, tiles = false, capped = false;
  };
  void apply_choice(const HostCsr& Op, int32_t rows, const SchedChoice& c, RowBins& bins, TileSched& tiles,
                    bool& streaming, const std::vector<int32_t>& ptr, const std::vector<int64_t>& off) {
    if (c.tiles) {
      tiles = device_tiles(ptr, off, nullptr);
      tiles.capped = c.capped;
    } else {
      tiles.on = false;
      streaming = c.streaming;
      bins = device_bins(make_bins(Op, wave, c.g, rounds), rows);
    }
  }
  static SchedChoice choice_of(const RowBins& bins, const TileSched& tiles, bool streaming) {
    SchedChoice c;
    c.g = bins.g;
    c.streaming = streaming;
    c.tiles = tiles.on;
    c.capped = tiles.capped;
    return c;
  }

  void autotune(const HostCsr& A, const HostCsr& AT) {
    const auto t0 = Clock::now();
    int64_t annz = static_cast<int64_t>(hA_ptr.empty() ? 0 : hA_ptr.back());
    const std::vector<int64_t> key{device, K, M, N, annz, opt.spmv_schedule, rounds, opt.lanes_per_row_a,
                                   opt.lanes_per_row_at};
    static std::mutex mu;
    static std::map<std::vector<int64_t>, std::pair<SchedChoice, SchedChoice>> chosen;
    {
      std::lock_guard<std::mutex> lock(mu);
      const auto it = chosen.find(key);
      if (it != chosen.end()) {
        apply_choice(AT, N, it->second.first, binsT, tilesT, streamT, hT_ptr, coff);
        apply_choice(A, M, it->second.second, binsA, tilesA, streamA, hA_ptr, roff);
        ltA = binsA.long_thr;
        ltT = binsT.long_thr;
        stats.autotune_seconds = seconds_since(t0);
        return;
      }
    }
    reset_state();
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
      return ms / 3.0;
    };
    auto tune = [&](const HostCsr& Op, int32_t rows, RowBins& bins, TileSched& tiles, bool& streaming,
                    const std::vector<int32_t>& ptr, const std::vector<int64_t>& off, auto&& enq) {
      double best = INFINITY;
      int best_g = bins.g;
      bool best_s = false;
      tiles.on = false;
      for (int g = 1; g <= 32; g *= 2) {
        bins = device_bins(make_bins(Op, wave, g, rounds), rows);
        for (int st = 0; st < 2; ++st) {
          streaming = st != 0;
          const double t = timed(enq);
          if (t < best) {
            best = t;
            best_g = g;
            best_s = streaming;
          }
        }
      }
      tiles = device_tiles(ptr, off, nullptr);
      double tbest = INFINITY;
      bool tcap = false;
      for (int cap = 0; cap < 2; ++cap) {
        tiles.capped = cap != 0;
        const double tt = timed(enq);
        if (tt < tbest) {
          tbest = tt;
          tcap = tiles.capped;
        }
      }
      if (tbest < best) {  // keep the tiles
        tiles.capped = tcap;
        return;
      }
      tiles.on = false;
      streaming = best_s;
      bins = device_bins(make_bins(Op, wave, best_g, rounds), rows);
    };
    tune(AT, N, binsT, tilesT, streamT, hT_ptr, coff, [&] { enqueue_primal(true, ck); });
    tune(A, M, binsA, tilesA, streamA, hA_ptr, roff, [&] { enqueue_dual(true, ck); });
    ltA = binsA.long_thr;
    ltT = binsT.long_thr;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
      std::lock_guard<std::mutex> lock(mu);
      chosen[key] = {choice_of(binsT, tilesT, streamT), choice_of(binsA, tilesA, streamA)};
    }
    stats.autotune_seconds = seconds_since(t0);
  }

  RowBins device_bins(const HostBins& hb, int32_t rows) {
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
    b.short_blocks = static_cast<int32_t>((static_cast<int64_t>(rows) * hb.g + kBlock - 1) / kBlock);
    b.g = hb.g;
    return b;
  }
  // Schedule over the rows of live instances only (instance compaction).
  RowBins live_bins(const std::vector<int32_t>& ptr, const std::vector<int64_t>& off, const std::vector<char>& done,
                    int g, int lt) {
    std::vector<int32_t> sh, lg, vl;
    for (int b = 0; b < K; ++b) {
      if (done[b]) continue;
      for (int64_t i = off[b]; i < off[b + 1]; ++i) {
        const int32_t len = ptr[i + 1] - ptr[i];
        if (len > kVeryLongRow)
          vl.push_back(static_cast<int32_t>(i));
        else if (len > lt)
          lg.push_back(static_cast<int32_t>(i));
        else
          sh.push_back(static_cast<int32_t>(i));
      }
    }
    RowBins r{};
    r.long_rows = upload(lg);
    r.vlong_rows = upload(vl);
    r.short_rows = upload(sh);
    r.n_short = static_cast<int32_t>(sh.size());
    r.n_long = static_cast<int32_t>(lg.size());
    r.n_vlong = static_cast<int32_t>(vl.size());
    r.long_thr = lt;
    r.vlong_blocks = r.n_vlong;
    r.long_blocks = (r.n_long + kBlock / 32 - 1) / (kBlock / 32);
    r.short_blocks = static_cast<int32_t>((static_cast<int64_t>(r.n_short) * g + kBlock - 1) / kBlock);
    r.g = g;
    return r;
  }

  // Rebuild the schedules when the live instances hold less than half of the
  // nonzeros the current ones cover; the graphs are captured again.
  void maybe_compact(const std::vector<char>& done) {
    int64_t live = 0;
    for (int b = 0; b < K; ++b)
      if (!done[b]) live += inst_nnz[b];
    if (live == 0 || 2 * live >= sched_nnz) return;
    B2P_CUDA(cudaStreamSynchronize(stream));
    if (tilesA.on) {
      const bool cap = tilesA.capped;
      tilesA = device_tiles(hA_ptr, roff, &done);
      tilesA.capped = cap;
    }
    else binsA = live_bins(hA_ptr, roff, done, binsA.g, ltA);
    if (tilesT.on) {
      const bool cap = tilesT.capped;
      tilesT = device_tiles(hT_ptr, coff, &done);
      tilesT.capped = cap;
    }
    else binsT = live_bins(hT_ptr, coff, done, binsT.g, ltT);
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    for (auto& g : graph_defs) cudaGraphDestroy(g.second);
    graphs.clear();
    graph_defs.clear();
    sched_nnz = live;
    ++compactions;
  }

  static unsigned bin_grid(const RowBins& b) {
    return static_cast<unsigned>(std::max(1, b.vlong_blocks + b.long_blocks + b.short_blocks));
  }

  void upload_steps(const std::vector<double>& omega) {
    for (int b = 0; b < K; ++b) {
      h_steps[b] = eta[b] / omega[b];
      h_steps[K + b] = eta[b] * omega[b];
    }
    B2P_CUDA(cudaMemcpyAsync(d_tau, h_steps, sizeof(double) * K, cudaMemcpyHostToDevice, stream));
    B2P_CUDA(cudaMemcpyAsync(d_sigma, h_steps + K, sizeof(double) * K, cudaMemcpyHostToDevice, stream));
    bytes_up += static_cast<int64_t>(2 * K * sizeof(double));
  }

  void enqueue_interval(int L) {
    const double rho = opt.reflection;
    for (int l = 0; l < L; ++l) {
      const IterClock ck{d_it_base, d_restart_at, l};
      enqueue_primal(l != L - 1, ck);
      enqueue_dual(l != L - 1, ck);
    }
    enqueue_aty();
    const IterClock ck{d_it_base, d_restart_at, L - 1};
    if (g_rows)
      k_check_rows_multi<<<g_rows, kBlock, 0, stream>>>(rtab, d_done, v[MAXP], v[MRL], v[MRU], v[MYP], v[MY], v[MY0],
                                                        d_rfac, d_prow);
    if (g_cols)
      k_check_cols_multi<<<g_cols, kBlock, 0, stream>>>(ctab, d_done, v[MATYP], v[MXP], v[MX], v[MX0], v[MC], v[MLO],
                                                        v[MUP], d_cfac, d_pcol);
    k_halpern_all_multi<<<blocks(static_cast<int64_t>(N) + M), kBlock, 0, stream>>>(
        N, M, d_cinst, d_rinst, d_done, v[MX], v[MXP], v[MX0], v[MY], v[MYP], v[MY0], v[MAX], v[MAXP], v[MAX0], ck, rho);
    k_check_finalize_multi<<<K, kBlock, 0, stream>>>(d_rblk_off, d_cblk_off, d_done, d_prow, d_pcol, d_sums, d_it_base,
                                                     L);
    B2P_CUDA(cudaGetLastError());
    B2P_CUDA(cudaMemcpyAsync(h_sums, d_sums, sizeof(double) * K * kNumSums, cudaMemcpyDeviceToHost, stream));
  }

  void run_interval(int L) {
    if (opt.use_graphs) {
      auto it = graphs.find(L);
      if (it == graphs.end()) {
        const auto tg = Clock::now();
        cudaGraph_t g;
        B2P_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
          enqueue_interval(L);
        } catch (...) {
          cudaStreamEndCapture(stream, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        B2P_CUDA(cudaStreamEndCapture(stream, &g));
        cudaGraphExec_t ge;
        B2P_CUDA(cudaGraphInstantiate(&ge, g, 0));
        graph_defs[L] = g;
        it = graphs.emplace(L, ge).first;
        stats.graph_seconds += seconds_since(tg);
      }
      B2P_CUDA(cudaGraphLaunch(it->second, stream));
    } else {
      enqueue_interval(L);
    }
    launches += static_cast<int64_t>(L) * (sched_launches(tilesT) + sched_launches(tilesA)) +
                sched_launches(tilesT) + 4;
    bytes_down += static_cast<int64_t>(sizeof(double) * K * kNumSums);
  }

  void extract(int b, int status, double relKkt, double pobj, double dobj, int64_t it) {
    const Prepared& p = P[b];
    std::vector<double> xp(p.n), yp(p.m);
    if (p.n)
      B2P_CUDA(cudaMemcpyAsync(xp.data(), v[MXP] + coff[b], sizeof(double) * p.n, cudaMemcpyDeviceToHost, stream));
    if (p.m)
      B2P_CUDA(cudaMemcpyAsync(yp.data(), v[MYP] + roff[b], sizeof(double) * p.m, cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaStreamSynchronize(stream));
    bytes_down += static_cast<int64_t>(sizeof(double) * (p.n + p.m));
    store_result(b, status, relKkt, pobj, dobj, it, xp.data(), yp.data());
  }

  // Unscaled answer of instance b from its scaled x+ and y+ (src/pdhg/pdhg.cpp:668-680).
  void store_result(int b, int status, double relKkt, double pobj, double dobj, int64_t it, const double* xp,
                    const double* yp) {
    const Prepared& p = P[b];
    xs[b].resize(p.n);
    ys[b].resize(p.m);
    for (int32_t j = 0; j < p.n; ++j) xs[b][j] = xp[j] * p.Cs[j] * p.beta;
    for (int32_t i = 0; i < p.m; ++i) ys[b][i] = yp[i] * p.R[i] * p.gamma;
    b2p_result& r = results[b];
    r.status = status;
    r.iterations = it;
    r.relative_kkt = relKkt;
    r.objective = pobj + p.offset;
    r.dual_objective = dobj + p.offset;
  }

  // runPdhg's loop for every instance at once (src/pdhg/pdhg.cpp:560-687).
  void solve(Clock::time_point deadline_start) {
    B2P_CUDA(cudaSetDevice(device));
    if (cta) {
      solve_cta(deadline_start);
      return;
    }
    const auto t_solve = Clock::now();
    launches = 0;
    reset_state();
    std::vector<double> omega = omega0;
    results.assign(K, b2p_result{});
    weights.assign(K, 1.0);
    xs.assign(K, {});
    ys.assign(K, {});
    stats.restarts = 0;
    std::vector<char> done(K, 0);
    std::vector<RestartTracker> restarts(K);
    int remaining = K;
    const int cE = opt.check_every;
    auto expired = [&]() {
      if (opt.cancel_flag && *opt.cancel_flag) return true;
      return opt.time_limit > 0 && seconds_since(deadline_start) >= opt.time_limit;
    };
    B2P_CUDA(cudaEventRecord(ev_start, stream));
    int64_t it = 0;
    bool expiredStop = false;
    while (it < opt.max_iterations) {
      const int L = static_cast<int>(std::min<int64_t>(cE, opt.max_iterations - it));
      run_interval(L);
      B2P_CUDA(cudaStreamSynchronize(stream));
      it += L - 1;
      bool anyRestart = false, anyDone = false;
      for (int b = 0; b < K; ++b) h_mask[b] = 0;
      for (int b = 0; b < K; ++b) {
        if (done[b]) continue;
        const double* s = h_sums + static_cast<size_t>(b) * kNumSums;
        const double scaleObj = P[b].beta * P[b].gamma;
        const double pobj = s[CS_POBJ] * scaleObj;
        const double dobj = (s[CS_ROW_DOBJ] + s[CS_COL_DOBJ]) * scaleObj;
        const double relP = std::sqrt(s[CS_ROW_RES2]) / (1.0 + rhsNorm[b]);
        const double relD = std::sqrt(s[CS_COL_RES2]) / (1.0 + cNorm[b]);
        const double gap = std::fabs(pobj - dobj) / (1.0 + std::fabs(pobj) + std::fabs(dobj));
        if (relP <= opt.tolerance && relD <= opt.tolerance && gap <= opt.tolerance) {
          extract(b, B2P_STATUS_OPTIMAL, smax(relP, smax(relD, gap)), pobj, dobj, it);
          weights[b] = omega[b] * P[b].gamma / P[b].beta;
          done[b] = 1;
          anyDone = true;
          --remaining;
          continue;
        }
        if (restarts[b].due(omega[b], s, it, cE)) {
          h_mask[b] = 1;
          anyRestart = true;
          restarts[b].restart(omega[b], s);
          stats.restarts++;
        }
      }
      if (anyRestart) upload_steps(omega);
      if (remaining == 0) break;
      if (expired()) {
        expiredStop = true;
        break;
      }
      if (anyDone) {
        for (int b = 0; b < K; ++b) h_done[b] = done[b];
        B2P_CUDA(cudaMemcpyAsync(d_done, h_done, sizeof(int32_t) * K, cudaMemcpyHostToDevice, stream));
        maybe_compact(done);
      }
      if (anyRestart) {
        B2P_CUDA(cudaMemcpyAsync(d_mask, h_mask, sizeof(int32_t) * K, cudaMemcpyHostToDevice, stream));
        k_restart_multi<<<blocks(std::max<int64_t>(static_cast<int64_t>(N) + M, K)), kBlock, 0, stream>>>(
            N, M, K, d_cinst, d_rinst, d_mask, v[MX], v[MX0], v[MXP], v[MY], v[MY0], v[MYP], v[MAX], v[MAX0],
            v[MAXP], d_it_base, d_restart_at);
        B2P_CUDA(cudaGetLastError());
        ++launches;
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
    for (int b = 0; b < K; ++b) {
      if (done[b]) continue;
      const double* s = h_sums + static_cast<size_t>(b) * kNumSums;
      const double scaleObj = P[b].beta * P[b].gamma;
      const double pobj = s[CS_POBJ] * scaleObj, dobj = (s[CS_ROW_DOBJ] + s[CS_COL_DOBJ]) * scaleObj;
      const double relP = std::sqrt(s[CS_ROW_RES2]) / (1 + rhsNorm[b]);
      const double relD = std::sqrt(s[CS_COL_RES2]) / (1 + cNorm[b]);
      const double gap = std::fabs(pobj - dobj) / (1 + std::fabs(pobj) + std::fabs(dobj));
      extract(b, (expiredStop || expired()) ? B2P_STATUS_TIME_LIMIT : B2P_STATUS_ITERATION_LIMIT,
              smax(relP, smax(relD, gap)), pobj, dobj, it);
      weights[b] = omega[b] * P[b].gamma / P[b].beta;
    }
    stats.kernel_launches = launches;
    stats.bytes_uploaded = bytes_up;
    stats.bytes_downloaded = bytes_down;
  }
};

}  // namespace
}  // namespace b2p

extern "C" int b2p_solve_pdhg_multi_warm(const b2p_lp* lps, int32_t num_lps, const b2p_options* opts,
                                         const double* const* x_start, const double* const* row_dual_start,
                                         const double* primal_weight_start, double* const* x,
                                         double* const* row_dual, double* primal_weight, b2p_result* results,
                                         b2p_stats* stats) {
  using namespace b2p;
  return guarded([&] {
    const auto t0 = Clock::now();
    MultiEngine e;
    e.create(lps, num_lps, opts);
    e.set_start(x_start, row_dual_start, primal_weight_start);
    e.solve(t0);
    for (int b = 0; b < e.K; ++b) {
      if (x && x[b] && !e.xs[b].empty()) std::memcpy(x[b], e.xs[b].data(), sizeof(double) * e.xs[b].size());
      if (row_dual && row_dual[b] && !e.ys[b].empty())
        std::memcpy(row_dual[b], e.ys[b].data(), sizeof(double) * e.ys[b].size());
      if (primal_weight) primal_weight[b] = e.weights[b];
      if (results) results[b] = e.results[b];
    }
    if (stats) *stats = e.stats;
  });
}

extern "C" int b2p_solve_pdhg_multi(const b2p_lp* lps, int32_t num_lps, const b2p_options* opts,
                                    const double* const* x_start, const double* const* row_dual_start,
                                    double* const* x, double* const* row_dual, b2p_result* results, b2p_stats* stats) {
  return b2p_solve_pdhg_multi_warm(lps, num_lps, opts, x_start, row_dual_start, nullptr, x, row_dual, nullptr,
                                   results, stats);
}
