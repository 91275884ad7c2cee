// Certification of OPTIMAL claims on the device, batched over cases of one A.
//
// The certifier of the reference runs on host threads, one case at a time
// (certify, src/cert/certifier.cpp:208-380, with its constraint-implied
// column bounds from Propagator::propagate, src/mip/propagate.cpp:23-138).
// Its two expensive parts are done here on the GPU, by methods of this
// project, for every case of a family at once:
//
// 1. Constraint-implied column bounds (b2p_implied_bounds).  Activity-based
//    bound tightening (Brearley, Mitra and Williams, Math. Programming 8
//    (1975) 54-83; Achterberg, Constraint Integer Programming, 2007,
//    sec. 7.1), organised as Jacobi sweeps: in each round every (row, case)
//    forms its smallest and largest activity over the current column bounds,
//    counting the infinite contributions apart (k_ib_activity); then every
//    (column, case) intersects its bounds with what each of its rows implies
//    once the column's own contribution is taken out (k_ib_tighten).  Each
//    operation is rounded in the safe direction by the hardware's directed-
//    rounding instructions (__dadd_rd, __dmul_ru, __ddiv_rd, ...), so the
//    bounds contain every feasible point of the exact LP and need no safety
//    margin.  Rounds repeat until no bound of a case moves by more than
//    kIbStep relative (or kIbMaxRounds); a case whose bounds cross is
//    infeasible and keeps the bounds it had.
// 2. The primal half of the verdict (b2p_certify_lp).  Per (row, case) the
//    row activity as a compensated dot product (Ogita, Rump and Oishi,
//    SIAM J. Sci. Comput. 26 (2005), Dot2: the exact product error from an
//    FMA and the exact addition error from TwoSum, carried in a second
//    word), its relative excess over the row bounds, and per case the largest
//    one with its row; per (column, case) the relative excess of x over the
//    column bounds; the objective c'x as a compensated sum.  Block partials
//    are combined in a fixed order, so results do not depend on scheduling.
// The dual half is the outward-rounded Neumaier-Shcherbina bound
// (pdhg_certify.cu), retried over the implied bounds where it is -inf; the
// acceptance rules are the certifier's: primal excess <= primal_feasibility,
// and either (pobj - LB) / max(1, |pobj|) <= relative_gap with LB rounded
// down, or, without a finite bound, the largest wrong-signed reduced cost
// <= dual_feasibility.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "pdhg_cert.h"
#include "pdhg_host_common.h"
#include "pdhg_kernels.cuh"
#include "pdhg_prepare.h"
#include "pdhg_sched.h"

namespace b2p {

constexpr int kIbMaxRounds = 1024;  // propagation rounds at most
constexpr int kIbPollEvery = 16;    // rounds between convergence polls by the host
constexpr double kIbStep = 1e-9;    // a move smaller than this (relative) is not progress

namespace cert {

__device__ __forceinline__ bool fin(double v) { return fabs(v) < 1e20; }

// Exact error of s = fl(a + b) (TwoSum, Knuth).
__device__ __forceinline__ double add_error(double a, double b, double s) {
  const double bv = __dsub_rn(s, a);
  const double av = __dsub_rn(s, bv);
  return __dadd_rn(__dsub_rn(a, av), __dsub_rn(b, bv));
}

// A sum carried in two words: hi + lo, lo collecting the rounding errors.
struct TwoWord {
  double hi, lo;
  __device__ __forceinline__ void add(double v) {
    const double s = __dadd_rn(hi, v);
    if (!isfinite(s)) {
      hi = s;
      return;
    }
    lo = __dadd_rn(lo, add_error(hi, v, s));
    hi = s;
  }
  // the product a*x added with its exact error (FMA remainder)
  __device__ __forceinline__ void add_product(double a, double x) {
    const double p = __dmul_rn(a, x);
    if (!isfinite(p)) {
      hi = __dadd_rn(hi, p);
      return;
    }
    const double e = __fma_rn(a, x, -p);
    add(p);
    lo = __dadd_rn(lo, e);
  }
  __device__ __forceinline__ void merge(const TwoWord& o) {
    add(o.hi);
    lo = __dadd_rn(lo, o.lo);
  }
  __device__ __forceinline__ double value() const { return isfinite(hi) ? __dadd_rn(hi, lo) : hi; }
};

// How far v lies outside [lower, upper], relative to the bound it crosses;
// +inf for a non-finite v.  The measure of certify's primal checks.
__device__ __forceinline__ double rel_excess(double v, double lower, double upper) {
  if (!isfinite(v)) return INFINITY;
  double q = 0.0;
  if (fin(lower) && v < lower) q = (lower - v) / (1.0 + fabs(lower));
  if (fin(upper) && v > upper) {
    const double e = (v - upper) / (1.0 + fabs(upper));
    if (e > q) q = e;
  }
  return q;
}

// The larger (value, index) pair; among equal values the smaller index.
__device__ __forceinline__ void keep_worse(double& q, int32_t& at, double q2, int32_t at2) {
  if (q2 > q || (q2 == q && at2 < at)) {
    q = q2;
    at = at2;
  }
}

// Block-wide: the worst (value, index) and the two-word sum; thread 0 holds them.
__device__ __forceinline__ void block_combine(double& q, int32_t& at, TwoWord& s) {
  __shared__ double sq[kBlock / 32], sh[kBlock / 32], sl[kBlock / 32];
  __shared__ int32_t si[kBlock / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double q2 = __shfl_down_sync(0xffffffffu, q, off);
    const int32_t a2 = __shfl_down_sync(0xffffffffu, at, off);
    TwoWord o{__shfl_down_sync(0xffffffffu, s.hi, off), __shfl_down_sync(0xffffffffu, s.lo, off)};
    keep_worse(q, at, q2, a2);
    s.merge(o);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sq[w] = q;
    si[w] = at;
    sh[w] = s.hi;
    sl[w] = s.lo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int v = 1; v < kBlock / 32; ++v) {
      keep_worse(q, at, sq[v], si[v]);
      s.merge(TwoWord{sh[v], sl[v]});
    }
  }
}

}  // namespace cert

// ---- implied bounds --------------------------------------------------------

// Per (row i, case b): smallest / largest activity over the finite
// contributions, rounded down / up, and how many contributions are infinite.
__global__ void __launch_bounds__(kBlock) k_ib_activity(int32_t m, int32_t n, CsrView A, const double* __restrict__ lo,
                                                        const double* __restrict__ up, const int32_t* __restrict__ live,
                                                        const int32_t* __restrict__ infeasible,
                                                        double* __restrict__ act_lo, double* __restrict__ act_hi,
                                                        int32_t* __restrict__ inf_lo, int32_t* __restrict__ inf_hi) {
  const int b = blockIdx.y;
  if (!live[b] || infeasible[b]) return;
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double* lb = lo + static_cast<int64_t>(b) * n;
  const double* ub = up + static_cast<int64_t>(b) * n;
  double s_lo = 0.0, s_hi = 0.0;
  int32_t c_lo = 0, c_hi = 0;
  for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) {
    const double a = A.val[p];
    if (a == 0.0) continue;
    const int32_t j = A.idx[p];
    const double at_min = a > 0.0 ? lb[j] : ub[j];  // the bound where a*x_j is smallest
    const double at_max = a > 0.0 ? ub[j] : lb[j];
    if (cert::fin(at_min))
      s_lo = __dadd_rd(s_lo, __dmul_rd(a, at_min));
    else
      ++c_lo;
    if (cert::fin(at_max))
      s_hi = __dadd_ru(s_hi, __dmul_ru(a, at_max));
    else
      ++c_hi;
  }
  const int64_t t = static_cast<int64_t>(b) * m + i;
  act_lo[t] = s_lo;
  act_hi[t] = s_hi;
  inf_lo[t] = c_lo;
  inf_hi[t] = c_hi;
}

// Per (column j, case b): the bounds each row of the column implies, taken
// together with the column's own; AT is the CSR of A^T (the column's rows).
__global__ void __launch_bounds__(kBlock) k_ib_tighten(int32_t n, int32_t m, CsrView AT, const double* __restrict__ rl,
                                                       const double* __restrict__ ru,
                                                       const double* __restrict__ act_lo,
                                                       const double* __restrict__ act_hi,
                                                       const int32_t* __restrict__ inf_lo,
                                                       const int32_t* __restrict__ inf_hi, double* __restrict__ lo,
                                                       double* __restrict__ up, const int32_t* __restrict__ live,
                                                       int32_t* __restrict__ progress, int32_t* __restrict__ infeasible) {
  const int b = blockIdx.y;
  if (!live[b] || infeasible[b]) return;
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t t = static_cast<int64_t>(b) * n + j;
  const double l = lo[t], u = up[t];
  double nl = l, nu = u;
  for (int p = AT.ptr[j]; p < AT.ptr[j + 1]; ++p) {
    const double a = AT.val[p];
    if (a == 0.0) continue;
    const int64_t r = static_cast<int64_t>(b) * m + AT.idx[p];
    const double L = rl[r], U = ru[r];
    const double at_min = a > 0.0 ? l : u, at_max = a > 0.0 ? u : l;
    // the other entries' smallest activity (a lower bound of it) ...
    bool rest_lo_ok;
    double rest_lo;
    if (cert::fin(at_min)) {
      rest_lo_ok = inf_lo[r] == 0;
      rest_lo = __dsub_rd(act_lo[r], __dmul_ru(a, at_min));
    } else {
      rest_lo_ok = inf_lo[r] == 1;
      rest_lo = act_lo[r];
    }
    // ... and their largest (an upper bound of it)
    bool rest_hi_ok;
    double rest_hi;
    if (cert::fin(at_max)) {
      rest_hi_ok = inf_hi[r] == 0;
      rest_hi = __dsub_ru(act_hi[r], __dmul_rd(a, at_max));
    } else {
      rest_hi_ok = inf_hi[r] == 1;
      rest_hi = act_hi[r];
    }
    // a x_j <= U - rest  <=  U - rest_lo
    if (rest_lo_ok && cert::fin(U)) {
      const double room = __dsub_ru(U, rest_lo);
      if (a > 0.0) {
        const double v = __ddiv_ru(room, a);
        if (!cert::fin(nu) || v < nu) nu = v;
      } else {
        const double v = __ddiv_rd(room, a);
        if (!cert::fin(nl) || v > nl) nl = v;
      }
    }
    // a x_j >= L - rest  >=  L - rest_hi
    if (rest_hi_ok && cert::fin(L)) {
      const double need = __dsub_rd(L, rest_hi);
      if (a > 0.0) {
        const double v = __ddiv_rd(need, a);
        if (!cert::fin(nl) || v > nl) nl = v;
      } else {
        const double v = __ddiv_ru(need, a);
        if (!cert::fin(nu) || v < nu) nu = v;
      }
    }
  }
  if (cert::fin(nl) && cert::fin(nu) && nl > nu) {
    infeasible[b] = 1;  // no point of the exact LP satisfies the rows: the case is infeasible
    return;
  }
  const bool moved_lo = cert::fin(nl) && (!cert::fin(l) || nl - l > kIbStep * (1.0 + fabs(nl)));
  const bool moved_up = cert::fin(nu) && (!cert::fin(u) || u - nu > kIbStep * (1.0 + fabs(nu)));
  if (cert::fin(nl) && (!cert::fin(l) || nl > l)) lo[t] = nl;
  if (cert::fin(nu) && (!cert::fin(u) || nu < u)) up[t] = nu;
  if (moved_lo || moved_up) progress[b] = 1;
}

// Device state of the propagation over k cases (case-major bounds, updated in place).
struct ImpliedBoundsRun {
  int32_t m, n, k;
  CsrView A, AT;
  const double *rl, *ru;
  double *lo, *up;                      // in: the cases' bounds; out: implied
  double *act_lo, *act_hi;              // k x m
  int32_t *inf_lo, *inf_hi;             // k x m
  int32_t* progress;                    // (kIbMaxRounds + 1) x k; row 0 all ones
  int32_t* infeasible;                  // k
};

// Rounds until no case moves; returns the rounds run.
inline int run_implied_bounds(cudaStream_t s, const ImpliedBoundsRun& r) {
  const dim3 grow((r.m + kBlock - 1) / kBlock, r.k), gcol((r.n + kBlock - 1) / kBlock, r.k);
  std::vector<int32_t> ones(r.k, 1), poll(r.k);
  B2P_CUDA(cudaMemcpyAsync(r.progress, ones.data(), sizeof(int32_t) * r.k, cudaMemcpyHostToDevice, s));
  B2P_CUDA(cudaMemsetAsync(r.progress + r.k, 0, sizeof(int32_t) * r.k * kIbMaxRounds, s));
  B2P_CUDA(cudaMemsetAsync(r.infeasible, 0, sizeof(int32_t) * r.k, s));
  if (r.m == 0 || r.n == 0) {
    B2P_CUDA(cudaStreamSynchronize(s));
    return 0;
  }
  int round = 0;
  while (round < kIbMaxRounds) {
    const int32_t* live = r.progress + static_cast<int64_t>(round) * r.k;
    int32_t* next = r.progress + static_cast<int64_t>(round + 1) * r.k;
    k_ib_activity<<<grow, kBlock, 0, s>>>(r.m, r.n, r.A, r.lo, r.up, live, r.infeasible, r.act_lo, r.act_hi, r.inf_lo,
                                          r.inf_hi);
    k_ib_tighten<<<gcol, kBlock, 0, s>>>(r.n, r.m, r.AT, r.rl, r.ru, r.act_lo, r.act_hi, r.inf_lo, r.inf_hi, r.lo, r.up,
                                         live, next, r.infeasible);
    ++round;
    if (round % kIbPollEvery == 0 || round == kIbMaxRounds) {
      B2P_CUDA(cudaGetLastError());
      B2P_CUDA(cudaMemcpyAsync(poll.data(), next, sizeof(int32_t) * r.k, cudaMemcpyDeviceToHost, s));
      B2P_CUDA(cudaStreamSynchronize(s));
      if (std::none_of(poll.begin(), poll.end(), [](int32_t v) { return v != 0; })) break;
    }
  }
  B2P_CUDA(cudaGetLastError());
  return round;
}

// ---- primal checks ---------------------------------------------------------

// grid (row blocks, k): per block the worst row excess and its row.
__global__ void __launch_bounds__(kBlock) k_cert_rows(int32_t m, int32_t n, CsrView A, const double* __restrict__ x,
                                                      const double* __restrict__ rl, const double* __restrict__ ru,
                                                      double* __restrict__ part_q, int32_t* __restrict__ part_at) {
  const int b = blockIdx.y;
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  double q = -1.0;
  int32_t at = INT_MAX;
  cert::TwoWord unused{0.0, 0.0};
  if (i < m) {
    const double* xb = x + static_cast<int64_t>(b) * n;
    cert::TwoWord act{0.0, 0.0};
    for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) act.add_product(A.val[p], xb[A.idx[p]]);
    const int64_t t = static_cast<int64_t>(b) * m + i;
    q = cert::rel_excess(act.value(), rl[t], ru[t]);
    at = static_cast<int32_t>(i);
  }
  cert::block_combine(q, at, unused);
  if (threadIdx.x == 0) {
    part_q[static_cast<int64_t>(b) * gridDim.x + blockIdx.x] = q;
    part_at[static_cast<int64_t>(b) * gridDim.x + blockIdx.x] = at;
  }
}

// grid (column blocks, k): per block the worst column excess and the
// two-word partial of c'x.
__global__ void __launch_bounds__(kBlock) k_cert_cols(int32_t n, const double* __restrict__ x,
                                                      const double* __restrict__ c, const double* __restrict__ lo,
                                                      const double* __restrict__ up, double* __restrict__ part_q,
                                                      double* __restrict__ part_hi, double* __restrict__ part_lo) {
  const int b = blockIdx.y;
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  double q = -1.0;
  int32_t at = INT_MAX;
  cert::TwoWord obj{0.0, 0.0};
  if (j < n) {
    const int64_t t = static_cast<int64_t>(b) * n + j;
    q = cert::rel_excess(x[t], lo[t], up[t]);
    at = static_cast<int32_t>(j);
    obj.add_product(c[t], x[t]);
  }
  cert::block_combine(q, at, obj);
  if (threadIdx.x == 0) {
    const int64_t o = static_cast<int64_t>(b) * gridDim.x + blockIdx.x;
    part_q[o] = q;
    part_hi[o] = obj.hi;
    part_lo[o] = obj.lo;
  }
}

// Per-case results of the primal checks.
struct PrimalOut {
  double row_q, col_q, pobj;
  int32_t worst_row, pad;
};

// grid = k: the partials of every block, in block order.
__global__ void __launch_bounds__(kBlock) k_cert_primal_finalize(int32_t g_rows, int32_t g_cols, double offset,
                                                                 const double* __restrict__ rq,
                                                                 const int32_t* __restrict__ rat,
                                                                 const double* __restrict__ cq,
                                                                 const double* __restrict__ chi,
                                                                 const double* __restrict__ clo,
                                                                 PrimalOut* __restrict__ out) {
  const int b = blockIdx.x;
  double q = -1.0;
  int32_t at = INT_MAX;
  cert::TwoWord none{0.0, 0.0};
  for (int g = threadIdx.x; g < g_rows; g += blockDim.x)
    cert::keep_worse(q, at, rq[static_cast<int64_t>(b) * g_rows + g], rat[static_cast<int64_t>(b) * g_rows + g]);
  cert::block_combine(q, at, none);
  __syncthreads();
  double qc = -1.0;
  int32_t atc = INT_MAX;
  cert::TwoWord obj{0.0, 0.0};
  for (int g = threadIdx.x; g < g_cols; g += blockDim.x) {
    const int64_t o = static_cast<int64_t>(b) * g_cols + g;
    cert::keep_worse(qc, atc, cq[o], 0);
    obj.merge(cert::TwoWord{chi[o], clo[o]});
  }
  cert::block_combine(qc, atc, obj);
  if (threadIdx.x == 0) {
    PrimalOut r;
    r.row_q = q > 0.0 ? q : 0.0;
    r.worst_row = q > 0.0 ? at : -1;
    r.col_q = qc > 0.0 ? qc : 0.0;
    cert::TwoWord f{offset, 0.0};
    f.merge(obj);
    r.pobj = f.value();
    r.pad = 0;
    out[b] = r;
  }
}

// grid = k / 128: the bound with the objective offset, rounded down, and the
// relative gap.
__global__ void k_cert_gap(int32_t k, double offset, const double* __restrict__ bound,
                           const PrimalOut* __restrict__ primal, double* __restrict__ lb,
                           double* __restrict__ gap) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k) return;
  const double v = bound[b];
  if (isinf(v) || isnan(v)) {
    lb[b] = -INFINITY;
    gap[b] = INFINITY;
    return;
  }
  const double l = __dadd_rd(v, offset);
  const double p = primal[b].pobj;
  lb[b] = l;
  gap[b] = (p - l) / fmax(1.0, fabs(p));
}

// Case-major expansion of the per-case vectors (a case's own or the base's).
struct CaseVectors {
  std::vector<double> c, lo, up, rl, ru;
};

inline CaseVectors expand_cases(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases) {
  const int k = num_cases > 0 ? num_cases : 1;
  const size_t n = static_cast<size_t>(lp->num_cols), m = static_cast<size_t>(lp->num_rows);
  CaseVectors v;
  v.c.resize(k * n);
  v.lo.resize(k * n);
  v.up.resize(k * n);
  v.rl.resize(k * m);
  v.ru.resize(k * m);
  for (int b = 0; b < k; ++b) {
    const b2p_case* cs = num_cases > 0 ? &cases[b] : nullptr;
    const auto take = [&](const double* own, const double* base, size_t len, std::vector<double>& dst) {
      if (len) std::memcpy(dst.data() + b * len, (cs && own) ? own : base, sizeof(double) * len);
    };
    take(cs ? cs->cost : nullptr, lp->col_cost, n, v.c);
    take(cs ? cs->col_lower : nullptr, lp->col_lower, n, v.lo);
    take(cs ? cs->col_upper : nullptr, lp->col_upper, n, v.up);
    take(cs ? cs->row_lower : nullptr, lp->row_lower, m, v.rl);
    take(cs ? cs->row_upper : nullptr, lp->row_upper, m, v.ru);
  }
  return v;
}

// Device memory and the stream of one call, from the device's stream-ordered
// pool, released on every exit path.
struct CertBuffers {
  int dev;
  cudaStream_t s = nullptr;
  std::vector<void*> held;
  explicit CertBuffers(int d) : dev(d) { B2P_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~CertBuffers() {
    for (void* p : held) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  template <class T>
  T* get(size_t count, const T* from = nullptr) {
    void* p = nullptr;
    B2P_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(count, 1) * sizeof(T), device_pool(dev), s));
    held.push_back(p);
    if (from && count) B2P_CUDA(cudaMemcpyAsync(p, from, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return static_cast<T*>(p);
  }
};

// The operators on the device: A row-major (the CSR a stable counting sort of
// the CSC gives) and the CSC itself as the CSR of A^T.
struct DeviceOperators {
  CsrView A, AT;
};

inline DeviceOperators upload_operators(CertBuffers& B, const b2p_lp* lp) {
  const Prepared P = prepare_structure(lp->num_rows, lp->num_cols, lp->start, lp->index, lp->value, 0.0, true);
  const size_t nnz = static_cast<size_t>(lp->start[lp->num_cols]);
  DeviceOperators d;
  d.A = CsrView{B.get<int32_t>(P.A.ptr.size(), P.A.ptr.data()), B.get<int32_t>(nnz, P.A.idx.data()),
                B.get<double>(nnz, P.A.val.data()), lp->num_rows};
  d.AT = CsrView{B.get<int32_t>(static_cast<size_t>(lp->num_cols) + 1, lp->start), B.get<int32_t>(nnz, lp->index),
                 B.get<double>(nnz, lp->value), lp->num_cols};
  return d;
}

inline ImpliedBoundsRun make_ib_run(CertBuffers& B, const b2p_lp* lp, int k, const DeviceOperators& ops,
                                    const double* rl, const double* ru, double* lo, double* up) {
  const size_t m = static_cast<size_t>(lp->num_rows);
  ImpliedBoundsRun r;
  r.m = lp->num_rows;
  r.n = lp->num_cols;
  r.k = k;
  r.A = ops.A;
  r.AT = ops.AT;
  r.rl = rl;
  r.ru = ru;
  r.lo = lo;
  r.up = up;
  r.act_lo = B.get<double>(k * m);
  r.act_hi = B.get<double>(k * m);
  r.inf_lo = B.get<int32_t>(k * m);
  r.inf_hi = B.get<int32_t>(k * m);
  r.progress = B.get<int32_t>(static_cast<size_t>(kIbMaxRounds + 1) * k);
  r.infeasible = B.get<int32_t>(k);
  return r;
}

}  // namespace b2p

using namespace b2p;

extern "C" int b2p_implied_bounds(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, double* col_lower_out,
                                  double* col_upper_out) {
  return guarded([&] {
    check_lp(lp);
    if (!col_lower_out || !col_upper_out) throw Error(B2P_ERR_INVALID, "NULL output");
    if (num_cases > 0 && !cases) throw Error(B2P_ERR_INVALID, "cases is NULL");
    const int k = num_cases > 0 ? num_cases : 1;
    const CaseVectors v = expand_cases(lp, cases, num_cases);
    const int dev = pick_device(-1);
    B2P_CUDA(cudaSetDevice(dev));
    CertBuffers B(dev);
    const DeviceOperators ops = upload_operators(B, lp);
    double* lo = B.get<double>(v.lo.size(), v.lo.data());
    double* up = B.get<double>(v.up.size(), v.up.data());
    const ImpliedBoundsRun r = make_ib_run(B, lp, k, ops, B.get<double>(v.rl.size(), v.rl.data()),
                                           B.get<double>(v.ru.size(), v.ru.data()), lo, up);
    run_implied_bounds(B.s, r);
    B2P_CUDA(cudaMemcpyAsync(col_lower_out, lo, sizeof(double) * v.lo.size(), cudaMemcpyDeviceToHost, B.s));
    B2P_CUDA(cudaMemcpyAsync(col_upper_out, up, sizeof(double) * v.up.size(), cudaMemcpyDeviceToHost, B.s));
    B2P_CUDA(cudaStreamSynchronize(B.s));
  });
}

extern "C" int b2p_certify_lp(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const double* x,
                              const double* row_dual, const b2p_cert_tolerances* tol, b2p_certificate* out) {
  return guarded([&] {
    check_lp(lp);
    if (!x || !row_dual || !out) throw Error(B2P_ERR_INVALID, "NULL argument");
    if (num_cases > 0 && !cases) throw Error(B2P_ERR_INVALID, "cases is NULL");
    const b2p_cert_tolerances t = tol ? *tol : b2p_cert_tolerances{1e-6, 1e-6, 1e-6};
    const int k = num_cases > 0 ? num_cases : 1;
    const int32_t m = lp->num_rows, n = lp->num_cols;
    const CaseVectors v = expand_cases(lp, cases, num_cases);
    const int dev = pick_device(-1);
    B2P_CUDA(cudaSetDevice(dev));
    CertBuffers B(dev);
    cudaStream_t s = B.s;
    const DeviceOperators ops = upload_operators(B, lp);
    const double* dx = B.get<double>(static_cast<size_t>(k) * n, x);
    const double* dy = B.get<double>(static_cast<size_t>(k) * m, row_dual);
    const double* dc = B.get<double>(v.c.size(), v.c.data());
    const double* dlo = B.get<double>(v.lo.size(), v.lo.data());
    const double* dup = B.get<double>(v.up.size(), v.up.data());
    const double* drl = B.get<double>(v.rl.size(), v.rl.data());
    const double* dru = B.get<double>(v.ru.size(), v.ru.data());

    // primal checks and the objective
    const int gr = std::max(1, (m + kBlock - 1) / kBlock), gc = std::max(1, (n + kBlock - 1) / kBlock);
    double* rq = B.get<double>(static_cast<size_t>(k) * gr);
    int32_t* rat = B.get<int32_t>(static_cast<size_t>(k) * gr);
    double* cq = B.get<double>(static_cast<size_t>(k) * gc);
    double* chi = B.get<double>(static_cast<size_t>(k) * gc);
    double* clo = B.get<double>(static_cast<size_t>(k) * gc);
    PrimalOut* primal = B.get<PrimalOut>(k);
    k_cert_rows<<<dim3(gr, k), kBlock, 0, s>>>(m, n, ops.A, dx, drl, dru, rq, rat);
    k_cert_cols<<<dim3(gc, k), kBlock, 0, s>>>(n, dx, dc, dlo, dup, cq, chi, clo);
    k_cert_primal_finalize<<<k, kBlock, 0, s>>>(gr, gc, lp->obj_offset, rq, rat, cq, chi, clo, primal);
    B2P_CUDA(cudaGetLastError());

    // the dual bound from the given duals over the given column bounds
    const size_t len = static_cast<size_t>(m) + n;
    double* yp = B.get<double>(static_cast<size_t>(k) * m);
    double* terms = B.get<double>(k * len);
    double* stats1 = B.get<double>(static_cast<size_t>(k) * 4);
    int32_t* inf1 = B.get<int32_t>(k);
    double* bound1 = B.get<double>(k);
    enqueue_safe_bound(s, m, n, k, ops.AT, dy, dc, dlo, dup, drl, dru, yp, terms, stats1, inf1, bound1);
    std::vector<double> hb1(k), hs1(static_cast<size_t>(k) * 4);
    std::vector<int32_t> hi1(k);
    B2P_CUDA(cudaMemcpyAsync(hb1.data(), bound1, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaMemcpyAsync(hs1.data(), stats1, sizeof(double) * 4 * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaMemcpyAsync(hi1.data(), inf1, sizeof(int32_t) * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaStreamSynchronize(s));

    // where it is -inf: again over the constraint-implied column bounds
    std::vector<char> use2(k, 0);
    double* chosen = bound1;
    std::vector<double> hb2, hs2;
    std::vector<int32_t> hi2;
    if (std::any_of(hb1.begin(), hb1.end(), [](double b) { return std::isinf(b); })) {
      double* ilo = B.get<double>(v.lo.size(), v.lo.data());
      double* iup = B.get<double>(v.up.size(), v.up.data());
      run_implied_bounds(s, make_ib_run(B, lp, k, ops, drl, dru, ilo, iup));
      double* stats2 = B.get<double>(static_cast<size_t>(k) * 4);
      int32_t* inf2 = B.get<int32_t>(k);
      double* bound2 = B.get<double>(k);
      enqueue_safe_bound(s, m, n, k, ops.AT, dy, dc, ilo, iup, drl, dru, yp, terms, stats2, inf2, bound2);
      hb2.resize(k);
      hs2.resize(static_cast<size_t>(k) * 4);
      hi2.resize(k);
      B2P_CUDA(cudaMemcpyAsync(hb2.data(), bound2, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
      B2P_CUDA(cudaMemcpyAsync(hs2.data(), stats2, sizeof(double) * 4 * k, cudaMemcpyDeviceToHost, s));
      B2P_CUDA(cudaMemcpyAsync(hi2.data(), inf2, sizeof(int32_t) * k, cudaMemcpyDeviceToHost, s));
      B2P_CUDA(cudaStreamSynchronize(s));
      std::vector<double> pick(hb1);
      for (int b = 0; b < k; ++b)
        if (std::isinf(hb1[b]) && !std::isinf(hb2[b])) {
          use2[b] = 1;
          pick[b] = hb2[b];
        }
      chosen = B.get<double>(k, pick.data());
    }
    double* lb = B.get<double>(k);
    double* gap = B.get<double>(k);
    k_cert_gap<<<(k + 127) / 128, 128, 0, s>>>(k, lp->obj_offset, chosen, primal, lb, gap);
    B2P_CUDA(cudaGetLastError());
    std::vector<PrimalOut> hp(k);
    std::vector<double> hlb(k), hgap(k);
    B2P_CUDA(cudaMemcpyAsync(hp.data(), primal, sizeof(PrimalOut) * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaMemcpyAsync(hlb.data(), lb, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaMemcpyAsync(hgap.data(), gap, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaStreamSynchronize(s));

    for (int b = 0; b < k; ++b) {
      const double* st = use2[b] ? &hs2[static_cast<size_t>(b) * 4] : &hs1[static_cast<size_t>(b) * 4];
      b2p_certificate& o = out[b];
      std::memset(&o, 0, sizeof(o));
      o.primal_objective = hp[b].pobj;
      o.max_row_violation = hp[b].row_q;
      o.max_col_violation = hp[b].col_q;
      o.max_primal_violation = std::max(hp[b].row_q, hp[b].col_q);
      o.worst_row = hp[b].worst_row;
      o.used_implied_bounds = use2[b];
      o.infinite_terms = use2[b] ? hi2[b] : hi1[b];
      o.max_dual_violation = st[1];
      o.cost_perturbation = st[2];
      o.safe_dual_bound = hlb[b];
      o.certified_gap = hgap[b];
      const bool primal_ok = hp[b].col_q <= t.primal_feasibility && hp[b].row_q <= t.primal_feasibility;
      const bool has_bound = !std::isinf(hlb[b]);
      const bool dual_ok = has_bound ? hgap[b] <= t.relative_gap : st[1] <= t.dual_feasibility;
      o.accepted = primal_ok && dual_ok;
    }
  });
}
