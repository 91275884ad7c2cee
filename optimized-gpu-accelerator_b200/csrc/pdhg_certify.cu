// Rigorous (outward-rounded) Neumaier-Shcherbina lower bound of an LP from
// any row dual y, on the device, for many cases at once.
//
// Restates safeDualBound / safeBoundInterval (src/cert/certifier.cpp:58-118)
// with the interval helpers of src/cert/interval.h:14-91:
//   y' = projection of y onto its sign cone (free rows 0, upper-only <= 0,
//        lower-only >= 0)                                  (projectRowDuals)
//   z_j = [c_j, c_j] - sum_k [a_kj y'_k] as outward-rounded intervals, in the
//        column's entry order                               (reducedCostIntervals)
//   lb  = sum_i minProduct([y'_i], L_i, U_i) + sum_j minProduct(z_j, l_j, u_j)
//        added with downward rounding, rows first, then columns; a
//        wrong-signed z on an infinite bound is clipped when the implied cost
//        change is <= 1e-9 relative, otherwise the bound is -inf.
// The directed operations are written like the reference's: a round-to-
// nearest result, its exact error (TwoSum / FMA remainder), and a one-ulp
// step in the safe direction only when the result was inexact -- so every
// term, and the in-order sum of each case, is bit-identical to the
// reference's CPU result.  Cases run in parallel: one thread per column and
// case for the intervals, one thread per case for the ordered outward sum.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pdhg_cert.h"
#include "pdhg_host_common.h"
#include "pdhg_kernels.cuh"

namespace b2p {

namespace ns {

__device__ __forceinline__ bool fin(double v) { return fabs(v) < 1e20; }
__device__ __forceinline__ double clean(double v) { return fin(v) ? v : (v > 0 ? INFINITY : -INFINITY); }
// The neighbouring double toward -inf / +inf of a finite v (IEEE-754 binary64:
// the bit pattern of a non-negative double increases with its value).
__device__ __forceinline__ double step_down(double v) {
  if (v == 0.0) return -__longlong_as_double(1LL);  // -(smallest subnormal)
  const long long b = __double_as_longlong(v);
  return __longlong_as_double(v > 0 ? b - 1 : b + 1);
}
__device__ __forceinline__ double step_up(double v) {
  if (v == 0.0) return __longlong_as_double(1LL);
  const long long b = __double_as_longlong(v);
  return __longlong_as_double(v > 0 ? b + 1 : b - 1);
}
__device__ __forceinline__ double round_down(double v) { return (isinf(v) || isnan(v)) ? v : step_down(v); }
__device__ __forceinline__ double round_up(double v) { return (isinf(v) || isnan(v)) ? v : step_up(v); }

// exact error of s = fl(a + b)
__device__ __forceinline__ double two_sum_err(double a, double b, double s) {
  const double bb = __dsub_rn(s, a);
  return __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ double add_down(double a, double b) {
  const double s = __dadd_rn(a, b);
  if (isinf(s) || isnan(s)) return s;
  return two_sum_err(a, b, s) < 0 ? round_down(s) : s;
}
__device__ __forceinline__ double add_up(double a, double b) {
  const double s = __dadd_rn(a, b);
  if (isinf(s) || isnan(s)) return s;
  return two_sum_err(a, b, s) > 0 ? round_up(s) : s;
}
__device__ __forceinline__ double mul_down(double a, double b) {
  if (a == 0 || b == 0) return 0.0;
  const double p = __dmul_rn(a, b);
  if (isinf(p)) return p;
  return __fma_rn(a, b, -p) < 0 ? round_down(p) : p;
}
__device__ __forceinline__ double mul_up(double a, double b) {
  if (a == 0 || b == 0) return 0.0;
  const double p = __dmul_rn(a, b);
  if (isinf(p)) return p;
  return __fma_rn(a, b, -p) > 0 ? round_up(p) : p;
}

// rigorous lower bound of min{ z x : z in [zlo, zhi], x in [l, u] }
__device__ __forceinline__ double min_product(double zlo, double zhi, double l, double u) {
  if (zlo == 0 && zhi == 0) return 0.0;
  if (isinf(l) && zhi > 0) return -INFINITY;
  if (isinf(u) && zlo < 0) return -INFINITY;
  double best = INFINITY;
  const double zs[2] = {zlo, zhi}, xs[2] = {l, u};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const double zz = zs[a], xx = xs[b];
      double p;
      if (zz == 0 || xx == 0)
        p = 0.0;
      else if (isinf(xx))
        p = __dmul_rn(zz, xx);
      else
        p = mul_down(zz, xx);
      if (p < best) best = p;
    }
  return best;
}

// Non-negative double max as an integer atomic (order-independent, so deterministic).
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

}  // namespace ns

constexpr double kMaxAllowedPerturbation = 1e-9;  // SafeBoundResult::maxAllowedPerturbation

// Per case b: stats[b*4 + {0: row projection, 1: max dual infeasibility, 2: cost perturbation}], count[b].
// Row terms: terms[b*(m+n) + i]; projected duals yp[b*m + i].
__global__ void __launch_bounds__(kBlock) k_ns_rows(int32_t m, int32_t n, const double* __restrict__ y,
                                                    const double* __restrict__ rl, const double* __restrict__ ru,
                                                    double* __restrict__ yp, double* __restrict__ terms,
                                                    double* __restrict__ stats) {
  const int b = blockIdx.y;
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t t = static_cast<int64_t>(b) * m + i;
  const double L = rl[t], U = ru[t], y0 = y[t];
  const bool lo = ns::fin(L), up = ns::fin(U);
  double v = y0;
  if (!lo && !up)
    v = 0;
  else if (!lo)
    v = (0.0 < v) ? 0.0 : v;  // std::min(v, 0.0)
  else if (!up)
    v = (v < 0.0) ? 0.0 : v;  // std::max(v, 0.0)
  yp[t] = v;
  ns::atomic_max_nonneg(stats + b * 4 + 0, fabs(v - y0));
  terms[static_cast<int64_t>(b) * (m + n) + i] = ns::min_product(v, v, ns::clean(L), ns::clean(U));
}

// Column terms (NaN marks a column that makes the bound -inf).
__global__ void __launch_bounds__(kBlock) k_ns_cols(int32_t m, int32_t n, CsrView AT, const double* __restrict__ yp,
                                                    const double* __restrict__ c, const double* __restrict__ lo,
                                                    const double* __restrict__ up, double* __restrict__ terms,
                                                    double* __restrict__ stats, int32_t* __restrict__ inf_terms) {
  const int b = blockIdx.y;
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t t = static_cast<int64_t>(b) * n + j;
  const double* yb = yp + static_cast<int64_t>(b) * m;
  const double cj = c[t];
  double zlo = cj, zhi = cj;
  for (int p = AT.ptr[j]; p < AT.ptr[j + 1]; ++p) {
    const double a = AT.val[p], yv = yb[AT.idx[p]];
    const double plo = ns::mul_down(a, yv), phi = ns::mul_up(a, yv);
    zlo = ns::add_down(zlo, -phi);
    zhi = ns::add_up(zhi, -plo);
  }
  const double l = lo[t], u = up[t];
  double shift = 0;
  if (!ns::fin(l) && zhi > 0) {
    shift = (shift < zhi) ? zhi : shift;
    zhi = 0;
    zlo = (0.0 < zlo) ? 0.0 : zlo;
  }
  if (!ns::fin(u) && zlo < 0) {
    shift = (shift < -zlo) ? -zlo : shift;
    zlo = 0;
    zhi = (zhi < 0.0) ? 0.0 : zhi;
  }
  double term;
  bool minus_inf = false;
  if (shift > 0) {
    const double rel = shift / (1.0 + fabs(cj));
    ns::atomic_max_nonneg(stats + b * 4 + 2, rel);
    ns::atomic_max_nonneg(stats + b * 4 + 1, shift);
    if (rel > kMaxAllowedPerturbation) minus_inf = true;
  }
  if (!minus_inf) {
    term = ns::min_product(zlo, zhi, ns::clean(l), ns::clean(u));
    if (isinf(term)) minus_inf = true;
  }
  if (minus_inf) {
    atomicAdd(inf_terms + b, 1);
    term = NAN;
  }
  terms[static_cast<int64_t>(b) * (m + n) + m + j] = term;
}

// One thread per case: lb = 0; lb = add_down(lb, term) in index order (rows, then columns).
__global__ void k_ns_sum(int32_t k, int64_t len, const double* __restrict__ terms, const int32_t* __restrict__ inf_terms,
                         double* __restrict__ bound) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k) return;
  const double* tb = terms + static_cast<int64_t>(b) * len;
  double lb = 0;
  for (int64_t q = 0; q < len; ++q) {
    const double v = tb[q];
    if (!isnan(v)) lb = ns::add_down(lb, v);
  }
  bound[b] = inf_terms[b] > 0 ? -INFINITY : lb;
}

void enqueue_safe_bound(cudaStream_t s, int32_t m, int32_t n, int32_t k, CsrView AT, const double* y, const double* c,
                        const double* lo, const double* up, const double* rl, const double* ru, double* yp,
                        double* terms, double* stats, int32_t* inf_terms, double* bound) {
  B2P_CUDA(cudaMemsetAsync(stats, 0, sizeof(double) * 4 * k, s));
  B2P_CUDA(cudaMemsetAsync(inf_terms, 0, sizeof(int32_t) * k, s));
  if (m) k_ns_rows<<<dim3((m + kBlock - 1) / kBlock, k), kBlock, 0, s>>>(m, n, y, rl, ru, yp, terms, stats);
  if (n)
    k_ns_cols<<<dim3((n + kBlock - 1) / kBlock, k), kBlock, 0, s>>>(m, n, AT, yp, c, lo, up, terms, stats,
                                                                    inf_terms);
  k_ns_sum<<<(k + 127) / 128, 128, 0, s>>>(k, static_cast<int64_t>(m) + n, terms, inf_terms, bound);
  B2P_CUDA(cudaGetLastError());
}

// Device buffers and the stream of one call, released on every exit path;
// the buffers come from the device's stream-ordered pool (no cudaMalloc /
// cudaFree per call).
struct NsBuffers {
  int dev;
  cudaStream_t s;
  std::vector<void*> p;
  ~NsBuffers() {
    for (void* q : p) cudaFreeAsync(q, s);
    cudaStreamDestroy(s);
  }
  template <class T>
  T* put(const T* h, size_t count) {
    void* d = nullptr;
    B2P_CUDA(cudaMallocFromPoolAsync(&d, std::max<size_t>(count, 1) * sizeof(T), device_pool(dev), s));
    p.push_back(d);
    if (h && count) B2P_CUDA(cudaMemcpyAsync(d, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return static_cast<T*>(d);
  }
};

}  // namespace b2p

extern "C" int b2p_safe_dual_bound(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const double* row_dual,
                                   b2p_safe_bound* out) {
  using namespace b2p;
  return guarded([&] {
    if (!lp || !row_dual || !out) throw Error(B2P_ERR_INVALID, "NULL argument");
    if (lp->num_rows < 0 || lp->num_cols < 0 || !lp->start || lp->start[0] != 0)
      throw Error(B2P_ERR_INVALID, "bad dimensions or column pointers");
    const int32_t m = lp->num_rows, n = lp->num_cols, nnz = lp->start[n];
    for (int32_t j = 0; j < n; ++j)
      if (lp->start[j + 1] < lp->start[j]) throw Error(B2P_ERR_INVALID, "start must be non-decreasing");
    for (int32_t q = 0; q < nnz; ++q)
      if (lp->index[q] < 0 || lp->index[q] >= m) throw Error(B2P_ERR_INVALID, "row index out of range");
    if (num_cases > 0 && !cases) throw Error(B2P_ERR_INVALID, "cases is NULL");
    const int k = num_cases > 0 ? num_cases : 1;
    std::vector<double> c(static_cast<size_t>(k) * n), lo(c.size()), up(c.size()), rl(static_cast<size_t>(k) * m),
        ru(rl.size());
    for (int b = 0; b < k; ++b) {
      const b2p_case* cs = num_cases > 0 ? &cases[b] : nullptr;
      auto pick = [&](const double* v, const double* base) { return (cs && v) ? v : base; };
      if (n) {
        std::memcpy(&c[static_cast<size_t>(b) * n], pick(cs ? cs->cost : nullptr, lp->col_cost), sizeof(double) * n);
        std::memcpy(&lo[static_cast<size_t>(b) * n], pick(cs ? cs->col_lower : nullptr, lp->col_lower),
                    sizeof(double) * n);
        std::memcpy(&up[static_cast<size_t>(b) * n], pick(cs ? cs->col_upper : nullptr, lp->col_upper),
                    sizeof(double) * n);
      }
      if (m) {
        std::memcpy(&rl[static_cast<size_t>(b) * m], pick(cs ? cs->row_lower : nullptr, lp->row_lower),
                    sizeof(double) * m);
        std::memcpy(&ru[static_cast<size_t>(b) * m], pick(cs ? cs->row_upper : nullptr, lp->row_upper),
                    sizeof(double) * m);
      }
    }
    const int dev = pick_device(-1);
    B2P_CUDA(cudaSetDevice(dev));
    cudaStream_t s = nullptr;
    B2P_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    NsBuffers r{dev, s, {}};
    const CsrView AT{r.put(lp->start, static_cast<size_t>(n) + 1), r.put(lp->index, nnz), r.put(lp->value, nnz), n};
    const double* dy = r.put(row_dual, static_cast<size_t>(k) * m);
    const double* dc = r.put(c.data(), c.size());
    const double* dlo = r.put(lo.data(), lo.size());
    const double* dup = r.put(up.data(), up.size());
    const double* drl = r.put(rl.data(), rl.size());
    const double* dru = r.put(ru.data(), ru.size());
    double* dyp = r.put<double>(nullptr, static_cast<size_t>(k) * m);
    const int64_t len = static_cast<int64_t>(m) + n;
    double* dterms = r.put<double>(nullptr, static_cast<size_t>(k) * len);
    double* dstats = r.put<double>(nullptr, static_cast<size_t>(k) * 4);
    int32_t* dinf = r.put<int32_t>(nullptr, static_cast<size_t>(k));
    double* dbound = r.put<double>(nullptr, static_cast<size_t>(k));
    enqueue_safe_bound(s, m, n, k, AT, dy, dc, dlo, dup, drl, dru, dyp, dterms, dstats, dinf, dbound);
    std::vector<double> hb(k), hs(static_cast<size_t>(k) * 4);
    std::vector<int32_t> hi(k);
    B2P_CUDA(cudaMemcpyAsync(hb.data(), dbound, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaMemcpyAsync(hs.data(), dstats, sizeof(double) * 4 * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaMemcpyAsync(hi.data(), dinf, sizeof(int32_t) * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaStreamSynchronize(s));
    for (int b = 0; b < k; ++b) {
      out[b].bound = hb[b];
      out[b].infinite_terms = hi[b];
      out[b].pad0 = 0;
      out[b].row_projection = hs[static_cast<size_t>(b) * 4 + 0];
      out[b].max_dual_infeasibility = hs[static_cast<size_t>(b) * 4 + 1];
      out[b].cost_perturbation = hs[static_cast<size_t>(b) * 4 + 2];
    }
  });
}
