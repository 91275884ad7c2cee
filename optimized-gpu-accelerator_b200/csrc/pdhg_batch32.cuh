// FP32-state kernels of the mixed form for batches of k > 1 cases sharing A
// (k-interleaved vectors, element (i, b) at i*k + b).
//
// Operator values and iterates are stored in FP32; every row sum adds the
// exact FP32 x FP32 products in FP64, and the element-wise updates (primal
// and dual steps, projections, Halpern steps) are evaluated in FP64 from the
// FP32 operands and rounded to FP32 when stored.  The check reductions read
// the FP32 state against the FP64 costs and bounds and accumulate in FP64,
// so the host's termination, restart and primal-weight decisions see FP64
// sums.  Same structure as the FP64 kernels of pdhg_kernels.cuh.
#pragma once

#include <cstdint>

#include "pdhg_kernels.cuh"

namespace b2p {

struct CsrView32 {
  const int32_t* __restrict__ ptr;
  const int32_t* __restrict__ idx;
  const float* __restrict__ val;
  int32_t rows;
};

// Row sum in FP64 of exact FP32 products, left to right.
__device__ __forceinline__ double row_dot32(const CsrView32& M, const float* __restrict__ x, int64_t row, int k,
                                            int b) {
  int p = __ldg(M.ptr + row);
  const int e = __ldg(M.ptr + row + 1);
  double s = 0.0;
#pragma unroll 4
  for (; p < e; ++p)
    s = __dadd_rn(s, static_cast<double>(__ldg(M.val + p)) *
                         static_cast<double>(__ldg(x + static_cast<int64_t>(__ldg(M.idx + p)) * k + b)));
  return s;
}

template <bool HALPERN>
__global__ void __launch_bounds__(kBlock) k_primal32(int32_t n, int32_t k, CsrView32 AT, const float* __restrict__ y,
                                                     const float* __restrict__ c, const float* __restrict__ lo,
                                                     const float* __restrict__ up, float* __restrict__ x,
                                                     float* __restrict__ xp, const float* __restrict__ x0,
                                                     const double* __restrict__ tau, IterClock ck, double rho) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<int64_t>(n) * k) return;
  int64_t j;
  int b;
  split(t, k, j, b);
  pdl_wait();
  const double aty = row_dot32(AT, y, j, k, b);
  const double xv = x[t];
  double v = __dsub_rn(xv, __dmul_rn(tau[b], __dsub_rn(static_cast<double>(c[t]), aty)));
  const double l = lo[t], u = up[t];
  v = (v < l) ? l : v;
  v = (u < v) ? u : v;
  xp[t] = static_cast<float>(v);
  if (HALPERN) x[t] = static_cast<float>(halpern_step(xv, v, static_cast<double>(x0[t]), halpern_lambda(ck, b), rho));
  pdl_launch_dependents();
}

template <bool HALPERN>
__global__ void __launch_bounds__(kBlock) k_dual32(int32_t m, int32_t k, CsrView32 A, const float* __restrict__ xp,
                                                   const float* __restrict__ rl, const float* __restrict__ ru,
                                                   float* __restrict__ y, float* __restrict__ yp,
                                                   const float* __restrict__ y0, float* __restrict__ ax,
                                                   float* __restrict__ axp, const float* __restrict__ ax0,
                                                   const double* __restrict__ sigma, IterClock ck, double rho) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<int64_t>(m) * k) return;
  int64_t i;
  int b;
  split(t, k, i, b);
  pdl_wait();
  const double axpv = row_dot32(A, xp, i, k, b);
  const double s = sigma[b], yv = y[t], axv = ax[t];
  const double v = __dsub_rn(yv, __dmul_rn(s, __dsub_rn(__dmul_rn(2.0, axpv), axv)));
  double w = __ddiv_rn(-v, s);
  const double l = rl[t], u = ru[t];
  w = (w < l) ? l : w;
  w = (u < w) ? u : w;
  const double ypv = __dadd_rn(v, __dmul_rn(s, w));
  axp[t] = static_cast<float>(axpv);
  yp[t] = static_cast<float>(ypv);
  if (HALPERN) {
    const double lam = halpern_lambda(ck, b);
    y[t] = static_cast<float>(halpern_step(yv, ypv, static_cast<double>(y0[t]), lam, rho));
    ax[t] = static_cast<float>(halpern_step(axv, axpv, static_cast<double>(ax0[t]), lam, rho));
  }
  pdl_launch_dependents();
}

// Halpern steps of x, y and Ax at a check iteration (after the reductions).
static __global__ void __launch_bounds__(kBlock) k_halpern_all32(int32_t n, int32_t m, int32_t k, float* __restrict__ x,
                                                                 const float* __restrict__ xp,
                                                                 const float* __restrict__ x0, float* __restrict__ y,
                                                                 const float* __restrict__ yp,
                                                                 const float* __restrict__ y0, float* __restrict__ ax,
                                                                 const float* __restrict__ axp,
                                                                 const float* __restrict__ ax0, IterClock ck,
                                                                 double rho) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nx = static_cast<int64_t>(n) * k, ny = static_cast<int64_t>(m) * k;
  if (t < nx) {
    const int b = static_cast<int>(t % k);
    x[t] = static_cast<float>(halpern_step(x[t], xp[t], x0[t], halpern_lambda(ck, b), rho));
  } else if (t < nx + ny) {
    const int64_t u = t - nx;
    const int b = static_cast<int>(u % k);
    const double lam = halpern_lambda(ck, b);
    y[u] = static_cast<float>(halpern_step(y[u], yp[u], y0[u], lam, rho));
    ax[u] = static_cast<float>(halpern_step(ax[u], axp[u], ax0[u], lam, rho));
  }
}

// Row part of the check of the FP32 state against the FP64 row bounds (see
// k_check_rows).  grid = (G, k).
static __global__ void __launch_bounds__(kBlock) k_check_rows32(int32_t m, int32_t k, const float* __restrict__ axp,
                                                                const double* __restrict__ rl,
                                                                const double* __restrict__ ru,
                                                                const float* __restrict__ yp,
                                                                const float* __restrict__ y,
                                                                const float* __restrict__ y0,
                                                                const double* __restrict__ rfac,
                                                                double* __restrict__ partial) {
  __shared__ double sh[kRowSums * (kBlock / 32)];
  const int b = blockIdx.y;
  double s[kRowSums] = {0, 0, 0, 0, 0};
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i * k + b;
    const double a = axp[t], l = rl[t], u = ru[t];
    double e1 = l - a, e2 = a - u;
    e1 = (e1 < 0.0) ? 0.0 : e1;
    e2 = (e2 < 0.0) ? 0.0 : e2;
    const double res = (e1 + e2) * rfac[i];
    s[0] += res * res;
    const double yv = yp[t];
    if (yv > 0.0 && l > -1e300)
      s[1] += yv * l;
    else if (yv < 0.0 && u < 1e300)
      s[1] += yv * u;
    s[2] += yv * yv;
    const double d1 = static_cast<double>(y[t]) - yv, d2 = yv - static_cast<double>(y0[t]);
    s[3] += d1 * d1;
    s[4] += d2 * d2;
  }
  block_reduce<kRowSums>(s, sh);
  if (threadIdx.x == 0) {
    double* o = partial + (static_cast<int64_t>(b) * gridDim.x + blockIdx.x) * kRowSums;
#pragma unroll
    for (int q = 0; q < kRowSums; ++q) o[q] = s[q];
  }
}

// Column part: A^T y+ from the FP32 operator and state, against the FP64
// costs and column bounds (see k_check_cols).  grid = (G, k).
static __global__ void __launch_bounds__(kBlock) k_check_cols32(int32_t n, int32_t k, CsrView32 AT,
                                                                const float* __restrict__ yp,
                                                                const float* __restrict__ xp,
                                                                const float* __restrict__ x,
                                                                const float* __restrict__ x0,
                                                                const double* __restrict__ c,
                                                                const double* __restrict__ lo,
                                                                const double* __restrict__ up,
                                                                const double* __restrict__ cfac,
                                                                double* __restrict__ partial) {
  __shared__ double sh[kRowSums * (kBlock / 32)];
  const int b = blockIdx.y;
  double s[kRowSums] = {0, 0, 0, 0, 0};
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = j * k + b;
    const double atyp = row_dot32(AT, yp, j, k, b);
    const double cv = c[t], l = lo[t], u = up[t], xpv = xp[t];
    const double d = cv - atyp;
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
    const double d1 = static_cast<double>(x[t]) - xpv, d2 = xpv - static_cast<double>(x0[t]);
    s[3] += d1 * d1;
    s[4] += d2 * d2;
  }
  block_reduce<kRowSums>(s, sh);
  if (threadIdx.x == 0) {
    double* o = partial + (static_cast<int64_t>(b) * gridDim.x + blockIdx.x) * kRowSums;
#pragma unroll
    for (int q = 0; q < kRowSums; ++q) o[q] = s[q];
  }
}

}  // namespace b2p
