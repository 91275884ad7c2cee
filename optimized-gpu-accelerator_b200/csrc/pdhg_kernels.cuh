// Device kernels of the PDHG engine (sm_100a, FP64 plain form).
//
// One PDHG iteration is two fused kernels instead of the reference's eight
// launches (src/pdhg/pdhg.cpp:588-662, kernels.cpp:19-85):
//   k_primal : aty = A^T y (row j of A^T), x+ = proj(x - tau (c - aty)),
//              Halpern step of x                          (spmvT + primalStep + halpern x)
//   k_dual   : ax+ = A x+ (row i of A), y+ = v + sigma proj(-v/sigma),
//              Halpern steps of y and Ax                  (spmv + dualStep + halpern y, Ax)
// At a check iteration the Halpern steps are deferred to k_halpern_all so
// that the check reductions see the pre-Halpern x and y, as in the reference.
//
// Numerics: every row sum runs left to right from s = 0 with separately
// rounded products and sums (__dmul_rn/__dadd_rn, no FMA contraction), which
// is exactly CpuBackend::mult (src/pdhg/pdhg.cpp:93-103); the element-wise
// updates use the reference's operation order.  The iterates are therefore
// bit-identical to the reference CPU run as long as the host takes the same
// restart decisions.  The check reductions are deterministic trees.
//
// Vectors of k cases sharing A are k-interleaved: element (i, b) at i*k + b
// (src/pdhg/kernels.cpp:1-4).
#pragma once

#include <cstdint>

namespace b2p {

constexpr int kBlock = 256;
constexpr int kRowSums = 5;  // per case, per block: see CheckSum
constexpr int kNumSums = 10;

// Per-case results of one check (device -> host once per check interval).
enum CheckSum : int {
  CS_ROW_RES2 = 0,  // sum (unscaled primal residual)^2          (kkt_rows [0])
  CS_ROW_DOBJ = 1,  // row part of the dual objective            (kkt_rows [1])
  CS_Y2 = 2,        // sum y+^2                                  (kkt_rows [2])
  CS_DY2 = 3,       // sum (y - y+)^2                            (diff2(Y, YP))
  CS_AY2 = 4,       // sum (y+ - y0)^2                           (diff2(YP, Y0))
  CS_COL_RES2 = 5,  // sum (unscaled dual residual)^2            (kkt_cols [0])
  CS_POBJ = 6,      // c' x+                                     (kkt_cols [1])
  CS_COL_DOBJ = 7,  // column part of the dual objective         (kkt_cols [2])
  CS_DX2 = 8,       // sum (x - x+)^2                            (diff2(X, XP))
  CS_AX2 = 9        // sum (x+ - x0)^2                           (diff2(XP, X0))
};

// Programmatic dependent launch: a kernel launched with the PDL attribute
// waits here for the previous kernel's memory before reading what it wrote,
// and lets the next kernel start its launch once its own stores are issued.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" :::); }

struct CsrView {
  const int32_t* __restrict__ ptr;
  const int32_t* __restrict__ idx;
  const double* __restrict__ val;
  int32_t rows;
};

// Iteration counter of case b at the current iteration: the reference keeps
// iter[b] (reset to 0 at a restart, +1 after each Halpern step); here it is
// (it_base + local) - restart_at[b], so a captured interval can be replayed.
struct IterClock {
  const int64_t* __restrict__ it_base;
  const int64_t* __restrict__ restart_at;
  int32_t local;
};

__device__ __forceinline__ double halpern_lambda(const IterClock& ck, int b) {
  const double j = static_cast<double>(*ck.it_base + ck.local - ck.restart_at[b]);
  return __ddiv_rn(__dadd_rn(j, 1.0), __dadd_rn(j, 2.0));
}

// z = lam((1+rho) z+ - rho z) + (1-lam) z0          (src/pdhg/pdhg.cpp:138-146)
__device__ __forceinline__ double halpern_step(double z, double zp, double z0, double lam, double rho) {
  const double a = __dsub_rn(__dmul_rn(__dadd_rn(1.0, rho), zp), __dmul_rn(rho, z));
  return __dadd_rn(__dmul_rn(lam, a), __dmul_rn(__dsub_rn(1.0, lam), z0));
}

// Left-to-right row sum  s = (((0 + v0 x0) + v1 x1) + ...)
__device__ __forceinline__ double row_dot(const CsrView& M, const double* __restrict__ x, int64_t row, int k, int b) {
  int p = __ldg(M.ptr + row);
  const int e = __ldg(M.ptr + row + 1);
  double s = 0.0;
  if (k == 1) {
#pragma unroll 4
    for (; p < e; ++p) s = __dadd_rn(s, __dmul_rn(__ldg(M.val + p), __ldg(x + __ldg(M.idx + p))));
  } else {
#pragma unroll 4
    for (; p < e; ++p)
      s = __dadd_rn(s, __dmul_rn(__ldg(M.val + p), __ldg(x + static_cast<int64_t>(__ldg(M.idx + p)) * k + b)));
  }
  return s;
}

__device__ __forceinline__ void split(int64_t t, int k, int64_t& row, int& b) {
  if (k == 1) {
    row = t;
    b = 0;
  } else {
    row = t / k;
    b = static_cast<int>(t - row * k);
  }
}

// ---- per-iteration kernels ------------------------------------------------

// Loads and stores of vectors that one kernel touches once per element: with
// STREAM they are evict-first (ld.global.cs / st.global.cs), so that L2 keeps
// the vector the other kernel gathers (y for k_primal, x+ for k_dual).
template <bool STREAM>
__device__ __forceinline__ double ld_vec(const double* p) {
  return STREAM ? __ldcs(p) : *p;
}
template <bool STREAM>
__device__ __forceinline__ void st_vec(double* p, double v) {
  if (STREAM)
    __stcs(p, v);
  else
    *p = v;
}

// Left-to-right row sums of CPT cases of one row at once (cases b[q], valid
// when b[q] < k): the row's index and value are loaded once per entry and the
// CPT gathers are independent, so a thread keeps CPT loads in flight.  With
// WARPROW (every lane of the warp on the same row: k / CPT a multiple of 32)
// the lanes load 32 of the row's entries at a time, coalesced, and pass each
// entry's index and value by shuffle, so a gather waits on no index load.
template <int CPT, bool WARPROW>
__device__ __forceinline__ void row_dot_cases(const CsrView& M, const double* __restrict__ x, int64_t row, int k,
                                              const int (&b)[CPT], double (&s)[CPT]) {
  int p = __ldg(M.ptr + row);
  const int e = __ldg(M.ptr + row + 1);
#pragma unroll
  for (int q = 0; q < CPT; ++q) s[q] = 0.0;
  if (WARPROW) {
    const int lane = threadIdx.x & 31;
    for (; p < e; p += 32) {
      const int cnt = (e - p) < 32 ? (e - p) : 32;  // the same in every lane
      int my_idx = 0;
      double my_val = 0.0;
      if (lane < cnt) {
        my_idx = __ldg(M.idx + p + lane);
        my_val = __ldg(M.val + p + lane);
      }
#pragma unroll 4
      for (int r = 0; r < cnt; ++r) {
        const int64_t base = static_cast<int64_t>(__shfl_sync(0xffffffffu, my_idx, r)) * k;
        const double a = __shfl_sync(0xffffffffu, my_val, r);
#pragma unroll
        for (int q = 0; q < CPT; ++q)
          if (b[q] < k) s[q] = __dadd_rn(s[q], __dmul_rn(a, __ldg(x + base + b[q])));
      }
    }
  } else {
#pragma unroll 4
    for (; p < e; ++p) {
      const int64_t base = static_cast<int64_t>(__ldg(M.idx + p)) * k;
      const double a = __ldg(M.val + p);
#pragma unroll
      for (int q = 0; q < CPT; ++q)
        if (b[q] < k) s[q] = __dadd_rn(s[q], __dmul_rn(a, __ldg(x + base + b[q])));
    }
  }
}

// Row and first case of this thread in a batch kernel (the layouts TR are
// described with the kernels below); false for a thread past the last row or
// past kh.
template <int TR>
__device__ __forceinline__ bool batch_thread(int32_t rows, int kh, int64_t& row, int& b0) {
  if constexpr (TR == 0) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<int64_t>(rows) * kh) return false;
    row = t / kh;
    b0 = static_cast<int>(t - row * kh);
    return true;
  } else {
    const int64_t row_blocks = (static_cast<int64_t>(rows) + TR - 1) / TR;
    const int64_t chunk = blockIdx.x / row_blocks;
    row = (blockIdx.x - chunk * row_blocks) * TR + (threadIdx.x >> 5);
    b0 = static_cast<int>(chunk * 32) + static_cast<int>(threadIdx.x & 31);
    return row < rows && b0 < kh;
  }
}

// Threads per block and the register cap (blocks per SM) of a batch kernel.
constexpr int batch_block(int tr) { return tr ? 32 * tr : kBlock; }
constexpr int batch_min_blocks(int tr, int cpt) { return (2048 / batch_block(tr)) / cpt; }

// Batch kernels (k > 1 cases sharing A, k-interleaved vectors).  A thread
// takes one row and the cases b0 + q kh, q < CPT (kh = ceil(k / CPT)):
//   TR = 0: thread t of the grid takes row t / kh and b0 = t % kh (a row's
//           cases are spread over consecutive threads: the warps of a block
//           share the row's entries);
//   TR > 0: a block of TR warps takes TR consecutive rows, one per warp, for
//           one chunk of 32 consecutive b0 (blocks run chunk by chunk): where
//           nearby rows share columns, the warps of a block gather the same
//           256-byte slices of the k-interleaved vector, and the later ones
//           find them in L1; the slice of the gathered vector that one chunk
//           reads (rows x 32 x 8 bytes) stays in L2 while the chunk runs.
// WARPROW requires kh to be a multiple of 32 (whole warps per row).
// k_primal : aty = A^T y (row j of A^T), x+ = proj(x - tau (c - aty)),
//            Halpern step of x                    (spmvT + primalStep + halpern x)
// k_dual   : ax+ = A x+ (row i of A), y+ = v + sigma proj(-v/sigma),
//            Halpern steps of y and Ax            (spmv + dualStep + halpern y, Ax)
// The vectors a kernel reads but the kernel it may overlap (programmatic
// dependent launch) does not write are loaded before griddepcontrol.wait, so
// their latency overlaps the previous kernel's tail and this kernel's
// gathers.  (k_restart and k_halpern_all, which write x, x0, y, y0, Ax and
// A x0, do not trigger early: a kernel that follows them starts only when
// they have completed.)
template <bool HALPERN, bool STREAM = false, int CPT = 1, bool WARPROW = false, int TR = 0>
static __global__ void __launch_bounds__(batch_block(TR), batch_min_blocks(TR, CPT))
    k_primal(int32_t n, int32_t k, CsrView AT, const double* __restrict__ y, const double* __restrict__ c,
             const double* __restrict__ lo, const double* __restrict__ up, double* __restrict__ x,
             double* __restrict__ xp, const double* __restrict__ x0, const double* __restrict__ tau, IterClock ck,
             double rho) {
  const int kh = (k + CPT - 1) / CPT;
  int64_t j;
  int b0;
  if (!batch_thread<TR>(n, kh, j, b0)) return;
  int b[CPT];
#pragma unroll
  for (int q = 0; q < CPT; ++q) b[q] = b0 + q * kh;
  double xv[CPT], cv[CPT], l[CPT], u[CPT], x0v[CPT];
#pragma unroll
  for (int q = 0; q < CPT; ++q)
    if (b[q] < k) {
      const int64_t e = j * k + b[q];
      xv[q] = ld_vec<STREAM>(x + e);
      cv[q] = ld_vec<STREAM>(c + e);
      l[q] = ld_vec<STREAM>(lo + e);
      u[q] = ld_vec<STREAM>(up + e);
      x0v[q] = HALPERN ? ld_vec<STREAM>(x0 + e) : 0.0;
    }
  pdl_wait();
  double aty[CPT];
  row_dot_cases<CPT, WARPROW>(AT, y, j, k, b, aty);
#pragma unroll
  for (int q = 0; q < CPT; ++q)
    if (b[q] < k) {
      const int64_t e = j * k + b[q];
      // x+ = proj_[lo,up](x - tau (c - A^T y))          (src/pdhg/pdhg.cpp:116-125)
      double v = __dsub_rn(xv[q], __dmul_rn(tau[b[q]], __dsub_rn(cv[q], aty[q])));
      v = (v < l[q]) ? l[q] : v;
      v = (u[q] < v) ? u[q] : v;
      xp[e] = v;  // gathered by k_dual: kept in L2
      if (HALPERN) st_vec<STREAM>(x + e, halpern_step(xv[q], v, x0v[q], halpern_lambda(ck, b[q]), rho));
    }
  pdl_launch_dependents();
}

template <bool HALPERN, bool STREAM = false, int CPT = 1, bool WARPROW = false, int TR = 0>
static __global__ void __launch_bounds__(batch_block(TR), batch_min_blocks(TR, CPT))
    k_dual(int32_t m, int32_t k, CsrView A, const double* __restrict__ xp, const double* __restrict__ rl,
           const double* __restrict__ ru, double* __restrict__ y, double* __restrict__ yp,
           const double* __restrict__ y0, double* __restrict__ ax, double* __restrict__ axp,
           const double* __restrict__ ax0, const double* __restrict__ sigma, IterClock ck, double rho) {
  const int kh = (k + CPT - 1) / CPT;
  int64_t i;
  int b0;
  if (!batch_thread<TR>(m, kh, i, b0)) return;
  int b[CPT];
#pragma unroll
  for (int q = 0; q < CPT; ++q) b[q] = b0 + q * kh;
  double axv[CPT], yv[CPT], l[CPT], u[CPT], y0v[CPT], ax0v[CPT];
#pragma unroll
  for (int q = 0; q < CPT; ++q)
    if (b[q] < k) {
      const int64_t e = i * k + b[q];
      axv[q] = ld_vec<STREAM>(ax + e);
      yv[q] = ld_vec<STREAM>(y + e);
      l[q] = ld_vec<STREAM>(rl + e);
      u[q] = ld_vec<STREAM>(ru + e);
      y0v[q] = HALPERN ? ld_vec<STREAM>(y0 + e) : 0.0;
      ax0v[q] = HALPERN ? ld_vec<STREAM>(ax0 + e) : 0.0;
    }
  pdl_wait();
  double axpv[CPT];
  row_dot_cases<CPT, WARPROW>(A, xp, i, k, b, axpv);
#pragma unroll
  for (int q = 0; q < CPT; ++q)
    if (b[q] < k) {
      const int64_t e = i * k + b[q];
      // v = y - sigma (2 A x+ - A x);  y+ = v + sigma proj_[L,U](-v / sigma)   (src/pdhg/pdhg.cpp:126-137)
      const double s = sigma[b[q]];
      const double v = __dsub_rn(yv[q], __dmul_rn(s, __dsub_rn(__dmul_rn(2.0, axpv[q]), axv[q])));
      double w = __ddiv_rn(-v, s);
      w = (w < l[q]) ? l[q] : w;
      w = (u[q] < w) ? u[q] : w;
      const double ypv = __dadd_rn(v, __dmul_rn(s, w));
      st_vec<STREAM>(axp + e, axpv[q]);
      st_vec<STREAM>(yp + e, ypv);
      if (HALPERN) {
        const double lam = halpern_lambda(ck, b[q]);
        y[e] = halpern_step(yv[q], ypv, y0v[q], lam, rho);  // gathered by k_primal: kept in L2
        st_vec<STREAM>(ax + e, halpern_step(axv[q], axpv[q], ax0v[q], lam, rho));
      }
    }
  pdl_launch_dependents();
}

// Halpern steps of x, y and Ax at a check iteration (after the reductions).
static __global__ void __launch_bounds__(kBlock) k_halpern_all(int32_t n, int32_t m, int32_t k, double* __restrict__ x,
                                                        const double* __restrict__ xp, const double* __restrict__ x0,
                                                        double* __restrict__ y, const double* __restrict__ yp,
                                                        const double* __restrict__ y0, double* __restrict__ ax,
                                                        const double* __restrict__ axp,
                                                        const double* __restrict__ ax0, IterClock ck, double rho) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nx = static_cast<int64_t>(n) * k, ny = static_cast<int64_t>(m) * k;
  if (t < nx) {
    const int b = static_cast<int>(k == 1 ? 0 : t % k);
    x[t] = halpern_step(x[t], xp[t], x0[t], halpern_lambda(ck, b), rho);
  } else if (t < nx + ny) {
    const int64_t u = t - nx;
    const int b = static_cast<int>(k == 1 ? 0 : u % k);
    const double lam = halpern_lambda(ck, b);
    y[u] = halpern_step(y[u], yp[u], y0[u], lam, rho);
    ax[u] = halpern_step(ax[u], axp[u], ax0[u], lam, rho);
  }
}

// Masked restart z = z0 = z+ for x, y, Ax and iteration counter reset
// (src/pdhg/pdhg.cpp:153-165).  Runs after the interval's clock advanced, so
// the next iteration (index *it_base) has counter 0.  T: iterate type.
template <class T>
__global__ void __launch_bounds__(kBlock) k_restart(int32_t n, int32_t m, int32_t k, const int32_t* __restrict__ mask,
                                                    T* __restrict__ x, T* __restrict__ x0, const T* __restrict__ xp,
                                                    T* __restrict__ y, T* __restrict__ y0, const T* __restrict__ yp,
                                                    T* __restrict__ ax, T* __restrict__ ax0,
                                                    const T* __restrict__ axp, const int64_t* __restrict__ it_base,
                                                    int64_t* __restrict__ restart_at) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nx = static_cast<int64_t>(n) * k, ny = static_cast<int64_t>(m) * k;
  if (t < k && mask[t]) restart_at[t] = *it_base;
  if (t < nx) {
    if (mask[k == 1 ? 0 : t % k]) x[t] = x0[t] = xp[t];
  } else if (t < nx + ny) {
    const int64_t u = t - nx;
    if (mask[k == 1 ? 0 : u % k]) {
      y[u] = y0[u] = yp[u];
      ax[u] = ax0[u] = axp[u];
    }
  }
}

// dst = src with a change of floating-point type (round to nearest).
template <class S, class D>
__global__ void __launch_bounds__(kBlock) k_convert(int64_t len, const S* __restrict__ src, D* __restrict__ dst) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < len) dst[t] = static_cast<D>(src[t]);
}

// restart_at[b] = *it_base for all cases (a fresh restart at the next iteration).
static __global__ void k_restart_clock(int32_t k, const int64_t* __restrict__ it_base, int64_t* __restrict__ restart_at) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < k) restart_at[t] = *it_base;
}

// ---- check reductions --------------------------------------------------------

template <int NQ>
__device__ __forceinline__ void block_reduce(double (&s)[NQ], double* sh /* [NQ][kBlock/32] */) {
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) sh[q * (kBlock / 32) + warp] = s[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double v = lane < kBlock / 32 ? sh[q * (kBlock / 32) + lane] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      s[q] = v;
    }
  }
}

// Row part of the check at (x+, y+): kkt_rows (src/pdhg/pdhg.cpp:166-180) +
// diff2(Y, YP) + diff2(YP, Y0).  grid = (G, k); partial[(b*G + g)*5 + q].
static __global__ void __launch_bounds__(kBlock) k_check_rows(int32_t m, int32_t k, const double* __restrict__ axp,
                                                       const double* __restrict__ rl, const double* __restrict__ ru,
                                                       const double* __restrict__ yp, const double* __restrict__ y,
                                                       const double* __restrict__ y0,
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
    const double d1 = y[t] - yv, d2 = yv - y0[t];
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

// Column part: A^T y+ (spmvT(YP, ATYP)) fused with kkt_cols
// (src/pdhg/pdhg.cpp:181-196) + diff2(X, XP) + diff2(XP, X0).
// `atyp` (k = 1 only) is A^T y+ computed by the binned SpMV; when NULL the
// row sums are computed here.
static __global__ void __launch_bounds__(kBlock) k_check_cols(int32_t n, int32_t k, CsrView AT, const double* __restrict__ yp,
                                                       const double* __restrict__ atyp_in,
                                                       const double* __restrict__ xp, const double* __restrict__ x,
                                                       const double* __restrict__ x0, const double* __restrict__ c,
                                                       const double* __restrict__ lo, const double* __restrict__ up,
                                                       const double* __restrict__ cfac,
                                                       double* __restrict__ partial) {
  __shared__ double sh[kRowSums * (kBlock / 32)];
  const int b = blockIdx.y;
  double s[kRowSums] = {0, 0, 0, 0, 0};
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = j * k + b;
    const double atyp = atyp_in ? atyp_in[t] : row_dot(AT, yp, j, k, b);
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
    const double d1 = x[t] - xpv, d2 = xpv - x0[t];
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

// Sums the block partials of case b (grid = k) into out[b*10 + CheckSum] and
// advances the interval clock by L iterations.
static __global__ void __launch_bounds__(kBlock) k_check_finalize(int32_t k, int32_t g_rows, int32_t g_cols,
                                                           const double* __restrict__ prow,
                                                           const double* __restrict__ pcol, double* __restrict__ out,
                                                           int64_t* __restrict__ it_base, int32_t L) {
  __shared__ double sh[kNumSums * (kBlock / 32)];
  const int b = blockIdx.x;
  double s[kNumSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int g = threadIdx.x; g < g_rows; g += blockDim.x) {
    const double* p = prow + (static_cast<int64_t>(b) * g_rows + g) * kRowSums;
#pragma unroll
    for (int q = 0; q < kRowSums; ++q) s[q] += p[q];
  }
  for (int g = threadIdx.x; g < g_cols; g += blockDim.x) {
    const double* p = pcol + (static_cast<int64_t>(b) * g_cols + g) * kRowSums;
#pragma unroll
    for (int q = 0; q < kRowSums; ++q) s[kRowSums + q] += p[q];
  }
  block_reduce<kNumSums>(s, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < kNumSums; ++q) out[static_cast<int64_t>(b) * kNumSums + q] = s[q];
    if (b == 0) *it_base += L;
  }
}

// x = z / nz (one power-iteration normalisation step, src/pdhg/pdhg.cpp:419).
static __global__ void __launch_bounds__(kBlock) k_div_scalar(int32_t len, const double* __restrict__ z, double nz,
                                                             double* __restrict__ x) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < len) x[t] = __ddiv_rn(z[t], nz);
}

// Plain k-interleaved CSR SpMV y = M x (CpuBackend::mult order).
static __global__ void __launch_bounds__(kBlock) k_spmv(int32_t rows, int32_t k, CsrView M, const double* __restrict__ x,
                                                 double* __restrict__ y) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<int64_t>(rows) * k) return;
  int64_t i;
  int b;
  split(t, k, i, b);
  y[t] = row_dot(M, x, i, k, b);
}

}  // namespace b2p
