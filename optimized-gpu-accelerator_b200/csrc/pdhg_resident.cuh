// Resident PDHG kernel for one LP whose operators fit in the SMs' shared
// memory (about 30 MB on a B200: C1-C3-sized LPs).
//
// One cooperative launch runs a whole check interval (L iterations and the
// check).  Block b owns a contiguous range of columns [c0, c1) (rows of A^T)
// and of rows [r0, r1) (rows of A), chosen on the host so that nonzeros are
// balanced.  At launch the block copies its slices of A^T and A (values,
// indices, pointers) and every vector entry it owns (x, x0, c, l, u / y, y0,
// Ax, Ax0, L, U) into shared memory; during the interval the only global
// traffic is the exchange of x+ and y through two L2-resident vectors:
//
//   primal phase: aty_j = A^T[j,:] . y      (gather y),  x+_j, Halpern x_j,
//                 publish x+_j
//   grid barrier
//   dual phase:   ax+_i = A[i,:] . x+       (gather x+), y+_i, Halpern y_i, Ax_i,
//                 publish y_i (y+_i at the check iteration)
//   grid barrier
//
// At the end of the interval the block computes its part of the check
// (A^T y+ again for the dual residual, KKT sums, the four movement norms),
// applies the deferred Halpern step, writes its state back to global memory
// for the host's restart / extraction, and block 0 sums the per-block
// partials in a fixed order (deterministic).
//
// The kernel is templated on the iterate type T.  T = double is the plain
// form.  T = float is the mixed form: operator values, iterates and their
// updates in FP32 (each row sum still accumulates exact FP32 x FP32 products in
// FP64), while every check sum accumulates in FP64 against the FP64 costs and
// bounds, and the host's decisions stay FP64.
//
// The grid barrier is a monotonic arrival counter with a generation word;
// waits are bounded: after kSpinLimit polls a block records an error and all
// blocks leave the interval at the next barrier, so a fault can never hang
// the GPU.  Co-residency of all blocks is guaranteed by the cooperative launch.
#pragma once

#include <cstdint>

#include "pdhg_kernels.cuh"

namespace b2p {

constexpr int kResidentThreads = 1024;
constexpr int kResUnroll = 8;
constexpr unsigned kSpinLimit = 1u << 22;  // ~2 s of polling at ~0.5 us per poll

// Round-to-nearest arithmetic without contraction, per iterate type.
template <class T>
struct Rn;
template <>
struct Rn<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};
template <>
struct Rn<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
};

// z = lam((1+rho) z+ - rho z) + (1-lam) z0 in type T.
template <class T>
__device__ __forceinline__ T halpern_t(T z, T zp, T z0, T lam, T rho) {
  using R = Rn<T>;
  const T a = R::sub(R::mul(R::add(T(1), rho), zp), R::mul(rho, z));
  return R::add(R::mul(lam, a), R::mul(R::sub(T(1), lam), z0));
}

template <class T>
struct ResidentArgs {
  // partition: block b owns columns [cb[b], cb[b+1]) and rows [rb[b], rb[b+1])
  const int32_t* __restrict__ cb;
  const int32_t* __restrict__ rb;
  // A (CSR, m rows) and A^T (CSR, n rows): shared pointers, values of type T
  const int32_t *a_ptr, *a_idx, *t_ptr, *t_idx;
  const T *a_val, *t_val;
  // global state (type T)
  T *x, *x0, *xp, *y, *y0, *yp, *ax, *ax0, *axp;
  const T *c, *lo, *up, *rl, *ru;
  // FP64 data of the check
  const double *c64, *lo64, *up64, *rl64, *ru64, *rfac, *cfac;
  const double *tau, *sigma;
  IterClock ck;  // ck.local unused (the kernel walks l = 0..L-1)
  double rho;
  int32_t L;
  int32_t g_cols, g_rows;      // lanes per short row (A^T, A)
  int32_t lt_cols, lt_rows;    // longer rows go to the warp pass
  // synchronisation and output
  unsigned* arrive;
  unsigned* gen;
  int32_t* error;
  double* partial;  // gridDim.x * kNumSums
  double* sums;     // kNumSums
  int64_t* it_base;
};

// Bounded grid barrier.  Arrival is a fire-and-forget release add on a
// monotonic counter; each block's thread 0 then polls the counter with
// acquire loads until all gridDim.x blocks of this epoch have arrived (the
// __syncthreads on both sides extend the ordering to the whole block).
// Returns false (on every thread) once any block has recorded a timeout.
template <class T>
__device__ __forceinline__ bool grid_barrier(const ResidentArgs<T>& a, unsigned& epoch) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ++epoch;
    const unsigned target = epoch * gridDim.x;
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(a.arrive) : "memory");
    unsigned spins = 0;
    int ok = 1;
    while (true) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a.arrive) : "memory");
      if (v >= target) break;
      if (++spins > kSpinLimit || (spins % 64 == 0 && *reinterpret_cast<volatile int32_t*>(a.error))) {
        atomicExch(a.error, 1);
        ok = 0;
        break;
      }
      if (spins > 4096) __nanosleep(64);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <int W>
__device__ __forceinline__ double res_tree(double s) {
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, off));
  return s;
}

// Sum of entries p = p0, p0+S, ... < end of a shared-memory CSR slice, left
// to right; the gathers of each round of kResUnroll entries are issued
// together and the values are read from shared memory as they are consumed.
// The gathered vector is written by other blocks between phases, so it is
// read with ld.global.ca (L1-cacheable, not the read-only path): every phase
// starts after the grid barrier's acquire, which the PTX memory model orders
// before these loads through bar.sync, so a cached line can never be stale
// across phases, and entries repeated within a phase hit in L1.
template <class T>
__device__ __forceinline__ double res_lane_sum(const int32_t* s_idx, const T* s_val, int p0, int end, int S,
                                               const T* xg) {
  double s = 0.0;
  bool first = true;
  for (int p = p0; p < end; p += kResUnroll * S) {
    T xv[kResUnroll];
#pragma unroll
    for (int u = 0; u < kResUnroll; ++u) {
      const int q = p + u * S;
      xv[u] = q < end ? __ldca(xg + s_idx[q]) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kResUnroll; ++u) {
      const int q = p + u * S;
      if (q < end) {
        // exact for FP32 inputs; the reference's rounded product for FP64
        const double prod = __dmul_rn(static_cast<double>(s_val[q]), static_cast<double>(xv[u]));
        s = first ? prod : __dadd_rn(s, prod);
        first = false;
      }
    }
  }
  return s;
}

// Row-ordered list of the rows longer than lt, built by warp 0 with ballots
// (deterministic).  Returns the count (valid after the trailing barrier).
__device__ __forceinline__ int res_long_list(const int32_t* s_ptr, int nrows, int lt, int32_t* s_list,
                                             int* s_count) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int count = 0;
    for (int base = 0; base < nrows; base += 32) {
      const int r = base + lane;
      const bool lng = r < nrows && s_ptr[r + 1] - s_ptr[r] > lt;
      const unsigned bal = __ballot_sync(0xffffffffu, lng);
      if (lng) s_list[count + __popc(bal & ((1u << lane) - 1u))] = r;
      count += __popc(bal);
    }
    if (lane == 0) *s_count = count;
  }
  __syncthreads();
  return *s_count;
}

// One pass over the block's rows of a shared-memory CSR slice: short rows by
// groups of G lanes, then the long rows of `s_long` (> lt) by whole warps.
// epi(local_row, value) runs on one fixed thread per row.  Every thread of
// the block must call.
template <int G, class T, class Epi>
__device__ __forceinline__ void res_rows(const int32_t* s_ptr, const int32_t* s_idx, const T* s_val, int nrows, int lt,
                                         const int32_t* s_long, int nlong, const T* xg, Epi&& epi) {
  const int gid = threadIdx.x / G, gl = threadIdx.x & (G - 1);
  constexpr int kGroups = kResidentThreads / G;
  for (int base = 0; base < nrows; base += kGroups) {
    const int r = base + gid;
    int beg = 0, end = 0;
    bool mine = false;
    if (r < nrows) {
      beg = s_ptr[r];
      end = s_ptr[r + 1];
      mine = end - beg <= lt;
      if (!mine) end = beg;
    }
    double s = res_lane_sum(s_idx, s_val, beg + gl, end, G, xg);
    s = res_tree<G>(s);
    if (mine && gl == 0) epi(r, s);
  }
  // long rows go to the highest warps, which have no short row when the
  // block's rows fit in one short pass, so both passes overlap
  const int warp = kResidentThreads / 32 - 1 - (threadIdx.x >> 5), lane = threadIdx.x & 31;
  constexpr int kWarps = kResidentThreads / 32;
  for (int q = warp; q < nlong; q += kWarps) {
    const int r = s_long[q];
    double s = res_lane_sum(s_idx, s_val, s_ptr[r] + lane, s_ptr[r + 1], 32, xg);
    s = res_tree<32>(s);
    if (lane == 0) epi(r, s);
  }
}

// Fixed-order block reduction of NQ sums; the result is valid on thread 0.
template <int NQ>
__device__ __forceinline__ void res_block_sum(double (&v)[NQ], double* s_red /* NQ * 32 */) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = res_tree<32>(v[q]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) s_red[q * 32 + warp] = v[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = res_tree<32>(lane < kResidentThreads / 32 ? s_red[q * 32 + lane] : 0.0);
  }
  __syncthreads();
}

// Shared-memory bytes of a block with nc columns, nr rows, tn / an nonzeros
// in its A^T / A slices, iterates of type T.
template <class T>
__host__ __device__ inline size_t resident_smem_bytes(int nc, int nr, int tn, int an) {
  const size_t d = kNumSums * 32;
  const size_t t = static_cast<size_t>(tn) + an + 6ull * nc + 8ull * nr;
  const size_t i = static_cast<size_t>(tn) + an + nc + 1 + nr + 1 + nc + nr + 2;
  return 8 * d + sizeof(T) * t + 4 * i + 16;
}

template <int GC, int GR, class T>
__global__ void __launch_bounds__(kResidentThreads, 1) k_resident(ResidentArgs<T> a) {
  using R = Rn<T>;
  extern __shared__ __align__(16) unsigned char smem[];
  const int c0 = a.cb[blockIdx.x], c1 = a.cb[blockIdx.x + 1];
  const int r0 = a.rb[blockIdx.x], r1 = a.rb[blockIdx.x + 1];
  const int nc = c1 - c0, nr = r1 - r0;
  const int tb = a.t_ptr[c0], tn = a.t_ptr[c1] - tb;
  const int ab = a.a_ptr[r0], an = a.a_ptr[r1] - ab;
  double* s_red = reinterpret_cast<double*>(smem);
  T* s_tval = reinterpret_cast<T*>(s_red + kNumSums * 32);
  T* s_aval = s_tval + tn;
  T* s_x = s_aval + an;
  T* s_x0 = s_x + nc;
  T* s_c = s_x0 + nc;
  T* s_lo = s_c + nc;
  T* s_up = s_lo + nc;
  T* s_xp = s_up + nc;
  T* s_y = s_xp + nc;
  T* s_y0 = s_y + nr;
  T* s_ax = s_y0 + nr;
  T* s_ax0 = s_ax + nr;
  T* s_rl = s_ax0 + nr;
  T* s_ru = s_rl + nr;
  T* s_axp = s_ru + nr;
  T* s_yp = s_axp + nr;
  int32_t* s_tidx = reinterpret_cast<int32_t*>(s_yp + nr);
  int32_t* s_aidx = s_tidx + tn;
  int32_t* s_tptr = s_aidx + an;
  int32_t* s_aptr = s_tptr + nc + 1;
  int32_t* s_tlong = s_aptr + nr + 1;
  int32_t* s_along = s_tlong + nc;
  int32_t* s_counts = s_along + nr;

  // ---- load the block's slices and owned state ----
  for (int q = threadIdx.x; q < tn; q += blockDim.x) {
    s_tval[q] = __ldg(a.t_val + tb + q);
    s_tidx[q] = __ldg(a.t_idx + tb + q);
  }
  for (int q = threadIdx.x; q < an; q += blockDim.x) {
    s_aval[q] = __ldg(a.a_val + ab + q);
    s_aidx[q] = __ldg(a.a_idx + ab + q);
  }
  for (int q = threadIdx.x; q <= nc; q += blockDim.x) s_tptr[q] = a.t_ptr[c0 + q] - tb;
  for (int q = threadIdx.x; q <= nr; q += blockDim.x) s_aptr[q] = a.a_ptr[r0 + q] - ab;
  for (int q = threadIdx.x; q < nc; q += blockDim.x) {
    const int j = c0 + q;
    s_x[q] = __ldcg(a.x + j);
    s_x0[q] = __ldcg(a.x0 + j);
    s_c[q] = __ldg(a.c + j);
    s_lo[q] = __ldg(a.lo + j);
    s_up[q] = __ldg(a.up + j);
  }
  for (int q = threadIdx.x; q < nr; q += blockDim.x) {
    const int i = r0 + q;
    s_y[q] = __ldcg(a.y + i);
    s_y0[q] = __ldcg(a.y0 + i);
    s_ax[q] = __ldcg(a.ax + i);
    s_ax0[q] = __ldcg(a.ax0 + i);
    s_rl[q] = __ldg(a.rl + i);
    s_ru[q] = __ldg(a.ru + i);
  }
  const T tau = static_cast<T>(__ldcg(a.tau)), sigma = static_cast<T>(__ldcg(a.sigma));
  const T rho = static_cast<T>(a.rho);
  const int64_t it0 = *a.it_base - a.ck.restart_at[0];
  __syncthreads();
  const int ntlong = res_long_list(s_tptr, nc, a.lt_cols, s_tlong, s_counts);
  const int nalong = res_long_list(s_aptr, nr, a.lt_rows, s_along, s_counts + 1);

  unsigned epoch = 0;
  bool ok = true;
  T lam = T(0);
  for (int l = 0; l < a.L && ok; ++l) {
    const bool last = l == a.L - 1;
    const double jj = static_cast<double>(it0 + l);
    lam = static_cast<T>(__ddiv_rn(__dadd_rn(jj, 1.0), __dadd_rn(jj, 2.0)));
    // primal phase: x+ = proj(x - tau (c - A^T y)); publish x+; Halpern x
    res_rows<GC>(s_tptr, s_tidx, s_tval, nc, a.lt_cols, s_tlong, ntlong, a.y, [&](int q, double atyd) {
      const T aty = static_cast<T>(atyd);
      const T xv = s_x[q];
      T v = R::sub(xv, R::mul(tau, R::sub(s_c[q], aty)));
      v = (v < s_lo[q]) ? s_lo[q] : v;
      v = (s_up[q] < v) ? s_up[q] : v;
      s_xp[q] = v;
      a.xp[c0 + q] = v;
      if (!last) s_x[q] = halpern_t(xv, v, s_x0[q], lam, rho);
    });
    ok = grid_barrier(a, epoch);
    if (!ok) break;
    // dual phase: y+ = v + sigma proj(-v/sigma); Halpern y, Ax; publish y (y+ at the check)
    res_rows<GR>(s_aptr, s_aidx, s_aval, nr, a.lt_rows, s_along, nalong, a.xp, [&](int q, double axpd) {
      const T axpv = static_cast<T>(axpd);
      const T axv = s_ax[q], yv = s_y[q];
      const T v = R::sub(yv, R::mul(sigma, R::sub(R::mul(T(2), axpv), axv)));
      T w = R::div(-v, sigma);
      w = (w < s_rl[q]) ? s_rl[q] : w;
      w = (s_ru[q] < w) ? s_ru[q] : w;
      const T ypv = R::add(v, R::mul(sigma, w));
      s_axp[q] = axpv;
      s_yp[q] = ypv;
      if (!last) {
        const T yn = halpern_t(yv, ypv, s_y0[q], lam, rho);
        s_y[q] = yn;
        a.y[r0 + q] = yn;
        s_ax[q] = halpern_t(axv, axpv, s_ax0[q], lam, rho);
      } else {
        a.yp[r0 + q] = ypv;
      }
    });
    ok = grid_barrier(a, epoch);
  }

  // ---- check: the block's part of kkt_rows/kkt_cols and the movement norms, in FP64 ----
  double v[kNumSums];
#pragma unroll
  for (int q = 0; q < kNumSums; ++q) v[q] = 0.0;
  if (ok) {
    res_rows<GC>(s_tptr, s_tidx, s_tval, nc, a.lt_cols, s_tlong, ntlong, a.yp, [&](int q, double atyp) {
      const int j = c0 + q;
      const double cv = a.c64[j], l = a.lo64[j], u = a.up64[j], xpv = static_cast<double>(s_xp[q]);
      const double d = cv - atyp;
      const bool hl = l > -1e300, hu = u < 1e300;
      double res = 0.0;
      if (!hl && !hu)
        res = fabs(d);
      else if (!hl)
        res = (d < 0.0) ? 0.0 : d;
      else if (!hu)
        res = (-d < 0.0) ? 0.0 : -d;
      res *= a.cfac[j];
      v[CS_COL_RES2] += res * res;
      v[CS_POBJ] += cv * xpv;
      if (d > 0.0 && hl)
        v[CS_COL_DOBJ] += d * l;
      else if (d < 0.0 && hu)
        v[CS_COL_DOBJ] += d * u;
      const double d1 = static_cast<double>(s_x[q]) - xpv, d2 = xpv - static_cast<double>(s_x0[q]);
      v[CS_DX2] += d1 * d1;
      v[CS_AX2] += d2 * d2;
    });
    for (int q = threadIdx.x; q < nr; q += blockDim.x) {
      const int i = r0 + q;
      const double av = static_cast<double>(s_axp[q]), l = a.rl64[i], u = a.ru64[i];
      double e1 = l - av, e2 = av - u;
      e1 = (e1 < 0.0) ? 0.0 : e1;
      e2 = (e2 < 0.0) ? 0.0 : e2;
      const double res = (e1 + e2) * a.rfac[i];
      v[CS_ROW_RES2] += res * res;
      const double yv = static_cast<double>(s_yp[q]);
      if (yv > 0.0 && l > -1e300)
        v[CS_ROW_DOBJ] += yv * l;
      else if (yv < 0.0 && u < 1e300)
        v[CS_ROW_DOBJ] += yv * u;
      v[CS_Y2] += yv * yv;
      const double d1 = static_cast<double>(s_y[q]) - yv, d2 = yv - static_cast<double>(s_y0[q]);
      v[CS_DY2] += d1 * d1;
      v[CS_AY2] += d2 * d2;
    }
  }
  res_block_sum<kNumSums>(v, s_red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < kNumSums; ++q) a.partial[blockIdx.x * kNumSums + q] = v[q];

  // ---- deferred Halpern step and write-back of the block's state ----
  if (ok) {
    for (int q = threadIdx.x; q < nc; q += blockDim.x) a.x[c0 + q] = halpern_t(s_x[q], s_xp[q], s_x0[q], lam, rho);
    for (int q = threadIdx.x; q < nr; q += blockDim.x) {
      const int i = r0 + q;
      a.y[i] = halpern_t(s_y[q], s_yp[q], s_y0[q], lam, rho);
      a.ax[i] = halpern_t(s_ax[q], s_axp[q], s_ax0[q], lam, rho);
      a.axp[i] = s_axp[q];
    }
  }
  ok = grid_barrier(a, epoch) && ok;
  if (blockIdx.x == 0) {
    // fixed-order sum of the block partials
    double t[kNumSums];
#pragma unroll
    for (int q = 0; q < kNumSums; ++q) t[q] = 0.0;
    for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x)
#pragma unroll
      for (int q = 0; q < kNumSums; ++q) t[q] += __ldcg(a.partial + b * kNumSums + q);
    res_block_sum<kNumSums>(t, s_red);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < kNumSums; ++q) a.sums[q] = t[q];
      *a.it_base += a.L;
    }
  }
}

}  // namespace b2p
