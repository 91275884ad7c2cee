// The CTA form of the multi-LP engine: one thread block runs one LP's whole
// restarted reflected-Halpern PDHG loop (src/pdhg/pdhg.cpp:560-687) inside a
// single launch -- iterations, the check every `check_every` iterations, the
// termination test, the restart rule and the primal-weight update -- with no
// host round trip.  One block per LP, launched together; the hardware starts
// a waiting LP's block as soon as a finished one leaves its SM, so LPs of
// uneven size and uneven iteration counts share the GPU without padding.
//
// Storage, chosen per LP by the host (CtaLp::tier):
//   kCtaAll     : iterates, anchors, costs, bounds, scaling factors and both
//                 operators (CSR of A and A^T) in shared memory;
//   kCtaVectors : the nine iterate / anchor vectors in shared memory, the
//                 operators and constants read from global memory (L1/L2);
//   kCtaVectorsPtr : as kCtaVectors, plus both operators' row pointers in
//                 shared memory (one L2 round trip less at the head of every
//                 row sum's chain of dependent loads);
//   kCtaGlobal  : everything in global memory (the engine's state arrays).
// The iteration is the engine's arithmetic element by element: every row sum
// runs left to right with separately rounded products and sums (the
// reference's CpuBackend::mult order, pdhg.cpp:93-103), the primal, dual and
// Halpern updates are those of k_primal / k_dual / halpern_step, and the
// Halpern step of a check iteration is applied after the check has read the
// pre-Halpern point.  The check's ten sums are block reductions in a fixed
// order; one thread then takes the host's decisions (the same FP64 formulas;
// the primal weight's exp / log are the device's) on those sums and publishes
// them, with the decision state, in shared memory, so control flow stays
// uniform across the block.  Two variants share this loop: run_lp (any LP
// size, three storage tiers) and run_owner (max(m, n) <= R * threads: each
// thread keeps its own rows' and columns' state in registers).
//
// Mixed precision (run_lp with T = float): the operator values and the nine
// iterate / anchor vectors are FP32 -- half the shared memory, so larger LPs
// keep their iterates on chip -- while every row sum accumulates the exact
// FP32 x FP32 products in FP64, the updates are evaluated in FP64 from the
// FP32 operands and rounded once at the store, and the check sums, costs,
// bounds, scaling factors and every decision stay FP64.  The FP32 run of an LP
// ends when its FP32 point meets the tolerance, or when its KKT error has not
// fallen by 10% in `stall_checks` checks; the host then restarts it in FP64
// from that point (entry_check: the point is measured in FP64 first, and an LP
// it already satisfies stops there).
#pragma once

#include <cstdint>

#include "../../include/b2p_pdhg.h"
#include "pdhg_kernels.cuh"

namespace b2p {

enum CtaTier : int32_t { kCtaAll = 0, kCtaVectors = 1, kCtaGlobal = 2, kCtaVectorsPtr = 3 };

// Per LP: where it sits in the concatenated operators and vectors, and the
// scalars its decisions need (src/pdhg/pdhg.cpp:506-545).
struct CtaLp {
  int32_t roff, coff;  // first global row / column
  int32_t m, n;
  int32_t a_beg, t_beg;  // first entry of its rows in A / in A^T
  int32_t nnz;
  int32_t tier;    // storage tier of the FP64 run
  int32_t tier32;  // storage tier of the FP32 run (mixed precision)
  // Where the LP's operators sit: its first row pointer in A / in A^T and
  // the offset its column / row indices carry.  Its own block of the
  // concatenated operators (roff, coff, coff, roff), or -- for members of a
  // family that share one A -- the first LP's block (0, 0, 0, 0), which every
  // block then reads from L2.
  int32_t aptr_off, tptr_off, ashift, tshift;
  int32_t pad;
  int64_t it0;     // iteration the run starts at (> 0: continuing an earlier run)
  double eta;        // 0.998 / ||A||
  double omega0;     // initial primal weight
  double cnorm;      // ||c|| of the original LP
  double rhsnorm;    // ||finite row bounds|| of the original LP
  double scale_obj;  // beta * gamma
};

// Status of an FP32 run that stalled (host-internal; never returned).
constexpr int32_t kCtaStalled = 100;

// Per LP result, written by the block when its loop ends.
struct CtaOut {
  int32_t status;  // B2P_STATUS_*
  int32_t restarts;
  int64_t iterations;
  double rel_kkt, pobj, dobj, omega;
};

struct CtaArgs {
  const CtaLp* __restrict__ lps;
  const int32_t* __restrict__ order;  // block b runs LP order[b]
  CtaOut* __restrict__ out;
  CsrView A, AT;  // concatenated operators (global row / column indices)
  const double *c, *lo, *up, *rl, *ru, *rfac, *cfac;
  const double *xinit, *yinit, *axinit;
  // global state (kCtaGlobal LPs iterate here); x+ and y+ of every LP are
  // left in xp and yp when its loop ends
  double *x, *xp, *x0, *y, *yp, *y0, *ax, *axp, *ax0;
  // FP32 run: the operators' values and the global-tier state in FP32 (its
  // x+ and y+ still go to xp and yp above, converted)
  const float *A32, *AT32;
  float *x32, *xp32, *x032, *y32, *yp32, *y032, *ax32, *axp32, *ax032;
  // sliced-ELL copies of the operators (NULL sbase: none): the entries of
  // rows 32 s .. 32 s + 31 of an LP interleaved, entry q of the row at
  // sbase[row] + 32 q (sbase indexed like the row pointers; the row's length
  // from them), so that the 32 lanes of a warp -- 32 consecutive rows -- load
  // one entry each from consecutive addresses
  const int32_t *sa_base, *sa_idx, *st_base, *st_idx;
  const double *sa_val, *st_val;
  const float *sa_val32, *st_val32;
  double tol, rho;
  int64_t max_it;
  int32_t check_every;
  int32_t entry_check;   // measure the starting point first; stop there if it meets tol
  int32_t stall_checks;  // > 0: end the run after this many checks without a 10% KKT gain
  int32_t pad;
  const volatile int32_t* stop;  // host-mapped; nonzero = stop at the next check
};

template <class T>
struct CtaState {
  T *x, *xp, *x0, *y, *yp, *y0, *ax, *axp, *ax0;
  const T *Av, *Tv;
  const T *SAv, *STv;  // sliced-ELL values
};
__device__ __forceinline__ CtaState<double> cta_state(const CtaArgs& a, double*) {
  return CtaState<double>{a.x,  a.xp,  a.x0,    a.y,      a.yp,     a.y0,    a.ax,
                          a.axp, a.ax0, a.A.val, a.AT.val, a.sa_val, a.st_val};
}
__device__ __forceinline__ CtaState<float> cta_state(const CtaArgs& a, float*) {
  return CtaState<float>{a.x32, a.xp32, a.x032, a.y32, a.yp32, a.y032, a.ax32,
                         a.axp32, a.ax032, a.A32, a.AT32, a.sa_val32, a.st_val32};
}

// Iterate / anchor vector elements of an LP in shared memory, rounded up so
// that the FP64 constants after them start on an 8-byte boundary.
__host__ __device__ inline int64_t cta_vector_elems(int64_t m, int64_t n, int esize) {
  const int64_t e = 3 * n + 6 * m;
  return esize == 4 ? (e + 1) / 2 * 2 : e;
}

// Shared-memory bytes an LP needs in each tier of run_lp with esize-byte
// iterates and operator values (vectors, FP64 constants, values, int32).
__host__ __device__ inline int64_t cta_tier_bytes(int tier, int64_t m, int64_t n, int64_t nnz, int esize = 8) {
  if (tier == kCtaGlobal) return 0;
  const int64_t vec = esize * cta_vector_elems(m, n, esize);
  if (tier == kCtaVectors) return vec;
  if (tier == kCtaVectorsPtr) return vec + (4 * ((m + 1) + (n + 1)) + 7) / 8 * 8;
  const int64_t vals = (esize * 2 * nnz + 7) / 8 * 8;
  return vec + 8 * (4 * n + 3 * m) + vals + 4 * ((m + 1) + (n + 1) + 2 * nnz);
}

// Shared-memory bytes of an LP in run_owner: x+, y, y+ and both operators'
// values and indices.
__host__ __device__ inline int64_t cta_owner_bytes(int64_t m, int64_t n, int64_t nnz) {
  return 8 * (n + 2 * m) + 8 * 2 * nnz + 4 * 2 * nnz;
}

namespace cta {

// Decision state of the block's LP (the host loop's per-instance variables,
// src/pdhg/pdhg.cpp:560-662), kept in shared memory and written by one thread.
struct Ctl {
  double omega, tau, sigma, fp_restart, fp_prev;
  double rel_p, rel_d, gap, pobj, dobj;
  int64_t since_restart, restart_at;
  int32_t restarts;
  int32_t status;   // 0 while running, else B2P_STATUS_* (or kCtaStalled)
  int32_t restart;  // restart at this check
  int32_t stop;     // the stop flag as read at this check
  double best_kkt;  // FP32 run: smallest KKT error a 10% gain last reached
  int32_t since_best;
  int32_t pad;
};

template <int NT>
struct Shared {
  double w[kNumSums][NT / 32];
  double tot[kNumSums];
  Ctl ctl;
};

__device__ __forceinline__ void init_ctl(Ctl& c, const CtaLp& L) {
  c.omega = L.omega0;
  c.tau = L.eta / L.omega0;
  c.sigma = L.eta * L.omega0;
  c.fp_restart = INFINITY;
  c.fp_prev = INFINITY;
  c.rel_p = c.rel_d = c.gap = c.pobj = c.dobj = 0.0;
  c.since_restart = 0;
  c.restart_at = 0;
  c.restarts = 0;
  c.status = 0;
  c.restart = 0;
  c.stop = 0;
  c.best_kkt = INFINITY;
  c.since_best = 0;
}

// The host's decisions at a check from the ten sums (src/pdhg/pdhg.cpp:598-662):
// termination, the restart rule, the primal-weight update and new step sizes.
// `it` is the index of the check iteration.  Out of line: the exp / log live
// here, not in the iteration loop's registers.
__device__ __noinline__ void decide(Ctl& c, const double* tot, double scale_obj, double rhsnorm, double cnorm,
                                    double eta, int64_t it, double tol, int cE, int stall_checks) {
  const double pobj = tot[CS_POBJ] * scale_obj;
  const double dobj = (tot[CS_ROW_DOBJ] + tot[CS_COL_DOBJ]) * scale_obj;
  const double relP = sqrt(tot[CS_ROW_RES2]) / (1.0 + rhsnorm);
  const double relD = sqrt(tot[CS_COL_RES2]) / (1.0 + cnorm);
  const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
  c.pobj = pobj;
  c.dobj = dobj;
  c.rel_p = relP;
  c.rel_d = relD;
  c.gap = gap;
  c.restart = 0;
  if (relP <= tol && relD <= tol && gap <= tol) {
    c.status = B2P_STATUS_OPTIMAL;
    return;
  }
  if (stall_checks > 0) {
    const double kkt = fmax(relP, fmax(relD, gap));
    if (kkt < 0.9 * c.best_kkt) {
      c.best_kkt = kkt;
      c.since_best = 0;
    } else if (++c.since_best >= stall_checks) {
      c.status = kCtaStalled;
      return;
    }
  }
  c.since_restart += cE;
  double omega = c.omega;
  const double fp = sqrt(omega * tot[CS_DX2] + tot[CS_DY2] / omega);
  if (c.fp_restart == INFINITY) c.fp_restart = fp;
  const bool restart = fp <= 0.2 * c.fp_restart || (fp <= 0.8 * c.fp_restart && fp > c.fp_prev) ||
                       c.since_restart >= static_cast<int64_t>(0.36 * static_cast<double>(it + 1));
  c.fp_prev = fp;
  if (restart) {
    const double dxn = sqrt(tot[CS_AX2]), dyn = sqrt(tot[CS_AY2]);
    if (dxn > 1e-10 && dyn > 1e-10) omega = exp(0.5 * log(dyn / dxn) + 0.5 * log(omega));
    c.omega = omega;
    c.fp_restart = sqrt(omega * tot[CS_DX2] + tot[CS_DY2] / omega);
    c.fp_prev = INFINITY;
    c.since_restart = 0;
    ++c.restarts;
  }
  if (c.stop) {
    c.status = B2P_STATUS_TIME_LIMIT;
    return;
  }
  if (restart) {
    c.restart = 1;
    c.tau = eta / omega;
    c.sigma = eta * omega;
    c.restart_at = it + 1;
  }
}

// Block sums of s in a fixed order, then the decisions; on return every
// thread sees sh.ctl of this check.  `it` = index of the check iteration.
template <int NT>
__device__ __forceinline__ void check_decide(double (&s)[kNumSums], Shared<NT>& sh, const CtaArgs& a,
                                             const CtaLp& L, int64_t it) {
#pragma unroll
  for (int q = 0; q < kNumSums; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < kNumSums; ++q) sh.w[q][warp] = s[q];
  if (threadIdx.x == 0) sh.ctl.stop = a.stop ? *a.stop : 0;
  __syncthreads();
  if (warp == 0) {
    if (lane < kNumSums) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < NT / 32; ++w) t += sh.w[lane][w];
      sh.tot[lane] = t;
    }
    __syncwarp();
    if (lane == 0)
      decide(sh.ctl, sh.tot, L.scale_obj, L.rhsnorm, L.cnorm, L.eta, it, a.tol, a.check_every, a.stall_checks);
  }
  __syncthreads();
}

// The termination test alone, on sums of the starting point (entry check):
// on return every thread sees sh.ctl.status.
template <int NT>
__device__ __forceinline__ void entry_decide(double (&s)[kNumSums], Shared<NT>& sh, const CtaArgs& a,
                                             const CtaLp& L) {
#pragma unroll
  for (int q = 0; q < kNumSums; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < kNumSums; ++q) sh.w[q][warp] = s[q];
  __syncthreads();
  if (warp == 0) {
    if (lane < kNumSums) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < NT / 32; ++w) t += sh.w[lane][w];
      sh.tot[lane] = t;
    }
    __syncwarp();
    if (lane == 0) {
      Ctl& c = sh.ctl;
      const double* tot = sh.tot;
      c.pobj = tot[CS_POBJ] * L.scale_obj;
      c.dobj = (tot[CS_ROW_DOBJ] + tot[CS_COL_DOBJ]) * L.scale_obj;
      c.rel_p = sqrt(tot[CS_ROW_RES2]) / (1.0 + L.rhsnorm);
      c.rel_d = sqrt(tot[CS_COL_RES2]) / (1.0 + L.cnorm);
      c.gap = fabs(c.pobj - c.dobj) / (1.0 + fabs(c.pobj) + fabs(c.dobj));
      if (c.rel_p <= a.tol && c.rel_d <= a.tol && c.gap <= a.tol) c.status = B2P_STATUS_OPTIMAL;
    }
  }
  __syncthreads();
}

template <int NT>
__device__ __forceinline__ void write_out(const CtaArgs& a, const Ctl& c, int lp, int64_t it) {
  if (threadIdx.x != 0) return;
  CtaOut o;
  o.status = c.status ? c.status : B2P_STATUS_ITERATION_LIMIT;
  o.restarts = c.restarts;
  o.iterations = it;
  const double mx = (c.rel_d < c.gap) ? c.gap : c.rel_d;
  o.rel_kkt = (c.rel_p < mx) ? mx : c.rel_p;
  o.pobj = c.pobj;
  o.dobj = c.dobj;
  o.omega = c.omega;
  a.out[lp] = o;
}

template <class T, class S>
__device__ __forceinline__ void copy_in(T* __restrict__ dst, const S* __restrict__ src, int64_t len) {
  for (int64_t t = threadIdx.x; t < len; t += blockDim.x) dst[t] = static_cast<T>(src[t]);
}

// Left-to-right row sum over entries [p, e) of (idx, val) against the local
// vector v (index minus `shift`): s = ((0 + a0 v0) + a1 v1) + ...  (A version
// that issued the loads of 4 or 8 entries before their additions measured
// slower: the block is bound by shared-memory wavefronts -- scattered row
// starts and gathers -- not by load latency.)
template <class T>
__device__ __forceinline__ double row_sum(int p, const int e, const int32_t* __restrict__ idx,
                                          const T* __restrict__ val, const T* __restrict__ v, int shift) {
  double s = 0.0;
#pragma unroll 4
  for (; p < e; ++p)
    s = __dadd_rn(s, __dmul_rn(static_cast<double>(val[p]), static_cast<double>(v[idx[p] - shift])));
  return s;
}

// The same left-to-right sum over a row of length len stored sliced-ELL from
// position b (entry q at b + 32 q).
template <class T>
__device__ __forceinline__ double row_sum_sliced(int b, const int len, const int32_t* __restrict__ idx,
                                                 const T* __restrict__ val, const T* __restrict__ v, int shift) {
  double s = 0.0;
#pragma unroll 4
  for (int q = 0; q < len; ++q, b += 32)
    s = __dadd_rn(s, __dmul_rn(static_cast<double>(val[b]), static_cast<double>(v[idx[b] - shift])));
  return s;
}

// Row sums of one operator of an LP: its CSR (row pointers local to the LP,
// in shared memory or global), or, when sbase is set, its sliced-ELL copy.
template <class T>
struct RowOp {
  const int32_t* ptr;
  const int32_t* idx;
  const T* val;
  const int32_t* sbase;  // NULL: CSR
  const int32_t* sidx;
  const T* sval;
  int shift;
  __device__ __forceinline__ double sum(int r, const T* __restrict__ v) const {
    const int p = ptr[r], e = ptr[r + 1];
    if (sbase) return row_sum_sliced(sbase[r], e - p, sidx, sval, v, shift);
    return row_sum(p, e, idx, val, v, shift);
  }
};

__device__ __forceinline__ double lambda_at(int64_t j) {
  const double jj = static_cast<double>(j);
  return __ddiv_rn(__dadd_rn(jj, 1.0), __dadd_rn(jj, 2.0));
}

// Row part of the check sums for one row (k_check_rows).
__device__ __forceinline__ void row_check(double (&s)[kNumSums], double av, double li, double ui, double rf,
                                          double yv, double yc, double y0v) {
  double e1 = li - av, e2 = av - ui;
  e1 = (e1 < 0.0) ? 0.0 : e1;
  e2 = (e2 < 0.0) ? 0.0 : e2;
  const double res = (e1 + e2) * rf;
  s[CS_ROW_RES2] += res * res;
  if (yv > 0.0 && li > -1e300)
    s[CS_ROW_DOBJ] += yv * li;
  else if (yv < 0.0 && ui < 1e300)
    s[CS_ROW_DOBJ] += yv * ui;
  s[CS_Y2] += yv * yv;
  const double d1 = yc - yv, d2 = yv - y0v;
  s[CS_DY2] += d1 * d1;
  s[CS_AY2] += d2 * d2;
}

// Column part for one column (k_check_cols), given A^T y+ of the column.
__device__ __forceinline__ void col_check(double (&s)[kNumSums], double atyp, double cv, double lj, double uj,
                                          double cf, double xpv, double xc, double x0v) {
  const double d = cv - atyp;
  const bool hl = lj > -1e300, hu = uj < 1e300;
  double res = 0.0;
  if (!hl && !hu)
    res = fabs(d);
  else if (!hl)
    res = (d < 0.0) ? 0.0 : d;
  else if (!hu)
    res = (-d < 0.0) ? 0.0 : -d;
  res *= cf;
  s[CS_COL_RES2] += res * res;
  s[CS_POBJ] += cv * xpv;
  if (d > 0.0 && hl)
    s[CS_COL_DOBJ] += d * lj;
  else if (d < 0.0 && hu)
    s[CS_COL_DOBJ] += d * uj;
  const double d1 = xc - xpv, d2 = xpv - x0v;
  s[CS_DX2] += d1 * d1;
  s[CS_AX2] += d2 * d2;
}

template <int NT, int TIER, class T>
__device__ __forceinline__ void run_lp(const CtaArgs& a, const CtaLp& L, int lp, unsigned char* smem,
                                       Shared<NT>& sh) {
  const int m = L.m, n = L.n, tid = threadIdx.x;
  const CtaState<T> g = cta_state(a, static_cast<T*>(nullptr));
  T *x, *xp, *x0, *y, *yp, *y0, *ax, *axp, *ax0;
  const double *c, *lo, *up, *cfac, *rl, *ru, *rfac;
  const int32_t *Ap, *Ai, *Tp, *Ti;
  const T *Av, *Tv;
  if (TIER == kCtaGlobal) {
    x = g.x + L.coff, xp = g.xp + L.coff, x0 = g.x0 + L.coff;
    y = g.y + L.roff, yp = g.yp + L.roff, y0 = g.y0 + L.roff;
    ax = g.ax + L.roff, axp = g.axp + L.roff, ax0 = g.ax0 + L.roff;
  } else {
    T* d = reinterpret_cast<T*>(smem);
    x = d, xp = x + n, x0 = xp + n;
    y = x0 + n, yp = y + m, y0 = yp + m, ax = y0 + m, axp = ax + m, ax0 = axp + m;
  }
  if (TIER == kCtaAll) {
    double* d = reinterpret_cast<double*>(smem + sizeof(T) * cta_vector_elems(m, n, sizeof(T)));
    double *sc = d, *slo = sc + n, *sup = slo + n, *scf = sup + n, *srl = scf + n, *sru = srl + m, *srf = sru + m;
    T *sAv = reinterpret_cast<T*>(srf + m), *sTv = sAv + L.nnz;
    int32_t* sAp = reinterpret_cast<int32_t*>(smem + sizeof(T) * cta_vector_elems(m, n, sizeof(T)) +
                                              8 * (4 * static_cast<int64_t>(n) + 3 * m) +
                                              (sizeof(T) * 2 * static_cast<int64_t>(L.nnz) + 7) / 8 * 8);
    int32_t *sAi = sAp + (m + 1), *sTp = sAi + L.nnz, *sTi = sTp + (n + 1);
    copy_in(sc, a.c + L.coff, n);
    copy_in(slo, a.lo + L.coff, n);
    copy_in(sup, a.up + L.coff, n);
    copy_in(scf, a.cfac + L.coff, n);
    copy_in(srl, a.rl + L.roff, m);
    copy_in(sru, a.ru + L.roff, m);
    copy_in(srf, a.rfac + L.roff, m);
    copy_in(sAv, g.Av + L.a_beg, L.nnz);
    copy_in(sTv, g.Tv + L.t_beg, L.nnz);
    copy_in(sAi, a.A.idx + L.a_beg, L.nnz);
    copy_in(sTi, a.AT.idx + L.t_beg, L.nnz);
    for (int t = tid; t <= m; t += NT) sAp[t] = a.A.ptr[L.aptr_off + t] - L.a_beg;
    for (int t = tid; t <= n; t += NT) sTp[t] = a.AT.ptr[L.tptr_off + t] - L.t_beg;
    c = sc, lo = slo, up = sup, cfac = scf, rl = srl, ru = sru, rfac = srf;
    Ap = sAp, Ai = sAi, Av = sAv, Tp = sTp, Ti = sTi, Tv = sTv;
  } else {
    c = a.c + L.coff, lo = a.lo + L.coff, up = a.up + L.coff, cfac = a.cfac + L.coff;
    rl = a.rl + L.roff, ru = a.ru + L.roff, rfac = a.rfac + L.roff;
    Ap = a.A.ptr + L.aptr_off, Ai = a.A.idx, Av = g.Av;
    Tp = a.AT.ptr + L.tptr_off, Ti = a.AT.idx, Tv = g.Tv;
    if (TIER == kCtaVectorsPtr) {
      int32_t* sp = reinterpret_cast<int32_t*>(smem + sizeof(T) * cta_vector_elems(m, n, sizeof(T)));
      copy_in(sp, Ap, m + 1);
      copy_in(sp + m + 1, Tp, n + 1);
      Ap = sp, Tp = sp + m + 1;
    }
  }
  // the operators' row sums: sliced-ELL where the engine built that copy and
  // the LP reads its operators from global memory but gathers from shared
  // memory (the vectors tiers: operator loads, scattered per lane in CSR,
  // are what the block waits on there; with the vectors in global memory
  // too, the CSR arrays' fewer bytes measured faster)
  const bool sliced = (TIER == kCtaVectors || TIER == kCtaVectorsPtr) && a.sa_base != nullptr;
  const RowOp<T> opA{Ap, Ai, Av, sliced ? a.sa_base + L.aptr_off : nullptr, a.sa_idx, g.SAv, L.ashift};
  const RowOp<T> opT{Tp, Ti, Tv, sliced ? a.st_base + L.tptr_off : nullptr, a.st_idx, g.STv, L.tshift};
  // starting point (x0 = x = x_init, y0 = y = y_init, A x0)
  for (int j = tid; j < n; j += NT) x[j] = x0[j] = static_cast<T>(a.xinit[L.coff + j]);
  for (int i = tid; i < m; i += NT) {
    y[i] = y0[i] = static_cast<T>(a.yinit[L.roff + i]);
    ax[i] = ax0[i] = static_cast<T>(a.axinit[L.roff + i]);
  }
  if (tid == 0) init_ctl(sh.ctl, L);
  __syncthreads();

  const double rho = a.rho;
  const int cE = a.check_every;
  double tau = sh.ctl.tau, sigma = sh.ctl.sigma;
  int64_t restartAt = L.it0, it = L.it0;
  if (a.entry_check) {
    // the starting point measured as it is (x+ = x, y+ = y, A x+ = A x)
    double s[kNumSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = tid; i < m; i += NT) {
      const double yv = static_cast<double>(y[i]);
      row_check(s, static_cast<double>(ax[i]), rl[i], ru[i], rfac[i], yv, yv, yv);
      axp[i] = ax[i];
      yp[i] = y[i];
    }
    for (int j = tid; j < n; j += NT) {
      const double xv = static_cast<double>(x[j]);
      col_check(s, opT.sum(j, y), c[j], lo[j], up[j], cfac[j], xv, xv, xv);
      xp[j] = x[j];
    }
    entry_decide<NT>(s, sh, a, L);
    if (sh.ctl.status) it = L.it0 - 1;  // reported as the check iteration that produced the point
  }
  while (!sh.ctl.status && it < a.max_it) {
    const int Lint = static_cast<int>((a.max_it - it) < cE ? (a.max_it - it) : cE);
    for (int l = 0; l < Lint; ++l) {
      const bool halpern = l != Lint - 1;
      const double lam = lambda_at(it + l - restartAt);
      // x+ = proj(x - tau (c - A^T y)), Halpern step of x
      for (int j = tid; j < n; j += NT) {
        const double aty = opT.sum(j, y);
        const double xv = static_cast<double>(x[j]);
        double v = __dsub_rn(xv, __dmul_rn(tau, __dsub_rn(c[j], aty)));
        const double lj = lo[j], uj = up[j];
        v = (v < lj) ? lj : v;
        v = (uj < v) ? uj : v;
        xp[j] = static_cast<T>(v);
        if (halpern) x[j] = static_cast<T>(halpern_step(xv, v, static_cast<double>(x0[j]), lam, rho));
      }
      __syncthreads();
      // A x+, y+ = v + sigma proj(-v / sigma), Halpern steps of y and A x
      for (int i = tid; i < m; i += NT) {
        const double axpv = opA.sum(i, xp);
        const double axv = static_cast<double>(ax[i]), yv = static_cast<double>(y[i]);
        const double v = __dsub_rn(yv, __dmul_rn(sigma, __dsub_rn(__dmul_rn(2.0, axpv), axv)));
        double w = __ddiv_rn(-v, sigma);
        const double li = rl[i], ui = ru[i];
        w = (w < li) ? li : w;
        w = (ui < w) ? ui : w;
        const double ypv = __dadd_rn(v, __dmul_rn(sigma, w));
        axp[i] = static_cast<T>(axpv);
        yp[i] = static_cast<T>(ypv);
        if (halpern) {
          y[i] = static_cast<T>(halpern_step(yv, ypv, static_cast<double>(y0[i]), lam, rho));
          ax[i] = static_cast<T>(halpern_step(axv, axpv, static_cast<double>(ax0[i]), lam, rho));
        }
      }
      __syncthreads();
    }
    // ---- check at iteration it + Lint - 1, then the deferred Halpern step of
    // that iteration on the same elements
    const double lam = lambda_at(it + Lint - 1 - restartAt);
    double s[kNumSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = tid; i < m; i += NT) {
      const double yc = static_cast<double>(y[i]), yv = static_cast<double>(yp[i]);
      const double y0v = static_cast<double>(y0[i]), axpv = static_cast<double>(axp[i]);
      row_check(s, axpv, rl[i], ru[i], rfac[i], yv, yc, y0v);
      y[i] = static_cast<T>(halpern_step(yc, yv, y0v, lam, rho));
      ax[i] = static_cast<T>(halpern_step(static_cast<double>(ax[i]), axpv, static_cast<double>(ax0[i]), lam, rho));
    }
    for (int j = tid; j < n; j += NT) {
      const double atyp = opT.sum(j, yp);
      const double xc = static_cast<double>(x[j]), xpv = static_cast<double>(xp[j]), x0v = static_cast<double>(x0[j]);
      col_check(s, atyp, c[j], lo[j], up[j], cfac[j], xpv, xc, x0v);
      x[j] = static_cast<T>(halpern_step(xc, xpv, x0v, lam, rho));
    }
    it += Lint - 1;
    check_decide<NT>(s, sh, a, L, it);
    if (sh.ctl.status) break;
    if (sh.ctl.restart) {
      tau = sh.ctl.tau;
      sigma = sh.ctl.sigma;
      restartAt = sh.ctl.restart_at;
      for (int j = tid; j < n; j += NT) x[j] = x0[j] = xp[j];
      for (int i = tid; i < m; i += NT) {
        y[i] = y0[i] = yp[i];
        ax[i] = ax0[i] = axp[i];
      }
      __syncthreads();
    }
    ++it;
  }
  // results: x+ and y+ to the engine's FP64 arrays, the scalars to out[lp]
  if (TIER != kCtaGlobal || sizeof(T) != sizeof(double)) {
    for (int j = tid; j < n; j += NT) a.xp[L.coff + j] = static_cast<double>(xp[j]);
    for (int i = tid; i < m; i += NT) a.yp[L.roff + i] = static_cast<double>(yp[i]);
  }
  write_out<NT>(a, sh.ctl, lp, it);
}

// Owner variant: for LPs with max(m, n) <= R * NT and both operators in
// shared memory.  Thread t owns columns and rows t, t + NT, ...; the state
// only the owner touches -- x, x0, the costs and column bounds, y0, A x,
// A x0, the row bounds, x+ / y+ / A x+ of its elements and their entry
// ranges -- stays in registers; shared memory holds the operators and the
// vectors other threads gather (x+, y, and y+ at check iterations).
template <int NT, int R>
__device__ __forceinline__ void run_owner(const CtaArgs& a, const CtaLp& L, int lp, unsigned char* smem,
                                          Shared<NT>& sh) {
  const int m = L.m, n = L.n, tid = threadIdx.x;
  double* xp_s = reinterpret_cast<double*>(smem);
  double* y_s = xp_s + n;
  double* yp_s = y_s + m;
  double* Av = yp_s + m;
  double* Tv = Av + L.nnz;
  int32_t* Ai = reinterpret_cast<int32_t*>(Tv + L.nnz);
  int32_t* Ti = Ai + L.nnz;
  copy_in(Av, a.A.val + L.a_beg, L.nnz);
  copy_in(Tv, a.AT.val + L.t_beg, L.nnz);
  for (int t = tid; t < L.nnz; t += NT) {
    Ai[t] = a.A.idx[L.a_beg + t] - L.ashift;
    Ti[t] = a.AT.idx[L.t_beg + t] - L.tshift;
  }
  double x[R], x0[R], c[R], lo[R], up[R], xpr[R];
  double y[R], y0[R], ax[R], ax0[R], rl[R], ru[R], ypr[R], axpr[R];
  int tb[R], te[R], ab[R], ae[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int e = tid + r * NT;
    tb[r] = te[r] = ab[r] = ae[r] = 0;
    x[r] = x0[r] = c[r] = lo[r] = up[r] = xpr[r] = 0.0;
    y[r] = y0[r] = ax[r] = ax0[r] = rl[r] = ru[r] = ypr[r] = axpr[r] = 0.0;
    if (e < n) {
      tb[r] = a.AT.ptr[L.tptr_off + e] - L.t_beg;
      te[r] = a.AT.ptr[L.tptr_off + e + 1] - L.t_beg;
      x[r] = x0[r] = a.xinit[L.coff + e];
      c[r] = a.c[L.coff + e];
      lo[r] = a.lo[L.coff + e];
      up[r] = a.up[L.coff + e];
    }
    if (e < m) {
      ab[r] = a.A.ptr[L.aptr_off + e] - L.a_beg;
      ae[r] = a.A.ptr[L.aptr_off + e + 1] - L.a_beg;
      y[r] = y0[r] = a.yinit[L.roff + e];
      ax[r] = ax0[r] = a.axinit[L.roff + e];
      rl[r] = a.rl[L.roff + e];
      ru[r] = a.ru[L.roff + e];
      y_s[e] = y[r];
    }
  }
  if (tid == 0) init_ctl(sh.ctl, L);
  __syncthreads();

  const double rho = a.rho;
  const int cE = a.check_every;
  double tau = sh.ctl.tau, sigma = sh.ctl.sigma;
  int64_t restartAt = 0, it = 0;
  while (it < a.max_it) {
    const int Lint = static_cast<int>((a.max_it - it) < cE ? (a.max_it - it) : cE);
    for (int l = 0; l < Lint; ++l) {
      const bool halpern = l != Lint - 1;
      const double lam = lambda_at(it + l - restartAt);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = tid + r * NT;
        if (j < n) {
          const double aty = row_sum(tb[r], te[r], Ti, Tv, y_s, 0);
          double v = __dsub_rn(x[r], __dmul_rn(tau, __dsub_rn(c[r], aty)));
          v = (v < lo[r]) ? lo[r] : v;
          v = (up[r] < v) ? up[r] : v;
          xpr[r] = v;
          xp_s[j] = v;
          if (halpern) x[r] = halpern_step(x[r], v, x0[r], lam, rho);
        }
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = tid + r * NT;
        if (i < m) {
          const double axpv = row_sum(ab[r], ae[r], Ai, Av, xp_s, 0);
          const double v = __dsub_rn(y[r], __dmul_rn(sigma, __dsub_rn(__dmul_rn(2.0, axpv), ax[r])));
          double w = __ddiv_rn(-v, sigma);
          w = (w < rl[r]) ? rl[r] : w;
          w = (ru[r] < w) ? ru[r] : w;
          const double ypv = __dadd_rn(v, __dmul_rn(sigma, w));
          axpr[r] = axpv;
          ypr[r] = ypv;
          if (halpern) {
            y[r] = halpern_step(y[r], ypv, y0[r], lam, rho);
            ax[r] = halpern_step(ax[r], axpv, ax0[r], lam, rho);
            y_s[i] = y[r];
          } else {
            yp_s[i] = ypv;  // gathered by the check's A^T y+
          }
        }
      }
      __syncthreads();
    }
    // ---- check at iteration it + Lint - 1, then the deferred Halpern step
    const double lam = lambda_at(it + Lint - 1 - restartAt);
    double s[kNumSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = tid + r * NT;
      if (i < m) {
        row_check(s, axpr[r], rl[r], ru[r], a.rfac[L.roff + i], ypr[r], y[r], y0[r]);
        y[r] = halpern_step(y[r], ypr[r], y0[r], lam, rho);
        ax[r] = halpern_step(ax[r], axpr[r], ax0[r], lam, rho);
        y_s[i] = y[r];
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = tid + r * NT;
      if (j < n) {
        const double atyp = row_sum(tb[r], te[r], Ti, Tv, yp_s, 0);
        col_check(s, atyp, c[r], lo[r], up[r], a.cfac[L.coff + j], xpr[r], x[r], x0[r]);
        x[r] = halpern_step(x[r], xpr[r], x0[r], lam, rho);
      }
    }
    it += Lint - 1;
    check_decide<NT>(s, sh, a, L, it);
    if (sh.ctl.status) break;
    if (sh.ctl.restart) {
      tau = sh.ctl.tau;
      sigma = sh.ctl.sigma;
      restartAt = sh.ctl.restart_at;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int e = tid + r * NT;
        if (e < n) x[r] = x0[r] = xpr[r];
        if (e < m) {
          y[r] = y0[r] = ypr[r];
          ax[r] = ax0[r] = axpr[r];
          y_s[e] = y[r];
        }
      }
      __syncthreads();
    }
    ++it;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int e = tid + r * NT;
    if (e < n) a.xp[L.coff + e] = xpr[r];
    if (e < m) a.yp[L.roff + e] = ypr[r];
  }
  write_out<NT>(a, sh.ctl, lp, it);
}

}  // namespace cta

// T = double: the plain FP64 run; T = float: the FP32 run of the mixed form.
// MINB > 1: compiled so that MINB blocks fit one SM's registers (64 per
// thread at MINB x NT = 1,024): more warps to hide the latency of the
// operators' loads from L2, at the price of a few spilled registers; the
// autotuner decides.
template <int NT, class T = double, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) k_lp_cta(CtaArgs a) {
  extern __shared__ __align__(16) unsigned char cta_smem[];
  __shared__ cta::Shared<NT> sh;
  const int lp = a.order[blockIdx.x];
  const CtaLp L = a.lps[lp];
  const int tier = sizeof(T) == sizeof(double) ? L.tier : L.tier32;
  if (tier == kCtaAll)
    cta::run_lp<NT, kCtaAll, T>(a, L, lp, cta_smem, sh);
  else if (tier == kCtaVectorsPtr)
    cta::run_lp<NT, kCtaVectorsPtr, T>(a, L, lp, cta_smem, sh);
  else if (tier == kCtaVectors)
    cta::run_lp<NT, kCtaVectors, T>(a, L, lp, cta_smem, sh);
  else
    cta::run_lp<NT, kCtaGlobal, T>(a, L, lp, cta_smem, sh);
}

template <int NT, int R>
__global__ void __launch_bounds__(NT) k_lp_owner(CtaArgs a) {
  extern __shared__ __align__(16) unsigned char cta_smem[];
  __shared__ cta::Shared<NT> sh;
  const int lp = a.order[blockIdx.x];
  const CtaLp L = a.lps[lp];
  cta::run_owner<NT, R>(a, L, lp, cta_smem, sh);
}

}  // namespace b2p
