// Row-length-binned CSR row sums for one LP (k = 1), used by the fused
// iteration kernels.
//
// Rows are split by length on the host (RowBins):
//   short rows (len <= long_thr = kUnroll * G): a group of G lanes per row
//       (G = 1..32, a power of two chosen so that the grid fits in one wave),
//       32/G rows per warp, in the original row order;
//   long rows  (long_thr < len <= kVeryLongRow): one warp per row;
//   very long rows: one 256-thread block per row.
// Each lane accumulates the products of entries p = lane, lane+S, lane+2S, ...
// left to right; the lanes are then combined by a fixed xor-shuffle tree, so
// the sum is deterministic (it differs from the reference's strictly
// sequential row sum only in rounding order).
//
// STREAM (operators much larger than L2): every load that is used once per
// launch -- the operator's indices and values and the epilogue's vectors --
// is an evict-first streaming load (ld.global.cs), so that L2 keeps the one
// vector the rows gather from (written by the previous kernel).
//
// Latency hiding: a lane loads the column indices and values of its first
// kUnroll chunks before anything else (these are constant during a solve, so
// this happens before griddepcontrol.wait, while the previous kernel is still
// draining under programmatic dependent launch); after the wait the kernel
// issues its epilogue loads and all kUnroll gathers of x together, so a short
// row costs three dependent memory round trips (pointers, indices, x).
#pragma once

#include <cstdint>

#include "pdhg_kernels.cuh"

namespace b2p {

constexpr int kUnroll = 4;
constexpr int kVeryLongRow = 2048;  // rows longer than this get a 256-thread block

struct RowBins {
  const int32_t* __restrict__ long_rows;   // rows for the warp path
  const int32_t* __restrict__ vlong_rows;  // rows for the block path
  const int32_t* __restrict__ short_rows;  // rows for the short path (NULL: every row 0..rows-1)
  int32_t n_short;                         // entries of short_rows
  int32_t n_long, n_vlong;
  int32_t long_thr;      // rows longer than this are not in the short path
  int32_t vlong_blocks;  // == n_vlong
  int32_t long_blocks;   // ceil(n_long / warps per block)
  int32_t short_blocks;
  int32_t g;             // lanes per short row
};


// Several LPs solved together as one block-diagonal operator: inst[row] is
// the row's instance, done[instance] != 0 once that instance has terminated
// (its rows are then skipped).  Unused (null) for a single LP.
struct InstanceMap {
  const int32_t* __restrict__ inst;
  const int32_t* __restrict__ done;
};

// What one thread does for its row: entries beg+lane0, +stride, ... < end.
struct RowPlan {
  int32_t row;     // -1: no row
  int32_t p;       // first entry of this lane
  int32_t end;
  int32_t stride;
  int32_t path;    // 0 short, 1 warp, 2 block
  bool leader;     // runs the row's epilogue
  int32_t ci[kUnroll];
  double cv[kUnroll];
};

template <bool STREAM, class T>
__device__ __forceinline__ T ld_once(const T* p) {
  return STREAM ? __ldcs(p) : __ldg(p);
}

// Pre-wait part: row assignment and the first kUnroll (index, value) pairs.
template <int G, bool MULTI = false, bool STREAM = false>
__device__ __forceinline__ RowPlan plan_row(const CsrView& M, const RowBins& bins, InstanceMap im = {nullptr, nullptr}) {
  RowPlan pl;
  pl.row = -1;
  pl.p = 0;
  pl.end = 0;
  pl.leader = false;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int blk = blockIdx.x;
  if (blk < bins.vlong_blocks) {
    pl.path = 2;
    pl.stride = kBlock;
    pl.row = __ldg(bins.vlong_rows + blk);
    pl.p = __ldg(M.ptr + pl.row) + threadIdx.x;
    pl.end = __ldg(M.ptr + pl.row + 1);
    pl.leader = threadIdx.x == 0;
  } else if ((blk -= bins.vlong_blocks) < bins.long_blocks) {
    pl.path = 1;
    pl.stride = 32;
    const int q = blk * (kBlock / 32) + warp;
    if (q < bins.n_long) {
      pl.row = __ldg(bins.long_rows + q);
      pl.p = __ldg(M.ptr + pl.row) + lane;
      pl.end = __ldg(M.ptr + pl.row + 1);
      pl.leader = lane == 0;
    }
  } else {
    blk -= bins.long_blocks;
    pl.path = 0;
    pl.stride = G;
    const int q = (blk * kBlock + threadIdx.x) / G;
    const int row = bins.short_rows ? (q < bins.n_short ? __ldg(bins.short_rows + q) : M.rows) : q;
    if (row < M.rows) {
      const int beg = __ldg(M.ptr + row), end = __ldg(M.ptr + row + 1);
      if (end - beg <= bins.long_thr) {
        pl.row = row;
        pl.p = beg + (threadIdx.x & (G - 1));
        pl.end = end;
        pl.leader = (threadIdx.x & (G - 1)) == 0;
      }
    }
  }
  // multi-LP: the row's instance is fetched beside the pairs, and a
  // terminated instance's row drops its gathers and epilogue afterwards (so
  // the pair loads do not wait for the instance's done flag)
  const int32_t inst = (MULTI && pl.row >= 0) ? __ldg(im.inst + pl.row) : 0;
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const int q = pl.p + u * pl.stride;
    const bool ok = q < pl.end;
    pl.ci[u] = ok ? ld_once<STREAM>(M.idx + q) : 0;
    pl.cv[u] = ok ? ld_once<STREAM>(M.val + q) : 0.0;
  }
  if (MULTI && pl.row >= 0 && __ldcg(im.done + inst)) {
    pl.end = pl.p;  // terminated instance: no work
    pl.leader = false;
  }
  return pl;
}

template <int W>
__device__ __forceinline__ double lane_tree(double s) {
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, off));
  return s;
}

// Post-wait part: the gathers, the lane sums and the tree.  Called by every
// thread of the block (warp shuffles; __syncthreads on the block path, which
// is block-uniform).  The result is valid on the leader thread.
template <int G, bool STREAM = false>
__device__ __forceinline__ double finish_row(const RowPlan& pl, const CsrView& M, const double* __restrict__ x,
                                             double* sh /* kBlock/32 doubles */) {
  double xv[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) xv[u] = (pl.p + u * pl.stride < pl.end) ? __ldcg(x + pl.ci[u]) : 0.0;
  double s = 0.0;
#pragma unroll
  for (int u = 0; u < kUnroll; ++u)
    if (pl.p + u * pl.stride < pl.end) s = (u == 0) ? __dmul_rn(pl.cv[0], xv[0]) : __dadd_rn(s, __dmul_rn(pl.cv[u], xv[u]));
  // Rows longer than kUnroll chunks (warp and block paths): further rounds.
  for (int p = pl.p + kUnroll * pl.stride; p < pl.end; p += kUnroll * pl.stride) {
    int ci[kUnroll];
    double cv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int q = p + u * pl.stride;
      ci[u] = q < pl.end ? ld_once<STREAM>(M.idx + q) : 0;
      cv[u] = q < pl.end ? ld_once<STREAM>(M.val + q) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) xv[u] = (p + u * pl.stride < pl.end) ? __ldcg(x + ci[u]) : 0.0;
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
      if (p + u * pl.stride < pl.end) s = __dadd_rn(s, __dmul_rn(cv[u], xv[u]));
  }
  if (pl.path == 0) return lane_tree<G>(s);
  s = lane_tree<32>(s);
  if (pl.path == 1) return s;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = s;
  __syncthreads();
  double v = lane < kBlock / 32 ? sh[lane] : 0.0;
  return lane_tree<32>(v);
}

// x+ = proj(x - tau (c - A^T y)), Halpern step of x (skipped at a check
// iteration).  A^T rows binned.  MULTI: several LPs, per-row instance b
// selects tau[b] and the Halpern counter of b.
// (the kernel bodies are device functions so that the tiled kernels can run
// the long rows in the same launch; sh: kBlock / 32 doubles of shared memory)
template <int G, bool HALPERN, bool MULTI, bool STREAM>
__device__ __forceinline__ void primal_binned_body(const CsrView& AT, const RowBins& bins, const double* __restrict__ y,
                                                   const double* __restrict__ c, const double* __restrict__ lo,
                                                   const double* __restrict__ up, double* __restrict__ x,
                                                   double* __restrict__ xp, const double* __restrict__ x0,
                                                   const double* __restrict__ tau, const IterClock& ck, double rho,
                                                   const InstanceMap& im, double* sh) {
  const RowPlan pl = plan_row<G, MULTI, STREAM>(AT, bins, im);
  const int j = pl.row;
  const int b = (MULTI && pl.leader) ? im.inst[j] : 0;
  double cj = 0, l = 0, u = 0;
  if (pl.leader) {
    cj = ld_once<STREAM>(c + j);
    l = ld_once<STREAM>(lo + j);
    u = ld_once<STREAM>(up + j);
  }
  pdl_wait();
  double xv = 0, x0v = 0, t = 0, lam = 0;
  if (pl.leader) {
    xv = STREAM ? __ldcs(x + j) : __ldcg(x + j);
    t = __ldcg(tau + b);
    if (HALPERN) {
      x0v = STREAM ? __ldcs(x0 + j) : __ldcg(x0 + j);
      lam = halpern_lambda(ck, b);
    }
  }
  const double aty = finish_row<G, STREAM>(pl, AT, y, sh);
  pdl_launch_dependents();
  if (!pl.leader) return;
  double v = __dsub_rn(xv, __dmul_rn(t, __dsub_rn(cj, aty)));
  v = (v < l) ? l : v;
  v = (u < v) ? u : v;
  xp[j] = v;
  if (HALPERN) x[j] = halpern_step(xv, v, x0v, lam, rho);
}

template <int G, bool HALPERN, bool MULTI = false, bool STREAM = false>
__global__ void __launch_bounds__(kBlock) k_primal_binned(CsrView AT, RowBins bins, const double* __restrict__ y,
                                                          const double* __restrict__ c, const double* __restrict__ lo,
                                                          const double* __restrict__ up, double* __restrict__ x,
                                                          double* __restrict__ xp, const double* __restrict__ x0,
                                                          const double* __restrict__ tau, IterClock ck, double rho,
                                                          InstanceMap im = {nullptr, nullptr}) {
  __shared__ double sh[kBlock / 32];
  primal_binned_body<G, HALPERN, MULTI, STREAM>(AT, bins, y, c, lo, up, x, xp, x0, tau, ck, rho, im, sh);
}

// y+ = v + sigma proj(-v/sigma), v = y - sigma (2 A x+ - A x); Halpern steps of y and Ax.
template <int G, bool HALPERN, bool MULTI, bool STREAM>
__device__ __forceinline__ void dual_binned_body(const CsrView& A, const RowBins& bins, const double* __restrict__ xp,
                                                 const double* __restrict__ rl, const double* __restrict__ ru,
                                                 double* __restrict__ y, double* __restrict__ yp,
                                                 const double* __restrict__ y0, double* __restrict__ ax,
                                                 double* __restrict__ axp, const double* __restrict__ ax0,
                                                 const double* __restrict__ sigma, const IterClock& ck, double rho,
                                                 const InstanceMap& im, double* sh) {
  const RowPlan pl = plan_row<G, MULTI, STREAM>(A, bins, im);
  const int i = pl.row;
  const int b = (MULTI && pl.leader) ? im.inst[i] : 0;
  double l = 0, u = 0;
  if (pl.leader) {
    l = ld_once<STREAM>(rl + i);
    u = ld_once<STREAM>(ru + i);
  }
  pdl_wait();
  double axv = 0, yv = 0, s = 0, y0v = 0, ax0v = 0, lam = 0;
  if (pl.leader) {
    axv = STREAM ? __ldcs(ax + i) : __ldcg(ax + i);
    yv = STREAM ? __ldcs(y + i) : __ldcg(y + i);
    s = __ldcg(sigma + b);
    if (HALPERN) {
      y0v = STREAM ? __ldcs(y0 + i) : __ldcg(y0 + i);
      ax0v = STREAM ? __ldcs(ax0 + i) : __ldcg(ax0 + i);
      lam = halpern_lambda(ck, b);
    }
  }
  const double axpv = finish_row<G, STREAM>(pl, A, xp, sh);
  pdl_launch_dependents();
  if (!pl.leader) return;
  const double v = __dsub_rn(yv, __dmul_rn(s, __dsub_rn(__dmul_rn(2.0, axpv), axv)));
  double w = __ddiv_rn(-v, s);
  w = (w < l) ? l : w;
  w = (u < w) ? u : w;
  const double ypv = __dadd_rn(v, __dmul_rn(s, w));
  axp[i] = axpv;
  yp[i] = ypv;
  if (HALPERN) {
    y[i] = halpern_step(yv, ypv, y0v, lam, rho);
    ax[i] = halpern_step(axv, axpv, ax0v, lam, rho);
  }
}

template <int G, bool HALPERN, bool MULTI = false, bool STREAM = false>
__global__ void __launch_bounds__(kBlock) k_dual_binned(CsrView A, RowBins bins, const double* __restrict__ xp,
                                                        const double* __restrict__ rl, const double* __restrict__ ru,
                                                        double* __restrict__ y, double* __restrict__ yp,
                                                        const double* __restrict__ y0, double* __restrict__ ax,
                                                        double* __restrict__ axp, const double* __restrict__ ax0,
                                                        const double* __restrict__ sigma, IterClock ck, double rho,
                                                        InstanceMap im = {nullptr, nullptr}) {
  __shared__ double sh[kBlock / 32];
  dual_binned_body<G, HALPERN, MULTI, STREAM>(A, bins, xp, rl, ru, y, yp, y0, ax, axp, ax0, sigma, ck, rho, im, sh);
}

// out = M x with the binned schedule (used for A^T y+ at a check).
template <int G, bool MULTI, bool STREAM>
__device__ __forceinline__ void spmv_binned_body(const CsrView& M, const RowBins& bins, const double* __restrict__ x,
                                                 double* __restrict__ out, const InstanceMap& im, double* sh) {
  const RowPlan pl = plan_row<G, MULTI, STREAM>(M, bins, im);
  pdl_wait();
  const double s = finish_row<G, STREAM>(pl, M, x, sh);
  pdl_launch_dependents();
  if (pl.leader) out[pl.row] = s;
}

template <int G, bool MULTI = false>
__global__ void __launch_bounds__(kBlock) k_spmv_binned(CsrView M, RowBins bins, const double* __restrict__ x,
                                                        double* __restrict__ out, InstanceMap im = {nullptr, nullptr}) {
  __shared__ double sh[kBlock / 32];
  spmv_binned_body<G, MULTI, false>(M, bins, x, out, im, sh);
}

}  // namespace b2p
