// Row-length-binned CSR row sums for one LP (k = 1), used by the fused
// iteration kernels.
//
// Rows are split by length on the host (RowBins):
//   short rows (len <= long_thr): a group of G lanes per row (G = 1..32, a
//       power of two picked from the average row length), 32/G rows per warp,
//       in the original row order;
//   long rows  (long_thr < len <= vlong_thr): one warp per row;
//   very long rows (len > vlong_thr): one 256-thread block per row.
// Each lane accumulates the products of the entries p = lane, lane+G, ...
// left to right; the lanes are then combined by a fixed xor-shuffle tree, so
// the sum is deterministic (it differs from the reference's strictly
// sequential row sum only in rounding order).
//
// Programmatic dependent launch: the row pointers and the first chunk of
// column indices and values (constant during a solve) are loaded before
// griddepcontrol.wait, i.e. while the previous kernel is still draining;
// everything that kernel wrote is read after the wait.
#pragma once

#include <cstdint>

#include "pdhg_kernels.cuh"

namespace b2p {

struct RowBins {
  const int32_t* __restrict__ long_rows;   // rows for the warp path
  const int32_t* __restrict__ vlong_rows;  // rows for the block path
  int32_t n_long, n_vlong;
  int32_t long_thr;      // rows longer than this are not in the short path
  int32_t vlong_blocks;  // == n_vlong
  int32_t long_blocks;   // ceil(n_long / warps per block)
  int32_t short_blocks;
  int32_t g;             // lanes per short row
};

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// Result of the calling thread: `row` >= 0 and `leader` set on exactly one
// thread per row, which then runs the row's epilogue.
struct RowSum {
  int32_t row;
  bool leader;
  double value;
};

template <int G>
__device__ __forceinline__ double group_sum(double s) {
#pragma unroll
  for (int off = G / 2; off > 0; off >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, off));
  return s;
}

// Sum of the row's entries p = beg+lane0, +stride, ... with the first entry
// prefetched before the dependency wait.
template <int STRIDE>
__device__ __forceinline__ double strided_dot(const CsrView& M, const double* __restrict__ x, int beg, int end,
                                              int lane0) {
  int p = beg + lane0;
  int ci = 0;
  double cv = 0.0;
  if (p < end) {
    ci = __ldg(M.idx + p);
    cv = __ldg(M.val + p);
  }
  pdl_wait();
  double s = 0.0;
  if (p < end) s = __dmul_rn(cv, __ldcg(x + ci));
  for (p += STRIDE; p < end; p += STRIDE) s = __dadd_rn(s, __dmul_rn(__ldg(M.val + p), __ldcg(x + __ldg(M.idx + p))));
  return s;
}

// Dispatch of one thread of a binned row-sum grid.  Every thread of the
// block calls this (it contains warp shuffles and, on the block path, a
// __syncthreads); it performs griddepcontrol.wait exactly once.
template <int G>
__device__ __forceinline__ RowSum binned_row_sum(const CsrView& M, const RowBins& bins, const double* __restrict__ x,
                                                 double* sh /* kBlock/32 doubles */) {
  RowSum r{-1, false, 0.0};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int blk = blockIdx.x;
  if (blk < bins.vlong_blocks) {
    // one block per very long row
    const int row = __ldg(bins.vlong_rows + blk);
    const int beg = __ldg(M.ptr + row), end = __ldg(M.ptr + row + 1);
    double s = strided_dot<kBlock>(M, x, beg, end, threadIdx.x);
    s = group_sum<32>(s);
    if (lane == 0) sh[warp] = s;
    __syncthreads();
    if (warp == 0) {
      double v = lane < kBlock / 32 ? sh[lane] : 0.0;
      v = group_sum<32>(v);
      if (lane == 0) r = RowSum{row, true, v};
    }
    return r;
  }
  blk -= bins.vlong_blocks;
  if (blk < bins.long_blocks) {
    // one warp per long row
    const int q = blk * (kBlock / 32) + warp;
    int beg = 0, end = 0, row = -1;
    if (q < bins.n_long) {
      row = __ldg(bins.long_rows + q);
      beg = __ldg(M.ptr + row);
      end = __ldg(M.ptr + row + 1);
    }
    double s = strided_dot<32>(M, x, beg, end, lane);
    s = group_sum<32>(s);
    if (row >= 0 && lane == 0) r = RowSum{row, true, s};
    return r;
  }
  blk -= bins.long_blocks;
  // G lanes per short row
  const int row = (blk * kBlock + threadIdx.x) / G;
  const int gl = threadIdx.x & (G - 1);
  int beg = 0, end = 0;
  bool mine = false;
  if (row < M.rows) {
    beg = __ldg(M.ptr + row);
    end = __ldg(M.ptr + row + 1);
    mine = end - beg <= bins.long_thr;
    if (!mine) end = beg;  // handled by the warp or block path
  }
  double s = strided_dot<G>(M, x, beg, end, gl);
  s = group_sum<G>(s);
  if (mine && gl == 0) r = RowSum{row, true, s};
  return r;
}

// x+ = proj(x - tau (c - A^T y)), Halpern step of x (skipped at a check
// iteration).  One LP; A^T rows binned.
template <int G, bool HALPERN>
__global__ void __launch_bounds__(kBlock) k_primal_binned(CsrView AT, RowBins bins, const double* __restrict__ y,
                                                          const double* __restrict__ c, const double* __restrict__ lo,
                                                          const double* __restrict__ up, double* __restrict__ x,
                                                          double* __restrict__ xp, const double* __restrict__ x0,
                                                          const double* __restrict__ tau, IterClock ck, double rho) {
  __shared__ double sh[kBlock / 32];
  const RowSum r = binned_row_sum<G>(AT, bins, y, sh);
  pdl_launch_dependents();
  if (!r.leader) return;
  const int j = r.row;
  const double xv = __ldcg(x + j);
  double v = __dsub_rn(xv, __dmul_rn(__ldcg(tau), __dsub_rn(__ldg(c + j), r.value)));
  const double l = __ldg(lo + j), u = __ldg(up + j);
  v = (v < l) ? l : v;
  v = (u < v) ? u : v;
  xp[j] = v;
  if (HALPERN) x[j] = halpern_step(xv, v, __ldcg(x0 + j), halpern_lambda(ck, 0), rho);
}

// y+ = v + sigma proj(-v/sigma), v = y - sigma (2 A x+ - A x); Halpern steps of y and Ax.
template <int G, bool HALPERN>
__global__ void __launch_bounds__(kBlock) k_dual_binned(CsrView A, RowBins bins, const double* __restrict__ xp,
                                                        const double* __restrict__ rl, const double* __restrict__ ru,
                                                        double* __restrict__ y, double* __restrict__ yp,
                                                        const double* __restrict__ y0, double* __restrict__ ax,
                                                        double* __restrict__ axp, const double* __restrict__ ax0,
                                                        const double* __restrict__ sigma, IterClock ck, double rho) {
  __shared__ double sh[kBlock / 32];
  const RowSum r = binned_row_sum<G>(A, bins, xp, sh);
  pdl_launch_dependents();
  if (!r.leader) return;
  const int i = r.row;
  const double axpv = r.value, axv = __ldcg(ax + i), yv = __ldcg(y + i);
  const double s = __ldcg(sigma);
  const double v = __dsub_rn(yv, __dmul_rn(s, __dsub_rn(__dmul_rn(2.0, axpv), axv)));
  double w = __ddiv_rn(-v, s);
  const double l = __ldg(rl + i), u = __ldg(ru + i);
  w = (w < l) ? l : w;
  w = (u < w) ? u : w;
  const double ypv = __dadd_rn(v, __dmul_rn(s, w));
  axp[i] = axpv;
  yp[i] = ypv;
  if (HALPERN) {
    const double lam = halpern_lambda(ck, 0);
    y[i] = halpern_step(yv, ypv, __ldcg(y0 + i), lam, rho);
    ax[i] = halpern_step(axv, axpv, __ldcg(ax0 + i), lam, rho);
  }
}

// out = M x with the binned schedule (used for A^T y+ at a check).
template <int G>
__global__ void __launch_bounds__(kBlock) k_spmv_binned(CsrView M, RowBins bins, const double* __restrict__ x,
                                                        double* __restrict__ out) {
  __shared__ double sh[kBlock / 32];
  const RowSum r = binned_row_sum<G>(M, bins, x, sh);
  pdl_launch_dependents();
  if (r.leader) out[r.row] = r.value;
}

}  // namespace b2p
