// Warp tiles of short rows for the fused iteration kernels of large
// operators (schedule B2P_SCHEDULE_TILED).
//
// The host cuts the short rows (<= kTileRowMax = 32 entries) of a CSR operator
// into tiles of consecutive rows -- at most 32 rows and kTileEntries = 256
// entries, never crossing an LP of a multi-LP batch -- and leaves the longer
// rows to the binned warp / block paths, which the first blocks of the same
// launch run (RowBins of the long rows only).  One warp per
// tile: the tile's (index, value) pairs are one contiguous range, so lane l
// loads entries e0 + l + 32k (k < 8; fully coalesced, all independent, issued
// before griddepcontrol.wait since the operator is constant), gathers the 8
// operands, and writes the products to its warp's slice of shared memory;
// then lane r sums the products of row r0 + r left to right -- the
// reference's own row order -- and runs that row's epilogue (primal / dual
// step, Halpern, stores).  No block-wide barrier: warps are independent.
// Operator and epilogue loads are evict-first streaming loads, so that L2
// keeps the vector the rows gather from.
//
// Why not bulk (TMA) copies of CTA-sized tiles: measured on the B200 with a
// 33M-nonzero random operator, double-buffered cp.async.bulk tiles of 1,536
// entries per CTA sustained 1.7 TB/s even with the gathers removed, against
// 6.7 TB/s for plain coalesced loads; warp tiles come within ~17% of the time
// the operator's random gathers alone take (one 32-byte L2 sector per 8-byte
// operand), which is what bounds an SpMV of that structure.
#pragma once

#include <cstdint>

#include "pdhg_kernels.cuh"
#include "pdhg_spmv.cuh"

namespace b2p {

constexpr int kTileEntries = 256;  // entries per warp tile
constexpr int kTileRowMax = 32;    // longer rows take the binned warp / block path
constexpr int kTileRows = 32;      // rows per warp tile (one per lane)
constexpr int kTilePad = 8;        // zero entries the operator arrays carry at the end
constexpr int kTileK = kTileEntries / 32;

struct TileSet {
  const int4* __restrict__ tiles;    // (row begin, row end, entry begin, entry end)
  const int32_t* __restrict__ inst;  // LP of each tile (multi-LP), or NULL
  int32_t n_tiles;
  int32_t grid;                      // blocks: the long-row blocks, then one warp per tile
};

namespace tiled {

// The lane's pairs of tile d: entries d.z + lane + 32k (streaming loads).
struct Pairs {
  int32_t ci[kTileK];
  double cv[kTileK];
};

__device__ __forceinline__ Pairs load_pairs(const CsrView& M, int4 d, int lane) {
  Pairs p;
#pragma unroll
  for (int k = 0; k < kTileK; ++k) {
    const int e = d.z + lane + 32 * k;
    const bool ok = e < d.w;
    p.ci[k] = ok ? __ldcs(M.idx + e) : 0;
    p.cv[k] = ok ? __ldcs(M.val + e) : 0.0;
  }
  return p;
}

// Products of the tile into the warp's shared slice (skip: terminated LP).
__device__ __forceinline__ void products(const Pairs& p, int4 d, int lane, const double* __restrict__ x, double* prod,
                                         bool skip) {
  if (!skip) {
    double xv[kTileK];
#pragma unroll
    for (int k = 0; k < kTileK; ++k) xv[k] = (d.z + lane + 32 * k < d.w) ? __ldcg(x + p.ci[k]) : 0.0;
#pragma unroll
    for (int k = 0; k < kTileK; ++k) prod[lane + 32 * k] = __dmul_rn(p.cv[k], xv[k]);
  }
  __syncwarp();
}

// Left-to-right sum of the products of entries [rb, re) (four loads ahead).
__device__ __forceinline__ double row_sum(const double* prod, int4 d, int rb, int re) {
  double s = 0.0;
  int q = rb - d.z;
  const int qe = re - d.z;
  for (; q + 4 <= qe; q += 4) {
    const double a = prod[q], b = prod[q + 1], c = prod[q + 2], e = prod[q + 3];
    s = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(s, a), b), c), e);
  }
  for (; q < qe; ++q) s = __dadd_rn(s, prod[q]);
  return s;
}

}  // namespace tiled

// x+ = proj(x - tau (c - A^T y)) and the Halpern step of x, over the tiled
// short rows of A^T (see k_primal_binned for the arithmetic).
template <bool HALPERN, bool MULTI, int MINB = 1>
__global__ void __launch_bounds__(kBlock, MINB) k_primal_tiled(CsrView AT, TileSet ts, RowBins lb, const double* __restrict__ y,
                                                         const double* __restrict__ c, const double* __restrict__ lo,
                                                         const double* __restrict__ up, double* __restrict__ x,
                                                         double* __restrict__ xp, const double* __restrict__ x0,
                                                         const double* __restrict__ tau, IterClock ck, double rho,
                                                         InstanceMap im) {
  __shared__ double prod_all[kBlock / 32][kTileEntries];
  const int nlb = lb.vlong_blocks + lb.long_blocks;  // leading blocks: the long rows
  if (static_cast<int>(blockIdx.x) < nlb) {
    primal_binned_body<1, HALPERN, MULTI, true>(AT, lb, y, c, lo, up, x, xp, x0, tau, ck, rho, im, &prod_all[0][0]);
    return;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int t = (static_cast<int>(blockIdx.x) - nlb) * (kBlock / 32) + w;
  if (t >= ts.n_tiles) return;
  const int4 d = __ldg(ts.tiles + t);
  const int b = MULTI ? __ldg(ts.inst + t) : 0;
  const tiled::Pairs pr = tiled::load_pairs(AT, d, lane);
  const int j = d.x + lane;
  const bool row = j < d.y;
  int rb = 0, re = 0;
  double cj = 0, l = 0, u = 0;
  if (row) {
    rb = __ldg(AT.ptr + j);
    re = __ldg(AT.ptr + j + 1);
    cj = __ldcs(c + j);
    l = __ldcs(lo + j);
    u = __ldcs(up + j);
  }
  pdl_wait();
  const bool skip = MULTI && __ldcg(im.done + b) != 0;
  double xv = 0, x0v = 0, tv = 0, lam = 0;
  if (row) {
    xv = __ldcs(x + j);
    tv = __ldcg(tau + b);
    if (HALPERN) {
      x0v = __ldcs(x0 + j);
      lam = halpern_lambda(ck, b);
    }
  }
  double* prod = prod_all[w];
  tiled::products(pr, d, lane, y, prod, skip);
  pdl_launch_dependents();
  if (!row || skip) return;
  const double aty = tiled::row_sum(prod, d, rb, re);
  double v = __dsub_rn(xv, __dmul_rn(tv, __dsub_rn(cj, aty)));
  v = (v < l) ? l : v;
  v = (u < v) ? u : v;
  xp[j] = v;
  if (HALPERN) x[j] = halpern_step(xv, v, x0v, lam, rho);
}

// y+ = v + sigma proj(-v/sigma), v = y - sigma (2 A x+ - A x); Halpern steps
// of y and Ax, over the tiled short rows of A (see k_dual_binned).
template <bool HALPERN, bool MULTI, int MINB = 1>
__global__ void __launch_bounds__(kBlock, MINB) k_dual_tiled(CsrView A, TileSet ts, RowBins lb, const double* __restrict__ xp,
                                                       const double* __restrict__ rl, const double* __restrict__ ru,
                                                       double* __restrict__ y, double* __restrict__ yp,
                                                       const double* __restrict__ y0, double* __restrict__ ax,
                                                       double* __restrict__ axp, const double* __restrict__ ax0,
                                                       const double* __restrict__ sigma, IterClock ck, double rho,
                                                       InstanceMap im) {
  __shared__ double prod_all[kBlock / 32][kTileEntries];
  const int nlb = lb.vlong_blocks + lb.long_blocks;  // leading blocks: the long rows
  if (static_cast<int>(blockIdx.x) < nlb) {
    dual_binned_body<1, HALPERN, MULTI, true>(A, lb, xp, rl, ru, y, yp, y0, ax, axp, ax0, sigma, ck, rho, im, &prod_all[0][0]);
    return;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int t = (static_cast<int>(blockIdx.x) - nlb) * (kBlock / 32) + w;
  if (t >= ts.n_tiles) return;
  const int4 d = __ldg(ts.tiles + t);
  const int b = MULTI ? __ldg(ts.inst + t) : 0;
  const tiled::Pairs pr = tiled::load_pairs(A, d, lane);
  const int i = d.x + lane;
  const bool row = i < d.y;
  int rb = 0, re = 0;
  double l = 0, u = 0;
  if (row) {
    rb = __ldg(A.ptr + i);
    re = __ldg(A.ptr + i + 1);
    l = __ldcs(rl + i);
    u = __ldcs(ru + i);
  }
  pdl_wait();
  const bool skip = MULTI && __ldcg(im.done + b) != 0;
  double axv = 0, yv = 0, s = 0, y0v = 0, ax0v = 0, lam = 0;
  if (row) {
    axv = __ldcs(ax + i);
    yv = __ldcs(y + i);
    s = __ldcg(sigma + b);
    if (HALPERN) {
      y0v = __ldcs(y0 + i);
      ax0v = __ldcs(ax0 + i);
      lam = halpern_lambda(ck, b);
    }
  }
  double* prod = prod_all[w];
  tiled::products(pr, d, lane, xp, prod, skip);
  pdl_launch_dependents();
  if (!row || skip) return;
  const double axpv = tiled::row_sum(prod, d, rb, re);
  const double v = __dsub_rn(yv, __dmul_rn(s, __dsub_rn(__dmul_rn(2.0, axpv), axv)));
  double wv = __ddiv_rn(-v, s);
  wv = (wv < l) ? l : wv;
  wv = (u < wv) ? u : wv;
  const double ypv = __dadd_rn(v, __dmul_rn(s, wv));
  axp[i] = axpv;
  yp[i] = ypv;
  if (HALPERN) {
    y[i] = halpern_step(yv, ypv, y0v, lam, rho);
    ax[i] = halpern_step(axv, axpv, ax0v, lam, rho);
  }
}

// out = M x over the tiled short rows (A^T y+ at a check).
template <bool MULTI>
__global__ void __launch_bounds__(kBlock) k_spmv_tiled(CsrView M, TileSet ts, RowBins lb, const double* __restrict__ x,
                                                       double* __restrict__ out, InstanceMap im) {
  __shared__ double prod_all[kBlock / 32][kTileEntries];
  const int nlb = lb.vlong_blocks + lb.long_blocks;  // leading blocks: the long rows
  if (static_cast<int>(blockIdx.x) < nlb) {
    spmv_binned_body<1, MULTI, true>(M, lb, x, out, im, &prod_all[0][0]);
    return;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int t = (static_cast<int>(blockIdx.x) - nlb) * (kBlock / 32) + w;
  if (t >= ts.n_tiles) return;
  const int4 d = __ldg(ts.tiles + t);
  const tiled::Pairs pr = tiled::load_pairs(M, d, lane);
  const int r = d.x + lane;
  const bool row = r < d.y;
  int rb = 0, re = 0;
  if (row) {
    rb = __ldg(M.ptr + r);
    re = __ldg(M.ptr + r + 1);
  }
  pdl_wait();
  const bool skip = MULTI && __ldcg(im.done + __ldg(ts.inst + t)) != 0;
  double* prod = prod_all[w];
  tiled::products(pr, d, lane, x, prod, skip);
  pdl_launch_dependents();
  if (row && !skip) out[r] = tiled::row_sum(prod, d, rb, re);
}

}  // namespace b2p
