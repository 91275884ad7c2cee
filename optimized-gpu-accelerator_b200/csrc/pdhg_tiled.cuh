// TMA-staged row tiles for the fused iteration kernels of large (HBM-bound)
// operators.
//
// The host cuts the short rows (<= kTileRowMax entries) of a CSR operator into
// tiles of consecutive rows -- at most kBlock rows and kTileEntries entries,
// never crossing an LP of a multi-LP batch -- and leaves the longer rows to
// the binned warp / block paths (a separate launch).  A tile's (index, value)
// pairs are one contiguous range, so a persistent CTA streams them into shared
// memory with two bulk asynchronous copies (cp.async.bulk, completing on an
// mbarrier), double-buffered: while tile t is processed, tile t + grid is
// already in flight.  Per tile every thread gathers up to
// kTileEntries / kBlock operands x[idx] (independent loads), writes the
// products to a third, ordinary shared array (so the copy buffers are only
// ever written by the copies and need no proxy fence before they are
// refilled), and then thread r sums the products of row
// r0 + r left to right -- the reference's own row order -- and runs that row's
// epilogue (primal / dual step, Halpern, stores; loads for it are issued
// before the wait).  The operator stream and the epilogue's vectors are
// evict-first in L2, so that L2 keeps the gathered vector.  Rows of terminated LPs are skipped per tile.
//
// Bulk copies need 16-byte aligned addresses and sizes: the copied range is
// widened to multiples of 4 entries (the operator arrays carry >= 8 entries of
// padding), and the rows index into it from the rounded start.  Every mbarrier
// wait is bounded; on a timeout the CTA records an error, waits (bounded) for
// the copy it still has in flight and leaves.
#pragma once

#include <cstdint>

#include "pdhg_kernels.cuh"
#include "pdhg_spmv.cuh"

namespace b2p {

constexpr int kTileEntries = 1536;
constexpr int kTileRowMax = 32;  // longer rows take the binned warp / block path
constexpr int kTileBuf = kTileEntries + 8;
constexpr int kTilePad = 8;      // entries of padding the operator arrays must carry
constexpr unsigned kTileSpinLimit = 1u << 24;
// dynamic shared memory of a tile CTA: two copy buffers of indices and values
// and one array of products (49,408 B: four CTAs per SM)
constexpr int kTileSmemBytes = 2 * kTileBuf * (4 + 8) + kTileBuf * 8;

struct TileSet {
  const int4* __restrict__ tiles;       // (row begin, row end, entry begin, entry end)
  const int32_t* __restrict__ inst;     // LP of each tile (multi-LP), or NULL
  int32_t n_tiles;
  int32_t grid;                         // persistent CTAs
  int32_t* err;                         // set to 1 on an mbarrier timeout
};

namespace tiled {

__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase) {
  for (unsigned spin = 0; spin < kTileSpinLimit; ++spin) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// L2 policy for the operator stream: evict first, so that L2 keeps the
// vector the rows gather from.
__device__ __forceinline__ uint64_t evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// Issue the copies of tile d's pairs into (sidx, sval), completing on bar.
__device__ __forceinline__ void issue(const CsrView& M, int4 d, int32_t* sidx, double* sval, uint32_t bar) {
  const int e0 = d.z & ~3, e1 = (d.w + 3) & ~3;
  const uint32_t n = static_cast<uint32_t>(e1 - e0);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(n * 12u) : "memory");
  if (n == 0) return;
  const uint64_t pol = evict_first_policy();
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          saddr(sidx)),
      "l"(M.idx + e0), "r"(n * 4u), "r"(bar), "l"(pol)
      : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          saddr(sval)),
      "l"(M.val + e0), "r"(n * 8u), "r"(bar), "l"(pol)
      : "memory");
}

// The pipeline state of one persistent CTA (buffers addressed arithmetically
// and phases kept as bits, so that nothing is indexed at run time in local
// memory).
struct Pipe {
  int32_t* sidx0;
  double* sval0;
  double* sprod;
  uint64_t* bars;
  int* fail;
  uint32_t phases;  // bit b: parity to wait for on buffer b
  __device__ __forceinline__ int32_t* idx(int b) const { return sidx0 + b * kTileBuf; }
  __device__ __forceinline__ double* val(int b) const { return sval0 + b * kTileBuf; }
  __device__ __forceinline__ uint32_t bar(int b) const { return saddr(bars + b); }
};

__device__ __forceinline__ Pipe setup(unsigned char* smem, uint64_t* bars, int* fail) {
  Pipe p;
  p.sidx0 = reinterpret_cast<int32_t*>(smem);
  p.sval0 = reinterpret_cast<double*>(smem + 2 * kTileBuf * 4);
  p.sprod = p.sval0 + 2 * kTileBuf;
  p.bars = bars;
  p.fail = fail;
  p.phases = 0;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&bars[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&bars[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *fail = 0;
  }
  __syncthreads();
  return p;
}

// Products x[idx] * val of tile d into sprod, then a block barrier.  Returns
// false (for the whole CTA) if the tile's copy did not arrive in time.
__device__ __forceinline__ bool products(Pipe& p, int buf, int4 d, const double* __restrict__ x, bool skip) {
  if (!bar_wait(p.bar(buf), (p.phases >> buf) & 1u)) *p.fail = 1;
  p.phases ^= 1u << buf;
  __syncthreads();
  if (*p.fail) return false;
  if (!skip) {
    const int e0 = d.z & ~3, lo = d.z - e0, hi = d.w - e0;
    const int32_t* si = p.idx(buf);
    const double* sv = p.val(buf);
    constexpr int kPer = kTileEntries / kBlock;
    double xv[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = lo + threadIdx.x + u * kBlock;
      xv[u] = e < hi ? __ldcg(x + si[e]) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = lo + threadIdx.x + u * kBlock;
      if (e < hi) p.sprod[e] = __dmul_rn(sv[e], xv[u]);
    }
  }
  __syncthreads();
  return true;
}

// Left-to-right sum of the products of entries [rb, re) of tile d.
__device__ __forceinline__ double row_sum(const Pipe& p, int4 d, int rb, int re) {
  const int e0 = d.z & ~3;
  const double* sv = p.sprod;
  double s = 0.0;
  int q = rb - e0;
  const int qe = re - e0;
  for (; q + 4 <= qe; q += 4) {  // four independent loads, then the in-order adds
    const double a = sv[q], b = sv[q + 1], c = sv[q + 2], e = sv[q + 3];
    s = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(s, a), b), c), e);
  }
  for (; q < qe; ++q) s = __dadd_rn(s, sv[q]);
  return s;
}

// End of a tile: every thread is done with its copy buffer and the products
// before either is reused.
__device__ __forceinline__ void tile_done() { __syncthreads(); }

// After a timeout: wait (bounded) for the copy still in flight into `buf`.
__device__ __forceinline__ void drain(Pipe& p, int buf, bool pending, int32_t* err) {
  if (threadIdx.x == 0) {
    if (pending) bar_wait(p.bar(buf), (p.phases >> buf) & 1u);
    atomicExch(err, 1);
  }
}

}  // namespace tiled

// x+ = proj(x - tau (c - A^T y)) and the Halpern step of x, over the tiled
// short rows of A^T (see k_primal_binned for the arithmetic).
template <bool HALPERN, bool MULTI>
__global__ void __launch_bounds__(kBlock) k_primal_tiled(CsrView AT, TileSet ts, const double* __restrict__ y,
                                                         const double* __restrict__ c, const double* __restrict__ lo,
                                                         const double* __restrict__ up, double* __restrict__ x,
                                                         double* __restrict__ xp, const double* __restrict__ x0,
                                                         const double* __restrict__ tau, IterClock ck, double rho,
                                                         InstanceMap im) {
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int fail;
  tiled::Pipe p = tiled::setup(tsm, bars, &fail);
  int t = blockIdx.x;
  if (threadIdx.x == 0 && t < ts.n_tiles)
    tiled::issue(AT, __ldg(ts.tiles + t), p.idx(0), p.val(0), p.bar(0));
  pdl_wait();
  for (int it = 0; t < ts.n_tiles; t += ts.grid, ++it) {
    const int buf = it & 1;
    const int tn = t + ts.grid;
    if (threadIdx.x == 0 && tn < ts.n_tiles)
      tiled::issue(AT, __ldg(ts.tiles + tn), p.idx(buf ^ 1), p.val(buf ^ 1), p.bar(buf ^ 1));
    const int4 d = __ldg(ts.tiles + t);
    const int b = MULTI ? __ldg(ts.inst + t) : 0;
    const bool skip = MULTI && __ldcg(im.done + b) != 0;
    const int j = d.x + threadIdx.x;
    const bool row = j < d.y;  // loads need only the tile; the done flag gates the work
    int rb = 0, re = 0;
    double cj = 0, l = 0, u = 0, xv = 0, x0v = 0, tv = 0, lam = 0;
    if (row) {
      rb = __ldg(AT.ptr + j);
      re = __ldg(AT.ptr + j + 1);
      cj = __ldcs(c + j);
      l = __ldcs(lo + j);
      u = __ldcs(up + j);
      xv = __ldcs(x + j);
      tv = __ldcg(tau + b);
      if (HALPERN) {
        x0v = __ldcs(x0 + j);
        lam = halpern_lambda(ck, b);
      }
    }
    if (!tiled::products(p, buf, d, y, skip)) {
      tiled::drain(p, buf ^ 1, tn < ts.n_tiles, ts.err);
      return;
    }
    if (row && !skip) {
      const double aty = tiled::row_sum(p, d, rb, re);
      double v = __dsub_rn(xv, __dmul_rn(tv, __dsub_rn(cj, aty)));
      v = (v < l) ? l : v;
      v = (u < v) ? u : v;
      xp[j] = v;
      if (HALPERN) x[j] = halpern_step(xv, v, x0v, lam, rho);
    }
    tiled::tile_done();
  }
  pdl_launch_dependents();
}

// y+ = v + sigma proj(-v/sigma), v = y - sigma (2 A x+ - A x); Halpern steps
// of y and Ax, over the tiled short rows of A (see k_dual_binned).
template <bool HALPERN, bool MULTI>
__global__ void __launch_bounds__(kBlock) k_dual_tiled(CsrView A, TileSet ts, const double* __restrict__ xp,
                                                       const double* __restrict__ rl, const double* __restrict__ ru,
                                                       double* __restrict__ y, double* __restrict__ yp,
                                                       const double* __restrict__ y0, double* __restrict__ ax,
                                                       double* __restrict__ axp, const double* __restrict__ ax0,
                                                       const double* __restrict__ sigma, IterClock ck, double rho,
                                                       InstanceMap im) {
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int fail;
  tiled::Pipe p = tiled::setup(tsm, bars, &fail);
  int t = blockIdx.x;
  if (threadIdx.x == 0 && t < ts.n_tiles)
    tiled::issue(A, __ldg(ts.tiles + t), p.idx(0), p.val(0), p.bar(0));
  pdl_wait();
  for (int it = 0; t < ts.n_tiles; t += ts.grid, ++it) {
    const int buf = it & 1;
    const int tn = t + ts.grid;
    if (threadIdx.x == 0 && tn < ts.n_tiles)
      tiled::issue(A, __ldg(ts.tiles + tn), p.idx(buf ^ 1), p.val(buf ^ 1), p.bar(buf ^ 1));
    const int4 d = __ldg(ts.tiles + t);
    const int b = MULTI ? __ldg(ts.inst + t) : 0;
    const bool skip = MULTI && __ldcg(im.done + b) != 0;
    const int i = d.x + threadIdx.x;
    const bool row = i < d.y;
    int rb = 0, re = 0;
    double l = 0, u = 0, axv = 0, yv = 0, s = 0, y0v = 0, ax0v = 0, lam = 0;
    if (row) {
      rb = __ldg(A.ptr + i);
      re = __ldg(A.ptr + i + 1);
      l = __ldcs(rl + i);
      u = __ldcs(ru + i);
      axv = __ldcs(ax + i);
      yv = __ldcs(y + i);
      s = __ldcg(sigma + b);
      if (HALPERN) {
        y0v = __ldcs(y0 + i);
        ax0v = __ldcs(ax0 + i);
        lam = halpern_lambda(ck, b);
      }
    }
    if (!tiled::products(p, buf, d, xp, skip)) {
      tiled::drain(p, buf ^ 1, tn < ts.n_tiles, ts.err);
      return;
    }
    if (row && !skip) {
      const double axpv = tiled::row_sum(p, d, rb, re);
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
    tiled::tile_done();
  }
  pdl_launch_dependents();
}

// out = M x over the tiled short rows (A^T y+ at a check).
template <bool MULTI>
__global__ void __launch_bounds__(kBlock) k_spmv_tiled(CsrView M, TileSet ts, const double* __restrict__ x,
                                                       double* __restrict__ out, InstanceMap im) {
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int fail;
  tiled::Pipe p = tiled::setup(tsm, bars, &fail);
  int t = blockIdx.x;
  if (threadIdx.x == 0 && t < ts.n_tiles)
    tiled::issue(M, __ldg(ts.tiles + t), p.idx(0), p.val(0), p.bar(0));
  pdl_wait();
  for (int it = 0; t < ts.n_tiles; t += ts.grid, ++it) {
    const int buf = it & 1;
    const int tn = t + ts.grid;
    if (threadIdx.x == 0 && tn < ts.n_tiles)
      tiled::issue(M, __ldg(ts.tiles + tn), p.idx(buf ^ 1), p.val(buf ^ 1), p.bar(buf ^ 1));
    const int4 d = __ldg(ts.tiles + t);
    const bool skip = MULTI && __ldcg(im.done + __ldg(ts.inst + t)) != 0;
    const int r = d.x + threadIdx.x;
    const bool row = r < d.y;
    int rb = 0, re = 0;
    if (row) {
      rb = __ldg(M.ptr + r);
      re = __ldg(M.ptr + r + 1);
    }
    if (!tiled::products(p, buf, d, x, skip)) {
      tiled::drain(p, buf ^ 1, tn < ts.n_tiles, ts.err);
      return;
    }
    if (row && !skip) out[r] = tiled::row_sum(p, d, rb, re);
    tiled::tile_done();
  }
  pdl_launch_dependents();
}

}  // namespace b2p
