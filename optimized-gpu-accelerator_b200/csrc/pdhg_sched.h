// Host-side helpers shared by the single-LP and multi-LP engines: model
// validation, the row-length bins of the fused SpMV kernels, and the launch
// helper with programmatic dependent launch.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "pdhg_host_common.h"
#include "pdhg_prepare.h"
#include "pdhg_spmv.cuh"
#include "pdhg_tiled.cuh"

namespace b2p {

inline void check_lp(const b2p_lp* lp) {
  if (!lp) throw Error(B2P_ERR_INVALID, "lp is NULL");
  if (lp->num_rows < 0 || lp->num_cols < 0) throw Error(B2P_ERR_INVALID, "negative dimension");
  if (!lp->start) throw Error(B2P_ERR_INVALID, "start is NULL");
  if (lp->start[0] != 0) throw Error(B2P_ERR_INVALID, "start[0] must be 0");
  for (int32_t j = 0; j < lp->num_cols; ++j)
    if (lp->start[j + 1] < lp->start[j]) throw Error(B2P_ERR_INVALID, "start must be non-decreasing");
  const int32_t nnz = lp->start[lp->num_cols];
  if (nnz > 0 && (!lp->index || !lp->value)) throw Error(B2P_ERR_INVALID, "index/value are NULL");
  for (int32_t q = 0; q < nnz; ++q)
    if (lp->index[q] < 0 || lp->index[q] >= lp->num_rows) throw Error(B2P_ERR_INVALID, "row index out of range");
  if (lp->num_cols > 0 && (!lp->col_cost || !lp->col_lower || !lp->col_upper))
    throw Error(B2P_ERR_INVALID, "column vectors are NULL");
  if (lp->num_rows > 0 && (!lp->row_lower || !lp->row_upper)) throw Error(B2P_ERR_INVALID, "row vectors are NULL");
}

// Row-length bins of one CSR operator (see pdhg_spmv.cuh).
struct HostBins {
  std::vector<int32_t> long_rows, vlong_rows;
  int g = 1;
  int long_thr = kUnroll;
};

// Lanes per short row: enough that 90% of the rows finish in one round of
// kUnroll entries per lane; when fewer lanes would let the whole grid fit in
// one wave of `wave_threads` (a latency-bound operator), the most that fit.
// Operators too large for one wave keep the row-length choice (their waves
// pipeline and the kernels are bandwidth-bound).  `rounds` rounds of kUnroll
// entries stay on the short path.
inline HostBins make_bins(const HostCsr& M, int64_t wave_threads, int g_override, int rounds) {
  HostBins hb;
  std::vector<int32_t> len(M.rows);
  for (int32_t i = 0; i < M.rows; ++i) len[i] = M.ptr[i + 1] - M.ptr[i];
  if (g_override > 0) {
    while (hb.g < 32 && hb.g * 2 <= g_override) hb.g *= 2;
  } else if (M.rows > 0) {
    std::vector<int32_t> sorted(len);
    const size_t q = static_cast<size_t>(0.9 * (sorted.size() - 1));
    std::nth_element(sorted.begin(), sorted.begin() + q, sorted.end());
    const int p90 = sorted[q];
    while (hb.g < 32 && hb.g * kUnroll < p90) hb.g *= 2;
    if (static_cast<int64_t>(M.rows) <= wave_threads)
      while (hb.g > 1 && static_cast<int64_t>(M.rows) * hb.g > wave_threads) hb.g /= 2;
  }
  hb.long_thr = std::max(1, rounds) * kUnroll * hb.g;
  for (int32_t i = 0; i < M.rows; ++i) {
    if (len[i] > kVeryLongRow)
      hb.vlong_rows.push_back(i);
    else if (len[i] > hb.long_thr)
      hb.long_rows.push_back(i);
  }
  return hb;
}

// Warp tiles of consecutive short rows (pdhg_tiled.cuh) over the row ranges
// [off[b], off[b+1]) of the LPs not marked done: at most kTileRows rows and
// kTileEntries entries per tile, never crossing an LP; rows longer than
// kTileRowMax go to the binned long / very-long lists.
struct HostTiles {
  std::vector<int4> tiles;
  std::vector<int32_t> inst;
  std::vector<int32_t> long_rows, vlong_rows;
};

inline HostTiles make_tiles(const std::vector<int32_t>& ptr, const std::vector<int64_t>& off,
                            const std::vector<char>* done) {
  HostTiles h;
  const int K = static_cast<int>(off.size()) - 1;
  for (int b = 0; b < K; ++b) {
    if (done && (*done)[b]) continue;
    int64_t r0 = -1;
    auto close = [&](int64_t r1) {
      if (r0 >= 0 && r1 > r0) {
        h.tiles.push_back(make_int4(static_cast<int>(r0), static_cast<int>(r1), ptr[r0], ptr[r1]));
        h.inst.push_back(b);
      }
      r0 = -1;
    };
    for (int64_t r = off[b]; r < off[b + 1]; ++r) {
      const int32_t len = ptr[r + 1] - ptr[r];
      if (len > kTileRowMax) {
        close(r);
        (len > kVeryLongRow ? h.vlong_rows : h.long_rows).push_back(static_cast<int32_t>(r));
        continue;
      }
      if (r0 >= 0 && (r - r0 + 1 > kTileRows || ptr[r + 1] - ptr[r0] > kTileEntries)) close(r);
      if (r0 < 0) r0 = r;
    }
    close(off[b + 1]);
  }
  return h;
}

template <typename... KArgs, typename... Args>
inline void launch_nt(void (*kern)(KArgs...), unsigned grid, unsigned block, cudaStream_t stream, bool pdl,
                      Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? attr : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  B2P_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

template <typename... KArgs, typename... Args>
inline void launch(void (*kern)(KArgs...), unsigned grid, cudaStream_t stream, bool pdl, Args... args) {
  launch_nt(kern, grid, kBlock, stream, pdl, args...);
}

#define B2P_G_SWITCH(g, F)                           \
  switch (g) {                                       \
    case 1: F(1); break;                             \
    case 2: F(2); break;                             \
    case 4: F(4); break;                             \
    case 8: F(8); break;                             \
    case 16: F(16); break;                           \
    default: F(32); break;                           \
  }

}  // namespace b2p
