// Roofline probe of the CSR SpMV on one large random operator (measurement
// tool, not part of the library): the engine's binned kernel
// (k_spmv_binned, 4 lanes per row) and warp-tile kernel (k_spmv_tiled) against
// two ceilings measured on the same data --
//   gathers only : sum of x[idx[e]] over every entry (the random operand
//                  reads alone: one 32-byte L2 sector per 8-byte operand);
//   stream       : a coalesced read of the index and value arrays (HBM).
// Usage: spmv_roofline [entries per row, default 12.8]
// The operator has 2.6M rows and 5.2M columns with Poisson row lengths capped
// at 32 and uniformly random columns (the structure of the config-2
// generator's A at the scale of a 64-LP uneven batch).
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "pdhg_sched.h"

using namespace b2p;

namespace {

__global__ void k_gathers_only(const int32_t* __restrict__ idx, int64_t n, const double* __restrict__ x,
                               double* out) {
  double s = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    s += __ldcg(x + __ldcs(idx + i));
  if (s == 12345.678) out[0] = s;  // keeps the loads alive
}

__global__ void k_stream(const int32_t* __restrict__ idx, const double* __restrict__ val, int64_t n, double* out) {
  double s = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    s += __ldcs(val + i) + __ldcs(idx + i);
  if (s == 12345.678) out[0] = s;
}

#define CHECK(call)                                                               \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      std::fprintf(stderr, "%s: %s\n", #call, cudaGetErrorString(e_));            \
      std::exit(1);                                                               \
    }                                                                             \
  } while (0)

}  // namespace

int main(int argc, char** argv) {
  const int m = 2600000, n = 5200000;
  const double per = argc > 1 ? std::atof(argv[1]) : 12.8;
  std::mt19937_64 rng(7);
  std::poisson_distribution<int> pois(per);
  std::vector<int32_t> ptr(static_cast<size_t>(m) + 1, 0), idx;
  std::vector<double> val;
  for (int i = 0; i < m; ++i) {
    const int len = std::min(pois(rng), 32);
    for (int k = 0; k < len; ++k) {
      idx.push_back(static_cast<int32_t>(rng() % n));
      val.push_back(1.0 + static_cast<double>(rng() % 100) * 0.01);
    }
    ptr[i + 1] = ptr[i] + len;
  }
  const int64_t nnz = ptr[m];
  int32_t *dp, *di;
  double *dv, *dx, *dy;
  CHECK(cudaMalloc(&dp, sizeof(int32_t) * (m + 1)));
  CHECK(cudaMalloc(&di, sizeof(int32_t) * (nnz + kTilePad)));
  CHECK(cudaMalloc(&dv, sizeof(double) * (nnz + kTilePad)));
  CHECK(cudaMalloc(&dx, sizeof(double) * n));
  CHECK(cudaMalloc(&dy, sizeof(double) * m));
  CHECK(cudaMemcpy(dp, ptr.data(), sizeof(int32_t) * (m + 1), cudaMemcpyHostToDevice));
  CHECK(cudaMemcpy(di, idx.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice));
  CHECK(cudaMemcpy(dv, val.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice));
  std::vector<double> hx(n, 1.0);
  CHECK(cudaMemcpy(dx, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  const CsrView M{dp, di, dv, m};
  const InstanceMap im{nullptr, nullptr};

  // warp tiles (every row here is short)
  const std::vector<int64_t> off{0, m};
  const HostTiles ht = make_tiles(ptr, off, nullptr);
  int4* dt;
  CHECK(cudaMalloc(&dt, sizeof(int4) * ht.tiles.size()));
  CHECK(cudaMemcpy(dt, ht.tiles.data(), sizeof(int4) * ht.tiles.size(), cudaMemcpyHostToDevice));
  TileSet ts{dt, nullptr, static_cast<int32_t>(ht.tiles.size()), 0};
  ts.grid = (ts.n_tiles + kBlock / 32 - 1) / (kBlock / 32);

  // binned schedule, 4 lanes per row (rows of up to 32 entries stay on the short path)
  HostCsr H;
  H.rows = m;
  H.cols = n;
  H.ptr = ptr;
  const HostBins hb = make_bins(H, int64_t(1) << 40, 4, 2);
  RowBins rb{};
  rb.long_thr = hb.long_thr;
  rb.short_blocks = static_cast<int32_t>((static_cast<int64_t>(m) * hb.g + kBlock - 1) / kBlock);
  rb.g = hb.g;

  int sms = 0;
  CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
  const double spmv_bytes = 12.0 * nnz + 4.0 * (m + 1) + 8.0 * n + 8.0 * m;
  std::printf("operator: %d rows, %d cols, %lld nonzeros (%.1f per row); SpMV bytes %.0f MB; warp tiles %d\n", m, n,
              static_cast<long long>(nnz), static_cast<double>(nnz) / m, spmv_bytes / 1e6, ts.n_tiles);
  cudaEvent_t a, b;
  CHECK(cudaEventCreate(&a));
  CHECK(cudaEventCreate(&b));
  auto timeit = [&](const char* name, double bytes, auto&& f) {
    for (int w = 0; w < 3; ++w) f();
    CHECK(cudaEventRecord(a));
    for (int r = 0; r < 10; ++r) f();
    CHECK(cudaEventRecord(b));
    CHECK(cudaEventSynchronize(b));
    CHECK(cudaGetLastError());
    float ms = 0;
    CHECK(cudaEventElapsedTime(&ms, a, b));
    ms /= 10;
    std::printf("%-34s %8.1f us  %6.0f GB/s\n", name, ms * 1e3, bytes / (ms * 1e-3) / 1e9);
  };
  timeit("k_spmv_binned (4 lanes/row)", spmv_bytes,
         [&] { k_spmv_binned<4, false><<<rb.short_blocks, kBlock>>>(M, rb, dx, dy, im); });
  const RowBins no_long{};  // every row here is short: no leading long-row blocks
  timeit("k_spmv_tiled (warp tiles)", spmv_bytes,
         [&] { k_spmv_tiled<false><<<ts.grid, kBlock>>>(M, ts, no_long, dx, dy, im); });
  timeit("gathers only: x[idx[e]]", spmv_bytes, [&] { k_gathers_only<<<sms * 8, 256>>>(di, nnz, dx, dy); });
  timeit("stream: idx + val", 12.0 * nnz, [&] { k_stream<<<sms * 8, 256>>>(di, dv, nnz, dy); });
  return 0;
}
