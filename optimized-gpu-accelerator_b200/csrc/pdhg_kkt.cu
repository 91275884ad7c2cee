// Relative KKT error of given primal-dual points, on the device.
//
// For each case b, with (x_b, y_b) in the original space of the minimisation
// LP, this is the error runPdhg measures at every check
// (src/pdhg/pdhg.cpp:166-197 and 608-615), written directly in the original
// space (the reference's scaled sums multiplied by beta/R_i, gamma/C_j and
// beta*gamma are exactly these):
//   relP = || dist(A x, [L, U]) ||_2 / (1 + ||(finite L, finite U != L)||_2)
//   relD = || r ||_2 / (1 + ||c||_2),  d = c - A^T y,
//          r_j = |d_j| (free), max(d_j,0) (no lower bound), max(-d_j,0) (no upper bound), 0 (boxed)
//   pobj = c'x;  dobj = sum_i {y_i L_i if y_i > 0, y_i U_i if y_i < 0}
//                     + sum_j {d_j l_j if d_j > 0, d_j u_j if d_j < 0}   (finite bounds only)
//   gap  = |pobj - dobj| / (1 + |pobj| + |dobj|),   kkt = max(relP, relD, gap)
// Row sums of A x and A^T y run left to right (CpuBackend::mult order); the
// block partials are combined in a fixed order, so results are deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pdhg_host_common.h"
#include "pdhg_kernels.cuh"

namespace b2p {

constexpr int kKktRowSums = 3;  // residual^2, row part of dobj, rhs norm^2
constexpr int kKktColSums = 4;  // dual residual^2, pobj, column part of dobj, ||c||^2
constexpr int kKktMaxBlocks = 256;

__device__ __forceinline__ bool finite_bound_d(double v) { return v < 1e20 && v > -1e20; }

// grid = (G, k); partial[(b*G + g)*3 + q]
__global__ void __launch_bounds__(kBlock) k_kkt_point_rows(int32_t m, int32_t n, CsrView A, const double* __restrict__ x,
                                                           const double* __restrict__ y,
                                                           const double* __restrict__ rl,
                                                           const double* __restrict__ ru,
                                                           double* __restrict__ partial) {
  __shared__ double sh[kKktRowSums * (kBlock / 32)];
  const int b = blockIdx.y;
  const double* xb = x + static_cast<int64_t>(b) * n;
  double s[kKktRowSums] = {0, 0, 0};
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = static_cast<int64_t>(b) * m + i;
    const double ax = row_dot(A, xb, i, 1, 0);
    const double l = rl[t], u = ru[t], yv = y[t];
    const bool hl = finite_bound_d(l), hu = finite_bound_d(u);
    double e1 = hl ? l - ax : 0.0, e2 = hu ? ax - u : 0.0;
    e1 = (e1 < 0.0) ? 0.0 : e1;
    e2 = (e2 < 0.0) ? 0.0 : e2;
    const double res = e1 + e2;
    s[0] += res * res;
    if (yv > 0.0 && hl)
      s[1] += yv * l;
    else if (yv < 0.0 && hu)
      s[1] += yv * u;
    if (hl) s[2] += l * l;
    if (hu && u != l) s[2] += u * u;
  }
  block_reduce<kKktRowSums>(s, sh);
  if (threadIdx.x == 0) {
    double* o = partial + (static_cast<int64_t>(b) * gridDim.x + blockIdx.x) * kKktRowSums;
#pragma unroll
    for (int q = 0; q < kKktRowSums; ++q) o[q] = s[q];
  }
}

// AT is A in CSC form read as the CSR of A^T.
__global__ void __launch_bounds__(kBlock) k_kkt_point_cols(int32_t n, int32_t m, CsrView AT, const double* __restrict__ x,
                                                           const double* __restrict__ y, const double* __restrict__ c,
                                                           const double* __restrict__ lo,
                                                           const double* __restrict__ up,
                                                           double* __restrict__ partial) {
  __shared__ double sh[kKktColSums * (kBlock / 32)];
  const int b = blockIdx.y;
  const double* yb = y + static_cast<int64_t>(b) * m;
  double s[kKktColSums] = {0, 0, 0, 0};
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = static_cast<int64_t>(b) * n + j;
    const double aty = row_dot(AT, yb, j, 1, 0);
    const double cv = c[t], l = lo[t], u = up[t];
    const double d = cv - aty;
    const bool hl = finite_bound_d(l), hu = finite_bound_d(u);
    double r = 0.0;
    if (!hl && !hu)
      r = fabs(d);
    else if (!hl)
      r = (d < 0.0) ? 0.0 : d;
    else if (!hu)
      r = (-d < 0.0) ? 0.0 : -d;
    s[0] += r * r;
    s[1] += cv * x[t];
    if (d > 0.0 && hl)
      s[2] += d * l;
    else if (d < 0.0 && hu)
      s[2] += d * u;
    s[3] += cv * cv;
  }
  block_reduce<kKktColSums>(s, sh);
  if (threadIdx.x == 0) {
    double* o = partial + (static_cast<int64_t>(b) * gridDim.x + blockIdx.x) * kKktColSums;
#pragma unroll
    for (int q = 0; q < kKktColSums; ++q) o[q] = s[q];
  }
}

// grid = k: out[b*4 + {0,1,2,3}] = relP, relD, gap, kkt.
__global__ void __launch_bounds__(kBlock) k_kkt_point_finalize(int32_t g_rows, int32_t g_cols,
                                                               const double* __restrict__ prow,
                                                               const double* __restrict__ pcol,
                                                               double* __restrict__ out) {
  __shared__ double sh[(kKktRowSums + kKktColSums) * (kBlock / 32)];
  const int b = blockIdx.x;
  double s[kKktRowSums + kKktColSums] = {0, 0, 0, 0, 0, 0, 0};
  for (int g = threadIdx.x; g < g_rows; g += blockDim.x) {
    const double* p = prow + (static_cast<int64_t>(b) * g_rows + g) * kKktRowSums;
#pragma unroll
    for (int q = 0; q < kKktRowSums; ++q) s[q] += p[q];
  }
  for (int g = threadIdx.x; g < g_cols; g += blockDim.x) {
    const double* p = pcol + (static_cast<int64_t>(b) * g_cols + g) * kKktColSums;
#pragma unroll
    for (int q = 0; q < kKktColSums; ++q) s[kKktRowSums + q] += p[q];
  }
  block_reduce<kKktRowSums + kKktColSums>(s, sh);
  if (threadIdx.x == 0) {
    const double relP = sqrt(s[0]) / (1.0 + sqrt(s[2]));
    const double relD = sqrt(s[3]) / (1.0 + sqrt(s[6]));
    const double pobj = s[4], dobj = s[1] + s[5];
    const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    double kkt = (relD < gap) ? gap : relD;
    kkt = (relP < kkt) ? kkt : relP;
    double* o = out + static_cast<int64_t>(b) * 4;
    o[0] = relP;
    o[1] = relD;
    o[2] = gap;
    o[3] = kkt;
  }
}

inline int kkt_blocks(int64_t len) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(kKktMaxBlocks, (len + kBlock - 1) / kBlock)));
}

// Enqueues the three kernels on `stream`.  A: CSR of A (m rows); AT: CSC of A
// as the CSR of A^T (n rows).  Vectors are case-major (k x n, k x m).
inline void enqueue_kkt(cudaStream_t stream, int32_t m, int32_t n, int32_t k, CsrView A, CsrView AT, const double* x,
                        const double* y, const double* c, const double* lo, const double* up, const double* rl,
                        const double* ru, double* prow, double* pcol, double* out) {
  const int gr = kkt_blocks(m), gc = kkt_blocks(n);
  k_kkt_point_rows<<<dim3(gr, k), kBlock, 0, stream>>>(m, n, A, x, y, rl, ru, prow);
  k_kkt_point_cols<<<dim3(gc, k), kBlock, 0, stream>>>(n, m, AT, x, y, c, lo, up, pcol);
  k_kkt_point_finalize<<<k, kBlock, 0, stream>>>(gr, gc, prow, pcol, out);
}

namespace {

// Device buffers of one call, from the device's stream-ordered pool (freed
// blocks stay cached for the next call; no cudaMalloc / cudaFree per call).
struct DeviceBuffers {
  int dev;
  cudaStream_t stream;
  std::vector<void*> ptrs;
  ~DeviceBuffers() {
    for (void* p : ptrs) cudaFreeAsync(p, stream);
  }
  template <class T>
  T* put(const T* h, size_t count, cudaStream_t s) {
    void* p = nullptr;
    B2P_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(count, 1) * sizeof(T), device_pool(dev), s));
    ptrs.push_back(p);
    if (h && count) B2P_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return static_cast<T*>(p);
  }
};

}  // namespace

}  // namespace b2p

extern "C" int b2p_kkt_residual(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const double* x,
                                const double* row_dual, double* out) {
  using namespace b2p;
  return guarded([&] {
    if (!lp || !x || !row_dual || !out) throw Error(B2P_ERR_INVALID, "NULL argument");
    if (lp->num_rows < 0 || lp->num_cols < 0 || !lp->start || lp->start[0] != 0)
      throw Error(B2P_ERR_INVALID, "bad dimensions or column pointers");
    const int32_t m = lp->num_rows, n = lp->num_cols, nnz = lp->start[n];
    for (int32_t j = 0; j < n; ++j)
      if (lp->start[j + 1] < lp->start[j]) throw Error(B2P_ERR_INVALID, "start must be non-decreasing");
    for (int32_t q = 0; q < nnz; ++q)
      if (lp->index[q] < 0 || lp->index[q] >= m) throw Error(B2P_ERR_INVALID, "row index out of range");
    if (num_cases > 0 && !cases) throw Error(B2P_ERR_INVALID, "cases is NULL");
    const int k = num_cases > 0 ? num_cases : 1;
    // case-major expansion of the per-case vectors
    std::vector<double> c(static_cast<size_t>(k) * n), lo(c.size()), up(c.size()), rl(static_cast<size_t>(k) * m),
        ru(rl.size());
    for (int b = 0; b < k; ++b) {
      const b2p_case* cs = num_cases > 0 ? &cases[b] : nullptr;
      auto pick = [&](const double* v, const double* base) { return (cs && v) ? v : base; };
      const double* cc = pick(cs ? cs->cost : nullptr, lp->col_cost);
      const double* cl = pick(cs ? cs->col_lower : nullptr, lp->col_lower);
      const double* cu = pick(cs ? cs->col_upper : nullptr, lp->col_upper);
      const double* rlo = pick(cs ? cs->row_lower : nullptr, lp->row_lower);
      const double* rup = pick(cs ? cs->row_upper : nullptr, lp->row_upper);
      if (n) {
        std::memcpy(&c[static_cast<size_t>(b) * n], cc, sizeof(double) * n);
        std::memcpy(&lo[static_cast<size_t>(b) * n], cl, sizeof(double) * n);
        std::memcpy(&up[static_cast<size_t>(b) * n], cu, sizeof(double) * n);
      }
      if (m) {
        std::memcpy(&rl[static_cast<size_t>(b) * m], rlo, sizeof(double) * m);
        std::memcpy(&ru[static_cast<size_t>(b) * m], rup, sizeof(double) * m);
      }
    }
    // CSR of A (rows in increasing column order)
    std::vector<int32_t> aptr(static_cast<size_t>(m) + 1, 0), aidx(nnz);
    std::vector<double> aval(nnz);
    for (int32_t q = 0; q < nnz; ++q) aptr[lp->index[q] + 1]++;
    for (int32_t i = 0; i < m; ++i) aptr[i + 1] += aptr[i];
    {
      std::vector<int32_t> pos(aptr.begin(), aptr.end() - 1);
      for (int32_t j = 0; j < n; ++j)
        for (int32_t q = lp->start[j]; q < lp->start[j + 1]; ++q) {
          const int32_t p = pos[lp->index[q]]++;
          aidx[p] = j;
          aval[p] = lp->value[q];
        }
    }
    const int dev = pick_device(-1);
    B2P_CUDA(cudaSetDevice(dev));
    cudaStream_t s = nullptr;
    B2P_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
      cudaStream_t s;
      ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    DeviceBuffers buf{dev, s, {}};
    const CsrView A{buf.put(aptr.data(), aptr.size(), s), buf.put(aidx.data(), aidx.size(), s),
                    buf.put(aval.data(), aval.size(), s), m};
    const CsrView AT{buf.put(lp->start, static_cast<size_t>(n) + 1, s), buf.put(lp->index, nnz, s),
                     buf.put(lp->value, nnz, s), n};
    const double* dx = buf.put(x, static_cast<size_t>(k) * n, s);
    const double* dy = buf.put(row_dual, static_cast<size_t>(k) * m, s);
    const double* dc = buf.put(c.data(), c.size(), s);
    const double* dlo = buf.put(lo.data(), lo.size(), s);
    const double* dup = buf.put(up.data(), up.size(), s);
    const double* drl = buf.put(rl.data(), rl.size(), s);
    const double* dru = buf.put(ru.data(), ru.size(), s);
    double* prow = buf.put<double>(nullptr, static_cast<size_t>(k) * kKktMaxBlocks * kKktRowSums, s);
    double* pcol = buf.put<double>(nullptr, static_cast<size_t>(k) * kKktMaxBlocks * kKktColSums, s);
    double* dout = buf.put<double>(nullptr, static_cast<size_t>(k) * 4, s);
    enqueue_kkt(s, m, n, k, A, AT, dx, dy, dc, dlo, dup, drl, dru, prow, pcol, dout);
    B2P_CUDA(cudaGetLastError());
    B2P_CUDA(cudaMemcpyAsync(out, dout, sizeof(double) * 4 * k, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaStreamSynchronize(s));
  });
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the KKT evaluation.
//
// Some callers cannot allocate device memory: code running inside another
// framework's memory manager (a solver host that owns every device byte
// through its own pool), inside a stream-capture region where cudaMalloc is
// not allowed, or under a hard no-allocation rule on a latency-critical
// path.  For them b2p_kkt_residual_noalloc takes every input and output as a
// caller-owned device pointer and keeps its only scratch -- the per-block
// partial sums of the reductions -- in the file-scope array below, which
// every GPU that loads this library holds until the process exits.
// ---------------------------------------------------------------------------
namespace b2p {

constexpr int kNoAllocMaxPoints = 32;  // points per call
constexpr size_t kNoAllocScratchDoubles =
    static_cast<size_t>(kNoAllocMaxPoints) * kKktMaxBlocks * (kKktRowSums + kKktColSums);  // 458,752 bytes

static __device__ __align__(256) double g_kkt_noalloc_scratch[kNoAllocScratchDoubles];

namespace {

std::mutex g_noalloc_mu;
double* g_noalloc_scratch[64] = {};  // device address of the array, per device ordinal

// Device address of the scratch array on the current device.  The name of a
// __device__ array in host code is only a host-side stand-in, so the address
// is looked up once per device, with that device current.
double* noalloc_scratch_on_current_device() {
  int dev = 0;
  B2P_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Error(B2P_ERR_INVALID, "device ordinal beyond 63");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_scratch[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_kkt_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error(B2P_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                    cudaGetErrorString(e));
    g_noalloc_scratch[dev] = static_cast<double*>(p);
  }
  return g_noalloc_scratch[dev];
}

// Refuses, before anything is launched, an argument that is not device
// memory of the current device: a host pointer (pageable or page-locked), an
// unregistered address, or another GPU's allocation would reach the kernels
// as an illegal address.
void require_device_pointer(const void* p, const char* what, int dev) {
  if (!p) throw Error(B2P_ERR_INVALID, std::string(what) + " is NULL");
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // clears only the error this query itself raised
    throw Error(B2P_ERR_INVALID, std::string(what) + " is not a device pointer");
  }
  if (at.type == cudaMemoryTypeManaged) return;
  if (at.type != cudaMemoryTypeDevice)
    throw Error(B2P_ERR_INVALID, std::string(what) + " is not a device pointer");
  if (at.device != dev)
    throw Error(B2P_ERR_INVALID, std::string(what) + " is memory of device " + std::to_string(at.device) +
                                     ", not of the current device " + std::to_string(dev));
}

}  // namespace
}  // namespace b2p

extern "C" int b2p_kkt_residual_noalloc(int32_t num_rows, int32_t num_cols, int32_t num_points,
                                        const int32_t* a_ptr, const int32_t* a_idx, const double* a_val,
                                        const int32_t* at_ptr, const int32_t* at_idx, const double* at_val,
                                        const double* cost, const double* col_lower, const double* col_upper,
                                        const double* row_lower, const double* row_upper, const double* x,
                                        const double* row_dual, double* out, void* stream) {
  using namespace b2p;
  return guarded([&] {
    if (num_rows < 0 || num_cols < 0) throw Error(B2P_ERR_INVALID, "negative dimension");
    if (num_points < 1) throw Error(B2P_ERR_INVALID, "num_points must be at least 1");
    if (num_points > kNoAllocMaxPoints)
      throw Error(B2P_ERR_TOO_LARGE, "num_points " + std::to_string(num_points) + " exceeds the maximum of " +
                                         std::to_string(kNoAllocMaxPoints) + " points per call");
    int dev = 0;
    B2P_CUDA(cudaGetDevice(&dev));
    // An error left pending by the caller's own earlier work stays the
    // caller's: it is neither reported as this call's nor cleared.
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
      throw Error(B2P_ERR_CUDA, std::string("a CUDA error from earlier work is pending on this thread (") +
                                    cudaGetErrorName(pending) + "); nothing was launched and the error is left in place");
    // every array the kernels can touch: the operators' entries exist only
    // when both dimensions are nonzero
    require_device_pointer(out, "out", dev);
    require_device_pointer(a_ptr, "a_ptr", dev);
    require_device_pointer(at_ptr, "at_ptr", dev);
    if (num_rows > 0 && num_cols > 0) {
      require_device_pointer(a_idx, "a_idx", dev);
      require_device_pointer(a_val, "a_val", dev);
      require_device_pointer(at_idx, "at_idx", dev);
      require_device_pointer(at_val, "at_val", dev);
    }
    if (num_cols > 0) {
      require_device_pointer(cost, "cost", dev);
      require_device_pointer(col_lower, "col_lower", dev);
      require_device_pointer(col_upper, "col_upper", dev);
      require_device_pointer(x, "x", dev);
    }
    if (num_rows > 0) {
      require_device_pointer(row_lower, "row_lower", dev);
      require_device_pointer(row_upper, "row_upper", dev);
      require_device_pointer(row_dual, "row_dual", dev);
    }
    double* scratch = noalloc_scratch_on_current_device();
    double* prow = scratch;
    double* pcol = scratch + static_cast<size_t>(kNoAllocMaxPoints) * kKktMaxBlocks * kKktRowSums;
    const CsrView A{a_ptr, a_idx, a_val, num_rows};
    const CsrView AT{at_ptr, at_idx, at_val, num_cols};
    enqueue_kkt(static_cast<cudaStream_t>(stream), num_rows, num_cols, num_points, A, AT, x, row_dual, cost,
                col_lower, col_upper, row_lower, row_upper, prow, pcol, out);
    // nothing was pending before the launches, so an error now is theirs
    B2P_CUDA(cudaGetLastError());
  });
}
