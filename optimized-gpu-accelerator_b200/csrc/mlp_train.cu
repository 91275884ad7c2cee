// The learned warm-start network: forward, loss, backward and Adam kernels
// around the tcgen05 BF16 GEMM (mlp_gemm.cuh), and the C ABI of
// include/b2p_mlp.h.  Every reduction runs in a fixed order, so training is
// deterministic for a given seed.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <random>
#include <vector>

#include "../../include/b2p_mlp.h"
#include "mlp_gemm.cuh"
#include "pdhg_host_common.h"

namespace b2p {
namespace {

constexpr int kEw = 256;  // threads of the elementwise kernels
constexpr int kLossBlocks = 148;

inline int ew_blocks(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + kEw - 1) / kEw, 148 * 16))); }

// minibatch rows r <- samples perm[offset + r]: FP32 inputs to BF16, targets copied
__global__ void k_gather(int32_t rows, int32_t din, int32_t dout, const float* __restrict__ x,
                         const float* __restrict__ y, const int32_t* __restrict__ perm, int64_t offset,
                         __nv_bfloat16* __restrict__ xb, float* __restrict__ yt) {
  const int64_t nin = static_cast<int64_t>(rows) * din, nout = static_cast<int64_t>(rows) * dout;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < nin + nout;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (e < nin) {
      const int64_t r = e / din, c = e % din;
      const int64_t s = perm ? perm[offset + r] : offset + r;
      xb[e] = __float2bfloat16(x[s * din + c]);
    } else if (yt) {
      const int64_t f = e - nin, r = f / dout, c = f % dout;
      const int64_t s = perm ? perm[offset + r] : offset + r;
      yt[f] = y[s * dout + c];
    }
  }
}

// d = out - target; G = d / rows (FP32 and BF16); per-block sums of d^2
__global__ void __launch_bounds__(kEw) k_mse_grad(int64_t count, float inv_rows, const float* __restrict__ out,
                                                  const float* __restrict__ target, float* __restrict__ gf,
                                                  __nv_bfloat16* __restrict__ gb, double* __restrict__ partial) {
  double s = 0.0;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(kEw) + threadIdx.x; e < count;
       e += static_cast<int64_t>(gridDim.x) * kEw) {
    const float d = out[e] - target[e];
    const float gv = d * inv_rows;
    gf[e] = gv;
    gb[e] = __float2bfloat16(gv);
    s += static_cast<double>(d) * static_cast<double>(d);
  }
  __shared__ double red[kEw];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kEw / 2; w > 0; w >>= 1) {
    if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// loss = 0.5 * sum(partials) / rows; stored to *loss and added, times
// `weight`, to *accum (the epoch mean)
__global__ void k_loss_finish(int32_t nblocks, const double* __restrict__ partial, double inv_rows, double* loss,
                              double* accum, double weight) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < nblocks; ++i) s += partial[i];
  const double l = 0.5 * s * inv_rows;
  if (loss) *loss = l;
  if (accum) *accum += l * weight;
}

// bias gradient: db[c] = sum_r G[r, c] (rows summed in order)
__global__ void k_colsum(int32_t rows, int32_t cols, const float* __restrict__ g, float* __restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += g[static_cast<int64_t>(r) * cols + c];
  db[c] = s;
}

// Adam (decoupled weight decay on the entries flagged in `decay`), then the
// BF16 copy of the parameters
__global__ void k_adam(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, const uint8_t* __restrict__ decay, float lr, float b1, float b2,
                       float c1, float c2, float eps, float wd, __nv_bfloat16* __restrict__ pb) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi * c1, vh = vi * c2;
    float pi = p[i] - lr * (mh / (sqrtf(vh) + eps));
    if (wd > 0.0f && decay[i]) pi -= lr * wd * p[i];
    p[i] = pi;
    pb[i] = __float2bfloat16(pi);
  }
}

__global__ void k_to_bf16(int64_t n, const float* __restrict__ src, __nv_bfloat16* __restrict__ dst) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = __float2bfloat16(src[i]);
}

int gemm_sms[64] = {};  // SM count per device, set with the attributes

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); NULL if the driver does not offer it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor map of a K-contiguous operand X(r, k) = X[r * sr + k], r < R,
// k < K: 64 x box_rows boxes, 128-byte swizzle, zeros past the edges.
bool encode_operand(CUtensorMap* map, const __nv_bfloat16* X, int64_t sr, int R, int K, int box_rows) {
  const auto fn = tensor_map_encoder();
  if (!fn) return false;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(K), static_cast<cuuint64_t>(R)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(sr) * 2};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(kGemmBK), static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(X), dims, strides, box, elem,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The TMA form applies when both operands are K-contiguous with rows of a
// multiple of 16 bytes on a 16-byte aligned base (the tensor map's rules).
bool gemm_tma_ok(const GemmArgs& g) {
  auto ok = [&](const void* X, int64_t sr, int64_t sk) {
    return sk == 1 && sr >= g.K && sr % 8 == 0 && sr < (int64_t{1} << 38) &&
           (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  };
  return g.K > 0 && ok(g.A, g.sam, g.sak) && ok(g.B, g.sbn, g.sbk);
}

void set_gemm_attributes() {
  static std::once_flag once[64];
  int dev = 0;
  B2P_CUDA(cudaGetDevice(&dev));
  cudaError_t err = cudaSuccess;
  std::call_once(once[dev & 63], [&] {
    err = cudaFuncSetAttribute(k_gemm_bf16_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               GemmTile<128>::kSmemBytes);
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_gemm_bf16_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 GemmTile<256>::kSmemBytes);
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_gemm_bf16_tma<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 GemmTmaTile<128>::kSmemBytes);
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_gemm_bf16_tma<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 GemmTmaTile<256>::kSmemBytes);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&gemm_sms[dev & 63], cudaDevAttrMultiProcessorCount, dev);
  });
  B2P_CUDA(err);
}

// 128 x 256 tiles when they still give every SM a CTA, else 128 x 128
// (the network's small GEMMs need the wider grid); the TMA form when both
// operands are K-contiguous, the cp.async form otherwise.
void launch_gemm(const GemmArgs& g, cudaStream_t stream) {
  if (g.M <= 0 || g.N <= 0) return;
  int dev = 0;
  B2P_CUDA(cudaGetDevice(&dev));
  const int64_t mt = (g.M + kGemmBM - 1) / kGemmBM;
  const int sms = gemm_sms[dev & 63];
  const bool wide = sms > 0 && mt * ((g.N + 255) / 256) >= sms;
  if (sms > 0 && gemm_tma_ok(g)) {
    CUtensorMap ma, mb;
    if (encode_operand(&ma, g.A, g.sam, g.M, g.K, kGemmBM) && encode_operand(&mb, g.B, g.sbn, g.N, g.K, wide ? 256 : 128)) {
      if (wide) {
        const dim3 grid(static_cast<unsigned>(mt), (g.N + 255) / 256);
        k_gemm_bf16_tma<256><<<grid, kGemmThreads, GemmTmaTile<256>::kSmemBytes, stream>>>(ma, mb, g);
      } else {
        const dim3 grid(static_cast<unsigned>(mt), (g.N + 127) / 128);
        k_gemm_bf16_tma<128><<<grid, kGemmThreads, GemmTmaTile<128>::kSmemBytes, stream>>>(ma, mb, g);
      }
      B2P_CUDA(cudaGetLastError());
      return;
    }
  }
  if (wide) {
    const dim3 grid(static_cast<unsigned>(mt), (g.N + 255) / 256);
    k_gemm_bf16_tc<256><<<grid, kGemmThreads, GemmTile<256>::kSmemBytes, stream>>>(g);
  } else {
    const dim3 grid(static_cast<unsigned>(mt), (g.N + 127) / 128);
    k_gemm_bf16_tc<128><<<grid, kGemmThreads, GemmTile<128>::kSmemBytes, stream>>>(g);
  }
  B2P_CUDA(cudaGetLastError());
}

template <class T>
T* dalloc(size_t count) {
  void* p = nullptr;
  if (count) B2P_CUDA(cudaMalloc(&p, count * sizeof(T)));
  return static_cast<T*>(p);
}

struct Mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<int32_t> w;  // widths, L + 1 entries
  int L = 0;
  int32_t max_batch = 0;
  int64_t nparams = 0;
  std::vector<int64_t> woff, boff;
  int64_t step = 0;
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  uint8_t* decay = nullptr;
  __nv_bfloat16* pbf = nullptr;               // BF16 copy of params
  std::vector<__nv_bfloat16*> act;            // act[l]: max_batch x w[l], l = 0 .. L-1
  float* out = nullptr;                       // max_batch x w[L]
  float* target = nullptr;                    // max_batch x w[L]
  float *gf[2] = {nullptr, nullptr};          // gradient ping-pong, max_batch x max width
  __nv_bfloat16* gb[2] = {nullptr, nullptr};
  double* partial = nullptr;                  // kLossBlocks
  double* d_loss = nullptr;                   // [0] last loss, [1..] epoch sums
  int32_t* d_error = nullptr;
  std::vector<void*> owned;

  ~Mlp() {
    if (device >= 0) cudaSetDevice(device);
    for (void* p : owned) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }

  template <class T>
  T* alloc(size_t count) {
    T* p = dalloc<T>(count);
    if (p) owned.push_back(p);
    return p;
  }

  void create(const int32_t* widths, int32_t layers, int32_t mb, int32_t dev) {
    if (!widths || layers < 1) throw Error(B2P_ERR_INVALID, "network needs at least one layer");
    if (mb < 1) throw Error(B2P_ERR_INVALID, "max_batch must be positive");
    device = pick_device(dev);
    B2P_CUDA(cudaSetDevice(device));
    B2P_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    L = layers;
    max_batch = mb;
    w.assign(widths, widths + layers + 1);
    int32_t wmax = 0;
    for (int32_t x : w) {
      if (x < 8 || x % 8 != 0 || x > 65536) throw Error(B2P_ERR_INVALID, "every width must be a multiple of 8");
      wmax = std::max(wmax, x);
    }
    woff.resize(L);
    boff.resize(L);
    for (int l = 0; l < L; ++l) {
      woff[l] = nparams;
      nparams += static_cast<int64_t>(w[l + 1]) * w[l];
      boff[l] = nparams;
      nparams += w[l + 1];
    }
    params = alloc<float>(nparams);
    grads = alloc<float>(nparams);
    adam_m = alloc<float>(nparams);
    adam_v = alloc<float>(nparams);
    pbf = alloc<__nv_bfloat16>(nparams);
    decay = alloc<uint8_t>(nparams);
    B2P_CUDA(cudaMemsetAsync(params, 0, sizeof(float) * nparams, stream));
    B2P_CUDA(cudaMemsetAsync(pbf, 0, sizeof(__nv_bfloat16) * nparams, stream));
    std::vector<uint8_t> hd(nparams, 0);
    for (int l = 0; l < L; ++l) std::fill(hd.begin() + woff[l], hd.begin() + boff[l], uint8_t(1));
    B2P_CUDA(cudaMemcpyAsync(decay, hd.data(), nparams, cudaMemcpyHostToDevice, stream));
    act.resize(L);
    for (int l = 0; l < L; ++l) act[l] = alloc<__nv_bfloat16>(static_cast<size_t>(mb) * w[l]);
    out = alloc<float>(static_cast<size_t>(mb) * w[L]);
    target = alloc<float>(static_cast<size_t>(mb) * w[L]);
    for (int i = 0; i < 2; ++i) {
      gf[i] = alloc<float>(static_cast<size_t>(mb) * wmax);
      gb[i] = alloc<__nv_bfloat16>(static_cast<size_t>(mb) * wmax);
    }
    partial = alloc<double>(kLossBlocks);
    d_error = alloc<int32_t>(1);
    B2P_CUDA(cudaMemsetAsync(d_error, 0, sizeof(int32_t), stream));
    set_gemm_attributes();
    reset_moments();
    B2P_CUDA(cudaStreamSynchronize(stream));
  }

  void reset_moments() {
    B2P_CUDA(cudaMemsetAsync(adam_m, 0, sizeof(float) * nparams, stream));
    B2P_CUDA(cudaMemsetAsync(adam_v, 0, sizeof(float) * nparams, stream));
    step = 0;
  }

  GemmArgs gemm_base() const {
    GemmArgs g{};
    g.alpha = 1.0f;
    g.error = d_error;
    return g;
  }

  // forward on rows of act[0]; result in `y` (FP32, rows x w[L])
  void forward(int32_t rows, float* y, cudaStream_t s) {
    for (int l = 0; l < L; ++l) {
      GemmArgs g = gemm_base();
      g.M = rows;
      g.N = w[l + 1];
      g.K = w[l];
      g.A = act[l];
      g.sam = w[l];
      g.sak = 1;
      g.B = pbf + woff[l];
      g.sbk = 1;
      g.sbn = w[l];
      g.bias = params + boff[l];
      if (l + 1 < L) {
        g.relu = 1;
        g.cb = act[l + 1];
        g.ldcb = w[l + 1];
      } else {
        g.cf = y;
        g.ldcf = w[L];
      }
      launch_gemm(g, s);
    }
  }

  // loss of the forward output `out` against `target`, then all gradients
  void loss_backward(int32_t rows, double* accum, double weight) {
    const int64_t cnt = static_cast<int64_t>(rows) * w[L];
    const int nb = static_cast<int>(std::min<int64_t>(kLossBlocks, (cnt + kEw - 1) / kEw));
    k_mse_grad<<<nb, kEw, 0, stream>>>(cnt, 1.0f / static_cast<float>(rows), out, target, gf[0], gb[0], partial);
    B2P_CUDA(cudaGetLastError());
    k_loss_finish<<<1, 32, 0, stream>>>(nb, partial, 1.0 / rows, d_loss, accum, weight);
    B2P_CUDA(cudaGetLastError());
    int cur = 0;
    for (int l = L - 1; l >= 0; --l) {
      const int32_t wo = w[l + 1], wi = w[l];
      // dW_l = G^T h_l  (wo x wi, K = rows)
      GemmArgs g = gemm_base();
      g.M = wo;
      g.N = wi;
      g.K = rows;
      g.A = gb[cur];
      g.sam = 1;
      g.sak = wo;
      g.B = act[l];
      g.sbk = wi;
      g.sbn = 1;
      g.cf = grads + woff[l];
      g.ldcf = wi;
      launch_gemm(g, stream);
      k_colsum<<<(wo + kEw - 1) / kEw, kEw, 0, stream>>>(rows, wo, gf[cur], grads + boff[l]);
      B2P_CUDA(cudaGetLastError());
      if (l > 0) {
        // G_{l-1} = (G W_l) masked by relu'(h_l)  (rows x wi, K = wo)
        GemmArgs h = gemm_base();
        h.M = rows;
        h.N = wi;
        h.K = wo;
        h.A = gb[cur];
        h.sam = wo;
        h.sak = 1;
        h.B = pbf + woff[l];
        h.sbk = wi;
        h.sbn = 1;
        h.mask = act[l];
        h.ldm = wi;
        h.cf = gf[cur ^ 1];
        h.ldcf = wi;
        h.cb = gb[cur ^ 1];
        h.ldcb = wi;
        launch_gemm(h, stream);
        cur ^= 1;
      }
    }
  }

  void check_error() {
    int32_t h = 0;
    B2P_CUDA(cudaMemcpyAsync(&h, d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaStreamSynchronize(stream));
    if (h) throw Error(B2P_ERR_CUDA, "tensor-core GEMM: mbarrier wait timed out");
  }

  void set_params(const float* hp) {
    B2P_CUDA(cudaSetDevice(device));
    B2P_CUDA(cudaMemcpyAsync(params, hp, sizeof(float) * nparams, cudaMemcpyHostToDevice, stream));
    k_to_bf16<<<ew_blocks(nparams), kEw, 0, stream>>>(nparams, params, pbf);
    B2P_CUDA(cudaGetLastError());
    reset_moments();
    B2P_CUDA(cudaStreamSynchronize(stream));
  }

  void get_params(float* hp) {
    B2P_CUDA(cudaSetDevice(device));
    B2P_CUDA(cudaMemcpyAsync(hp, params, sizeof(float) * nparams, cudaMemcpyDeviceToHost, stream));
    B2P_CUDA(cudaStreamSynchronize(stream));
  }

  void forward_host(const float* x, int64_t batch, float* y) {
    B2P_CUDA(cudaSetDevice(device));
    if (batch < 0) throw Error(B2P_ERR_INVALID, "negative batch");
    float* dx = alloc_scratch_x(batch);
    float* dy = dalloc<float>(static_cast<size_t>(batch) * w[L]);
    try {
      if (batch) {
        B2P_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * batch * w[0], cudaMemcpyHostToDevice, stream));
        forward_dev(dx, batch, dy, stream);
        B2P_CUDA(cudaMemcpyAsync(y, dy, sizeof(float) * batch * w[L], cudaMemcpyDeviceToHost, stream));
      }
      check_error();
    } catch (...) {
      cudaFree(dx);
      cudaFree(dy);
      throw;
    }
    cudaFree(dx);
    cudaFree(dy);
  }

  float* alloc_scratch_x(int64_t batch) { return dalloc<float>(static_cast<size_t>(batch) * w[0]); }

  // chunks of max_batch rows through the activation buffers
  void forward_dev(const float* dx, int64_t batch, float* dy, cudaStream_t s) {
    for (int64_t r0 = 0; r0 < batch; r0 += max_batch) {
      const int32_t rows = static_cast<int32_t>(std::min<int64_t>(max_batch, batch - r0));
      k_gather<<<ew_blocks(static_cast<int64_t>(rows) * w[0]), kEw, 0, s>>>(rows, w[0], w[L], dx, nullptr, nullptr,
                                                                            r0, act[0], nullptr);
      B2P_CUDA(cudaGetLastError());
      forward(rows, dy + r0 * w[L], s);
    }
  }

  void loss_grad(const float* x, const float* y, int32_t batch, double* loss, float* grad) {
    B2P_CUDA(cudaSetDevice(device));
    if (batch < 1 || batch > max_batch) throw Error(B2P_ERR_INVALID, "batch must be in [1, max_batch]");
    float* dx = dalloc<float>(static_cast<size_t>(batch) * w[0]);
    float* dy = dalloc<float>(static_cast<size_t>(batch) * w[L]);
    double* dl = dalloc<double>(1);
    try {
      B2P_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * batch * w[0], cudaMemcpyHostToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(dy, y, sizeof(float) * batch * w[L], cudaMemcpyHostToDevice, stream));
      k_gather<<<ew_blocks(static_cast<int64_t>(batch) * (w[0] + w[L])), kEw, 0, stream>>>(batch, w[0], w[L], dx, dy,
                                                                                           nullptr, 0, act[0], target);
      B2P_CUDA(cudaGetLastError());
      forward(batch, out, stream);
      d_loss = dl;
      loss_backward(batch, nullptr, 0.0);
      double hl = 0;
      B2P_CUDA(cudaMemcpyAsync(&hl, dl, sizeof(double), cudaMemcpyDeviceToHost, stream));
      if (grad) B2P_CUDA(cudaMemcpyAsync(grad, grads, sizeof(float) * nparams, cudaMemcpyDeviceToHost, stream));
      check_error();
      if (loss) *loss = hl;
    } catch (...) {
      cudaFree(dx);
      cudaFree(dy);
      cudaFree(dl);
      d_loss = nullptr;
      throw;
    }
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dl);
    d_loss = nullptr;
  }

  void train(const float* x, const float* y, int64_t count, const b2p_mlp_train_options& o, float* epoch_loss) {
    B2P_CUDA(cudaSetDevice(device));
    if (count < 1) throw Error(B2P_ERR_INVALID, "no training samples");
    if (o.epochs < 0 || o.batch < 1 || o.batch > max_batch) throw Error(B2P_ERR_INVALID, "bad epochs / batch");
    if (count > INT32_MAX) throw Error(B2P_ERR_TOO_LARGE, "too many samples");
    const int32_t bs = static_cast<int32_t>(std::min<int64_t>(o.batch, count));
    const int64_t steps_per_epoch = count / bs;
    const int64_t total = steps_per_epoch * o.epochs;
    float* dx = dalloc<float>(static_cast<size_t>(count) * w[0]);
    float* dy = dalloc<float>(static_cast<size_t>(count) * w[L]);
    int32_t* dperm = dalloc<int32_t>(static_cast<size_t>(count));
    double* dl = dalloc<double>(1 + std::max(o.epochs, 1));
    auto release = [&] {
      cudaFree(dx);
      cudaFree(dy);
      cudaFree(dperm);
      cudaFree(dl);
      d_loss = nullptr;
    };
    try {
      B2P_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * count * w[0], cudaMemcpyHostToDevice, stream));
      B2P_CUDA(cudaMemcpyAsync(dy, y, sizeof(float) * count * w[L], cudaMemcpyHostToDevice, stream));
      B2P_CUDA(cudaMemsetAsync(dl, 0, sizeof(double) * (1 + std::max(o.epochs, 1)), stream));
      d_loss = dl;
      std::mt19937_64 rng(o.seed);
      std::vector<int32_t> perm(count);
      int64_t t = 0;
      for (int ep = 0; ep < o.epochs; ++ep) {
        std::iota(perm.begin(), perm.end(), 0);
        std::shuffle(perm.begin(), perm.end(), rng);
        B2P_CUDA(cudaMemcpyAsync(dperm, perm.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, stream));
        for (int64_t sidx = 0; sidx < steps_per_epoch; ++sidx, ++t) {
          k_gather<<<ew_blocks(static_cast<int64_t>(bs) * (w[0] + w[L])), kEw, 0, stream>>>(
              bs, w[0], w[L], dx, dy, dperm, sidx * bs, act[0], target);
          B2P_CUDA(cudaGetLastError());
          forward(bs, out, stream);
          loss_backward(bs, dl + 1 + ep, 1.0 / static_cast<double>(steps_per_epoch));
          ++step;
          const double frac = total > 1 ? static_cast<double>(t) / static_cast<double>(total - 1) : 1.0;
          const double lr = o.lr_final + 0.5 * (o.lr - o.lr_final) * (1.0 + std::cos(M_PI * frac));
          const double c1 = 1.0 / (1.0 - std::pow(static_cast<double>(o.beta1), static_cast<double>(step)));
          const double c2 = 1.0 / (1.0 - std::pow(static_cast<double>(o.beta2), static_cast<double>(step)));
          k_adam<<<ew_blocks(nparams), kEw, 0, stream>>>(nparams, params, grads, adam_m, adam_v, decay,
                                                         static_cast<float>(lr), o.beta1, o.beta2,
                                                         static_cast<float>(c1), static_cast<float>(c2), o.eps,
                                                         o.weight_decay, pbf);
          B2P_CUDA(cudaGetLastError());
        }
      }
      std::vector<double> hl(1 + std::max(o.epochs, 1));
      B2P_CUDA(cudaMemcpyAsync(hl.data(), dl, sizeof(double) * hl.size(), cudaMemcpyDeviceToHost, stream));
      check_error();
      if (epoch_loss)
        for (int ep = 0; ep < o.epochs; ++ep) epoch_loss[ep] = static_cast<float>(hl[1 + ep]);
    } catch (...) {
      release();
      throw;
    }
    release();
  }
};

Mlp* as_mlp(b2p_mlp* h) {
  if (!h) throw Error(B2P_ERR_INVALID, "network is NULL");
  return reinterpret_cast<Mlp*>(h);
}

}  // namespace
}  // namespace b2p

using namespace b2p;

extern "C" {

b2p_mlp_train_options b2p_mlp_default_train_options(void) {
  b2p_mlp_train_options o{};
  o.epochs = 200;
  o.batch = 512;
  o.lr = 1e-3f;
  o.lr_final = 1e-5f;
  o.beta1 = 0.9f;
  o.beta2 = 0.999f;
  o.eps = 1e-8f;
  o.weight_decay = 0.0f;
  o.seed = 0;
  return o;
}

int b2p_mlp_create(const int32_t* widths, int32_t num_layers, int32_t max_batch, int32_t device, b2p_mlp** out) {
  return guarded([&] {
    if (!out) throw Error(B2P_ERR_INVALID, "out is NULL");
    *out = nullptr;
    Mlp* m = new Mlp();
    try {
      m->create(widths, num_layers, max_batch, device);
    } catch (...) {
      delete m;
      throw;
    }
    *out = reinterpret_cast<b2p_mlp*>(m);
  });
}

int b2p_mlp_destroy(b2p_mlp* net) {
  return guarded([&] { delete reinterpret_cast<Mlp*>(net); });
}

int b2p_mlp_num_params(const b2p_mlp* net, int64_t* count) {
  return guarded([&] {
    if (!net || !count) throw Error(B2P_ERR_INVALID, "NULL argument");
    *count = reinterpret_cast<const Mlp*>(net)->nparams;
  });
}

int b2p_mlp_set_params(b2p_mlp* net, const float* params) {
  return guarded([&] {
    if (!params) throw Error(B2P_ERR_INVALID, "params is NULL");
    as_mlp(net)->set_params(params);
  });
}

int b2p_mlp_get_params(b2p_mlp* net, float* params) {
  return guarded([&] {
    if (!params) throw Error(B2P_ERR_INVALID, "params is NULL");
    as_mlp(net)->get_params(params);
  });
}

int b2p_mlp_forward(b2p_mlp* net, const float* x, int64_t batch, float* y) {
  return guarded([&] {
    if ((!x || !y) && batch > 0) throw Error(B2P_ERR_INVALID, "NULL buffer");
    as_mlp(net)->forward_host(x, batch, y);
  });
}

int b2p_mlp_forward_device(b2p_mlp* net, const float* x, int64_t batch, float* y, void* stream) {
  return guarded([&] {
    Mlp* m = as_mlp(net);
    if ((!x || !y) && batch > 0) throw Error(B2P_ERR_INVALID, "NULL buffer");
    if (batch < 0) throw Error(B2P_ERR_INVALID, "negative batch");
    B2P_CUDA(cudaSetDevice(m->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : m->stream;
    // the activation buffers belong to the network's stream: order the caller's stream after it
    if (s != m->stream) {
      cudaEvent_t ev;
      B2P_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      B2P_CUDA(cudaEventRecord(ev, m->stream));
      B2P_CUDA(cudaStreamWaitEvent(s, ev, 0));
      B2P_CUDA(cudaEventDestroy(ev));
    }
    m->forward_dev(x, batch, y, s);
    if (s != m->stream) {
      cudaEvent_t ev;
      B2P_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      B2P_CUDA(cudaEventRecord(ev, s));
      B2P_CUDA(cudaStreamWaitEvent(m->stream, ev, 0));
      B2P_CUDA(cudaEventDestroy(ev));
    }
  });
}

int b2p_mlp_loss_grad(b2p_mlp* net, const float* x, const float* target, int32_t batch, double* loss, float* grad) {
  return guarded([&] {
    if (!x || !target) throw Error(B2P_ERR_INVALID, "NULL buffer");
    as_mlp(net)->loss_grad(x, target, batch, loss, grad);
  });
}

int b2p_mlp_train(b2p_mlp* net, const float* x, const float* target, int64_t count,
                  const b2p_mlp_train_options* opts, float* epoch_loss) {
  return guarded([&] {
    if (!x || !target) throw Error(B2P_ERR_INVALID, "NULL buffer");
    const b2p_mlp_train_options o = opts ? *opts : b2p_mlp_default_train_options();
    as_mlp(net)->train(x, target, count, o, epoch_loss);
  });
}

int b2p_mlp_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* A, int64_t sam, int64_t sak,
                      const uint16_t* B, int64_t sbk, int64_t sbn, float alpha, const float* bias, int32_t relu,
                      const uint16_t* mask, int64_t ldm, float* cf, int64_t ldcf, uint16_t* cb, int64_t ldcb,
                      void* stream) {
  return guarded([&] {
    if (M < 0 || N < 0 || K < 0) throw Error(B2P_ERR_INVALID, "negative size");
    if ((!A || !B) && K > 0) throw Error(B2P_ERR_INVALID, "NULL operand");
    if (!cf && !cb) throw Error(B2P_ERR_INVALID, "no output");
    int dev = 0;
    B2P_CUDA(cudaGetDevice(&dev));
    int major = 0;
    B2P_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) throw Error(B2P_ERR_NO_DEVICE, "tcgen05 GEMM needs an sm_100 device");
    set_gemm_attributes();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int32_t* derr = dalloc<int32_t>(1);
    try {
      B2P_CUDA(cudaMemsetAsync(derr, 0, sizeof(int32_t), s));
      GemmArgs g{};
      g.M = M;
      g.N = N;
      g.K = K;
      g.A = reinterpret_cast<const __nv_bfloat16*>(A);
      g.sam = sam;
      g.sak = sak;
      g.B = reinterpret_cast<const __nv_bfloat16*>(B);
      g.sbk = sbk;
      g.sbn = sbn;
      g.alpha = alpha;
      g.bias = bias;
      g.relu = relu;
      g.mask = reinterpret_cast<const __nv_bfloat16*>(mask);
      g.ldm = ldm;
      g.cf = cf;
      g.ldcf = ldcf;
      g.cb = reinterpret_cast<__nv_bfloat16*>(cb);
      g.ldcb = ldcb;
      g.error = derr;
      launch_gemm(g, s);
      int32_t h = 0;
      B2P_CUDA(cudaMemcpyAsync(&h, derr, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      B2P_CUDA(cudaStreamSynchronize(s));
      if (h) throw Error(B2P_ERR_CUDA, "tensor-core GEMM: mbarrier wait timed out");
    } catch (...) {
      cudaFree(derr);
      throw;
    }
    cudaFree(derr);
  });
}

int b2p_mlp_gemm_bf16_time(int32_t M, int32_t N, int32_t K, const uint16_t* A, int64_t sam, int64_t sak,
                           const uint16_t* B, int64_t sbk, int64_t sbn, float* cf, int64_t ldcf, int32_t reps,
                           double* ms_per_launch) {
  return guarded([&] {
    if (M <= 0 || N <= 0 || K <= 0 || reps <= 0) throw Error(B2P_ERR_INVALID, "sizes and reps must be positive");
    if (!A || !B || !cf || !ms_per_launch) throw Error(B2P_ERR_INVALID, "NULL argument");
    int dev = 0, major = 0;
    B2P_CUDA(cudaGetDevice(&dev));
    B2P_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) throw Error(B2P_ERR_NO_DEVICE, "tcgen05 GEMM needs an sm_100 device");
    set_gemm_attributes();
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int32_t* derr = nullptr;
    struct Cleanup {
      cudaStream_t& s;
      cudaEvent_t &e0, &e1;
      int32_t*& derr;
      ~Cleanup() {
        if (s) cudaStreamSynchronize(s);
        if (derr) cudaFree(derr);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (s) cudaStreamDestroy(s);
      }
    } cleanup{s, e0, e1, derr};
    B2P_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    B2P_CUDA(cudaEventCreate(&e0));
    B2P_CUDA(cudaEventCreate(&e1));
    derr = dalloc<int32_t>(1);
    B2P_CUDA(cudaMemsetAsync(derr, 0, sizeof(int32_t), s));
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.A = reinterpret_cast<const __nv_bfloat16*>(A);
    g.sam = sam;
    g.sak = sak;
    g.B = reinterpret_cast<const __nv_bfloat16*>(B);
    g.sbk = sbk;
    g.sbn = sbn;
    g.alpha = 1.0f;
    g.cf = cf;
    g.ldcf = ldcf;
    g.error = derr;
    launch_gemm(g, s);  // warm-up (module load, attributes)
    B2P_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r) launch_gemm(g, s);
    B2P_CUDA(cudaEventRecord(e1, s));
    B2P_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    B2P_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    int32_t h = 0;
    B2P_CUDA(cudaMemcpyAsync(&h, derr, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    B2P_CUDA(cudaStreamSynchronize(s));
    if (h) throw Error(B2P_ERR_CUDA, "tensor-core GEMM: mbarrier wait timed out");
    *ms_per_launch = static_cast<double>(ms) / reps;
  });
}

}  // extern "C"
