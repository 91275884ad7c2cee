// BF16 tensor-core GEMM for the warm-start network, on the 5th-generation
// tensor cores (tcgen05): C[M x N] = alpha * A[M x K] B[K x N] with FP32
// accumulation in tensor memory, plus a fused epilogue (bias, ReLU, a 0/1
// mask from a BF16 array, FP32 and/or BF16 output).
//
// One CTA (128 threads) computes a 128 x BN tile, BN = 128 or 256 (the wide
// tile reads each A chunk once for twice the output and is chosen when the
// grid of wide tiles still fills every SM).  The K dimension runs in chunks
// of 64 through S shared-memory stages, refilled LAG chunks after the MMAs
// that read them were issued (BN = 128: S = 3, LAG = 1, two CTAs per SM;
// BN = 256: S = 4, LAG = 2, one CTA per SM, so that chunk c's MMAs are
// issued while chunk c - 1's still run): at chunk c the threads fetch chunk
// c + S - LAG into the stage chunk c - LAG used (16-byte cp.async copies from
// global memory when the operand is K-contiguous, element loads otherwise).
// Each stage holds A (128 x 64) and B (BN x 64) in the K-major, non-swizzled
// canonical layout of the UMMA
// descriptors -- core matrices of 8 rows x 16 bytes, the two 8-element K
// halves of a 16-wide slab LBO = 128 B apart, consecutive 8-row groups SBO =
// 256 B apart.  One elected thread issues four tcgen05.mma (K = 16 each) per
// chunk into the TMEM accumulator and commits them to the stage's mbarrier;
// a stage is refilled only after its mbarrier reports the MMAs that read it
// complete.  The epilogue reads the accumulator with tcgen05.ld (warp w owns
// TMEM lanes 32w..32w+31 = tile rows).  A and B are read through element
// strides, so either operand may be used transposed.  Waits are bounded: on
// a timeout the kernel records an error, frees its TMEM and returns.
//
// When both operands are K-contiguous, the TMA form at the end of this file
// (k_gemm_bf16_tma) replaces the threads' copies with tensor-map copies into
// 128-byte-swizzled stages and splits the CTA into producer and MMA warps.
#pragma once

#include <cuda.h>  // CUtensorMap (the type only; maps are encoded through the runtime's driver entry point)
#include <cuda_bf16.h>

#include <cstdint>

namespace b2p {

constexpr int kGemmBM = 128;
constexpr int kGemmBK = 64;
constexpr int kGemmThreads = 128;
constexpr unsigned kMbarSpinLimit = 1u << 24;

// Tile shape: BN output columns (= TMEM columns), S stages of A 16 KB + B
// BN x 64 x 2 bytes.  BN = 128: three stages (96 KB), at most two CTAs per
// SM (2 x 128 TMEM columns <= 512).  BN = 256: four stages (192 KB), one CTA
// per SM.
template <int BN>
struct GemmTile {
  static constexpr int kStages = BN == 256 ? 4 : 3;
  static constexpr int kLag = BN == 256 ? 2 : 1;  // stage refill lag, in chunks
  static constexpr int kAhead = kStages - kLag;   // chunks in flight ahead of the MMAs
  static constexpr int kStageBytes = (kGemmBM + BN) * kGemmBK * 2;
  static constexpr int kSmemBytes = kStages * kStageBytes;
  static_assert(BN == 128 || BN == 256, "tile width");
  static_assert(kSmemBytes <= 200 * 1024, "stages exceed the shared-memory budget");
};

struct GemmArgs {
  int32_t M, N, K;
  const __nv_bfloat16* A;
  int64_t sam, sak;  // A(m, k) = A[m * sam + k * sak]
  const __nv_bfloat16* B;
  int64_t sbk, sbn;  // B(k, n) = B[k * sbk + n * sbn]
  float alpha;
  const float* bias;  // bias[n] added after alpha, or NULL
  int32_t relu;
  const __nv_bfloat16* mask;  // C(m, n) *= (mask[m * ldm + n] > 0), or NULL
  int64_t ldm;
  float* cf;  // FP32 output C[m * ldcf + n], or NULL
  int64_t ldcf;
  __nv_bfloat16* cb;  // BF16 output, or NULL
  int64_t ldcb;
  int32_t* error;  // set to 1 on an mbarrier timeout
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, K-major, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFF);
  d |= static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= static_cast<uint64_t>(1) << 46;  // descriptor version (Blackwell)
  // base offset 0, legacy LBO mode, layout type 0 = SWIZZLE_NONE
  return d;
}

// Instruction descriptor: kind::f16, BF16 x BF16 -> F32, both K-major, M = 128,
// N = n (a multiple of 16 up to 256).
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
  return (1u << 4)                                   // D format F32
         | (1u << 7)                                 // A format BF16
         | (1u << 10)                                // B format BF16
         | (static_cast<uint32_t>(n >> 3) << 17)     // N / 8
         | (static_cast<uint32_t>(kGemmBM >> 4) << 24);  // M / 16
}

// byte offset of element (r, k) of a row-major-in-K chunk of 64 columns
__device__ __forceinline__ uint32_t chunk_offset(int r, int k, int rows) {
  const int s = k >> 4, kk = k & 15;
  return static_cast<uint32_t>(s * (rows / 8) * 256 + (r >> 3) * 256 + (kk >> 3) * 128 + (r & 7) * 16 + (kk & 7) * 2);
}

// Copy the rows [r0, r0 + rows) x K columns [k0, k0 + 64) of an operand
// X(r, k) = X[r * sr + k * sk] into the canonical layout, zero-filling past
// R and K.  vec: sk == 1 and 16-byte aligned rows, so one thread moves one
// 8-element core-matrix row (16 bytes) per step as an asynchronous cp.async
// (source size 0 past the edge: the hardware writes zeros); the caller waits
// for them with cp.async.wait_group.  Otherwise single elements, stored
// directly, row index fastest when sr == 1 (a transposed operand) for
// coalescing.
__device__ __forceinline__ void stage_operand(unsigned char* dst, const __nv_bfloat16* X, int64_t sr, int64_t sk,
                                              int r0, int R, int k0, int K, int rows, bool vec, int tid) {
  if (vec) {
    for (int e = tid; e < rows * (kGemmBK / 8); e += kGemmThreads) {
      const int r = e / (kGemmBK / 8), k = (e % (kGemmBK / 8)) * 8;
      const int gr = r0 + r, gk = k0 + k;
      const bool in = gr < R && gk < K;
      const __nv_bfloat16* src = in ? X + gr * sr + gk : X;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst + chunk_offset(r, k, rows))),
                   "l"(src), "r"(in ? 16 : 0)
                   : "memory");
    }
    return;
  }
  const bool row_fast = sr == 1;
  for (int e = tid; e < rows * kGemmBK; e += kGemmThreads) {
    const int r = row_fast ? e % rows : e / kGemmBK, k = row_fast ? e / rows : e % kGemmBK;
    const int gr = r0 + r, gk = k0 + k;
    __nv_bfloat16 v = __float2bfloat16(0.0f);
    if (gr < R && gk < K) v = X[gr * sr + gk * sk];
    *reinterpret_cast<__nv_bfloat16*>(dst + chunk_offset(r, k, rows)) = v;
  }
}

// vectorised staging applies: unit K stride, K and the row stride multiples
// of 8 elements, 16-byte aligned base
__host__ __device__ inline bool stage_vec_ok(const void* X, int64_t sr, int64_t sk, int K) {
  return sk == 1 && K % 8 == 0 && sr % 8 == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (unsigned spin = 0; spin < kMbarSpinLimit; ++spin) {
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

// Epilogue of one 128 x BN tile: thread = tile row (TMEM lane), 8 columns
// per tcgen05.ld; alpha, bias, ReLU and the 0/1 mask applied in FP32; a
// thread's 8 consecutive outputs go out as 16- or 32-byte vector stores when
// the row stride and base allow it (one sector per store instead of eight
// scattered ones).
template <int BN>
__device__ __forceinline__ void gemm_epilogue(const GemmArgs& g, uint32_t tmem, int m0, int n0, int warp, int lane) {
  constexpr int kGemmBN = BN;
  const int row = warp * 32 + lane;
  const int gm = m0 + row;
  const bool vec_f = g.cf && g.ldcf % 4 == 0 && (reinterpret_cast<uintptr_t>(g.cf) & 15) == 0;
  const bool vec_b = g.cb && g.ldcb % 8 == 0 && (reinterpret_cast<uintptr_t>(g.cb) & 15) == 0;
  for (int c = 0; c < kGemmBN; c += 8) {
    uint32_t r[8];
    const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (gm >= g.M || n0 + c >= g.N) continue;
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int gn = n0 + c + q;
      float t = __uint_as_float(r[q]) * g.alpha;
      if (gn < g.N) {
        if (g.bias) t += g.bias[gn];
        if (g.relu) t = t > 0.0f ? t : 0.0f;
        if (g.mask && !(__bfloat162float(g.mask[gm * g.ldm + gn]) > 0.0f)) t = 0.0f;
      }
      v[q] = t;
    }
    const bool full = n0 + c + 8 <= g.N;
    if (g.cf) {
      float* dst = g.cf + gm * g.ldcf + n0 + c;
      if (vec_f && full) {
        reinterpret_cast<float4*>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float4*>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (n0 + c + q < g.N) dst[q] = v[q];
      }
    }
    if (g.cb) {
      __nv_bfloat16* dst = g.cb + gm * g.ldcb + n0 + c;
      if (vec_b && full) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16(v[q]);
        *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(h);
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (n0 + c + q < g.N) dst[q] = __float2bfloat16(v[q]);
      }
    }
  }
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16_tc(GemmArgs g) {
  constexpr int kGemmBN = BN;
  constexpr int kGemmStages = GemmTile<BN>::kStages;
  constexpr int kGemmStageBytes = GemmTile<BN>::kStageBytes;
  constexpr int kLag = GemmTile<BN>::kLag, kAhead = GemmTile<BN>::kAhead;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[kGemmStages];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int failed_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * kGemmBN;

  if (tid == 0) {
#pragma unroll
    for (int st = 0; st < kGemmStages; ++st)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[st])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    failed_sh = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(kGemmBN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_sh;
  const uint32_t idesc = umma_idesc_bf16(kGemmBN);
  const int nchunks = (g.K + kGemmBK - 1) / kGemmBK;
  const bool vec_a = stage_vec_ok(g.A, g.sam, g.sak, g.K), vec_b = stage_vec_ok(g.B, g.sbn, g.sbk, g.K);
  uint32_t phase[kGemmStages] = {};  // parity of each stage's next completion
  auto stage_a = [&](int st) { return smem + st * kGemmStageBytes; };
  auto stage_b = [&](int st) { return smem + st * kGemmStageBytes + kGemmBM * kGemmBK * 2; };
  auto fetch = [&](int ch) {  // chunk ch into stage ch % kGemmStages, as one cp.async group
    const int st = ch % kGemmStages, k0 = ch * kGemmBK;
    stage_operand(stage_a(st), g.A, g.sam, g.sak, m0, g.M, k0, g.K, kGemmBM, vec_a, tid);
    stage_operand(stage_b(st), g.B, g.sbn, g.sbk, n0, g.N, k0, g.K, kGemmBN, vec_b, tid);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // prologue: the first kAhead chunks in flight
  for (int c = 0; c < kAhead; ++c)
    if (c < nchunks) fetch(c);
  for (int ch = 0; ch < nchunks; ++ch) {
    const int st = ch % kGemmStages;
    const int ahead = ch + kAhead;  // the chunk fetched in this step
    if (ahead < nchunks) {
      // its stage was last read by chunk ch - kLag's MMAs: refill it once
      // they are done (a stage not used yet needs no wait)
      const int nx = ahead % kGemmStages;
      if (ch >= kLag) {
        if (!mbar_wait(smem_u32(&mbar[nx]), phase[nx])) failed_sh = 1;
        phase[nx] ^= 1u;
      }
      __syncthreads();
      if (failed_sh) break;
      fetch(ahead);
      asm volatile("cp.async.wait_group %0;" ::"n"(kAhead) : "memory");  // chunk ch has landed
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_base = smem_u32(stage_a(st)), b_base = smem_u32(stage_b(st));
#pragma unroll
      for (int s = 0; s < kGemmBK / 16; ++s) {
        const uint64_t da = umma_desc(a_base + s * (kGemmBM / 8) * 256, 128, 256);
        const uint64_t db = umma_desc(b_base + s * (kGemmBN / 8) * 256, 128, 256);
        const uint32_t acc = (ch > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            :
            : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[st]))
                   : "memory");
    }
  }
  // the last commit tracks every MMA issued before it
  if (nchunks > 0 && !failed_sh) {
    const int st = (nchunks - 1) % kGemmStages;
    if (!mbar_wait(smem_u32(&mbar[st]), phase[st])) failed_sh = 1;
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!failed_sh) {
    gemm_epilogue<kGemmBN>(g, tmem, m0, n0, warp, lane);
  } else if (tid == 0) {
    atomicExch(g.error, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kGemmBN) : "memory");
}


// ---------------------------------------------------------------------------
// TMA form, for operands whose K dimension is contiguous (A row-major M x K,
// B stored N x K) with 16-byte aligned rows.  The same 128 x BN tiles and
// stage counts, but the operands are brought in by the tensor memory
// accelerator (cp.async.bulk.tensor.2d, one 64 x rows box per operand and
// chunk, zero-filled past the edges) into the 128-byte-swizzled K-major
// layout, and the CTA's roles are split: warp 0 issues the copies, warp 1
// the MMAs (one lane each, the other lanes following in step so that no lane
// spins beside them), and all four warps run the epilogue.  Each stage
// has a "full" mbarrier (the copies' bytes arrived) and an "empty" one (the
// MMAs that read it completed); the producer refills a stage once it is
// empty, so up to S chunks are in flight while the tensor core works.  Every
// wait is bounded: on a timeout the kernel records an error, waits (bounded)
// for the copies it issued, frees its TMEM and returns.

template <int BN>
struct GemmTmaTile {
  static constexpr int kStages = BN == 256 ? 4 : 3;
  static constexpr int kABytes = kGemmBM * kGemmBK * 2;  // 16 KB
  static constexpr int kBBytes = BN * kGemmBK * 2;
  static constexpr int kStageBytes = kABytes + kBBytes;
  // + 1 KB so that the stages can start on a 1,024-byte boundary (the
  // period of the 128-byte swizzle)
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024;
};

// UMMA shared-memory descriptor, K-major, 128-byte swizzle: rows of 64 BF16
// (128 bytes) as the copies wrote them, 8-row groups SBO = 1,024 bytes apart,
// LBO unused (1).  addr advances by 32 bytes per K = 16 step inside the
// 128-byte row; the swizzle is applied to the absolute address bits.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFF);
  d |= static_cast<uint64_t>(1) << 16;            // LBO (unused for swizzled K-major)
  d |= static_cast<uint64_t>(1024 >> 4) << 32;    // SBO
  d |= static_cast<uint64_t>(1) << 46;            // descriptor version (Blackwell)
  d |= static_cast<uint64_t>(2) << 61;            // layout type SWIZZLE_128B
  return d;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16_tma(const __grid_constant__ CUtensorMap map_a,
                                                                 const __grid_constant__ CUtensorMap map_b,
                                                                 GemmArgs g) {
  using Tile = GemmTmaTile<BN>;
  constexpr int S = Tile::kStages;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[S], empty[S], done;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int failed_sh, issued_sh, consumed_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * BN;
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;  // stage 0, 1,024-byte aligned
  const int nchunks = (g.K + kGemmBK - 1) / kGemmBK;

  if (tid == 0) {
    for (int st = 0; st < S; ++st) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[st])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[st])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&done)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    failed_sh = 0;
    issued_sh = 0;
    consumed_sh = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_sh;

  if (warp == 0) {
    // producer warp (lane 0 issues): chunk ch into stage ch % S once the MMAs
    // of chunk ch - S are done
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_a)) : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_b)) : "memory");
    }
    int ch = 0;
    for (; ch < nchunks; ++ch) {
      const int st = ch % S;
      bool ok = true;
      if (ch >= S) ok = mbar_wait(smem_u32(&empty[st]), static_cast<uint32_t>((ch / S - 1) & 1));
      if (!__all_sync(0xffffffffu, ok) || *reinterpret_cast<volatile int*>(&failed_sh)) {
        if (lane == 0) failed_sh = 1;
        break;
      }
      if (lane == 0) {
        const uint32_t sa = base + st * Tile::kStageBytes, sb = sa + Tile::kABytes;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&full[st])),
                     "r"(Tile::kStageBytes)
                     : "memory");
        tma_load_2d(sa, &map_a, ch * kGemmBK, m0, smem_u32(&full[st]));
        tma_load_2d(sb, &map_b, ch * kGemmBK, n0, smem_u32(&full[st]));
      }
      __syncwarp();
    }
    if (lane == 0) issued_sh = ch;
  } else if (warp == 1) {
    // MMA warp (lane 0 issues): four K = 16 steps per chunk, then commit the
    // stage back
    const uint32_t idesc = umma_idesc_bf16(BN);
    int ch = 0;
    for (; ch < nchunks; ++ch) {
      const int st = ch % S;
      const bool ok = mbar_wait(smem_u32(&full[st]), static_cast<uint32_t>((ch / S) & 1));
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) failed_sh = 1;
        break;
      }
      if (lane == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t sa = base + st * Tile::kStageBytes, sb = sa + Tile::kABytes;
#pragma unroll
        for (int s = 0; s < kGemmBK / 16; ++s) {
          const uint64_t da = umma_desc_sw128(sa + s * 32), db = umma_desc_sw128(sb + s * 32);
          const uint32_t acc = (ch > 0 || s > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
              :
              : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
              : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&empty[st]))
                     : "memory");
      }
      __syncwarp();
    }
    if (lane == 0) {
      consumed_sh = ch;
      // tracks every MMA issued before it
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&done))
                   : "memory");
    }
    __syncwarp();
  }
  if (!mbar_wait(smem_u32(&done), 0u)) failed_sh = 1;
  __syncthreads();
  __syncwarp();  // the producer and MMA lanes rejoin their warps before tcgen05.ld
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!failed_sh) {
    gemm_epilogue<BN>(g, tmem, m0, n0, warp, lane);
  } else if (tid == 0) {
    atomicExch(g.error, 1);
    // copies issued but not consumed still write into shared memory: wait for them
    for (int ch = consumed_sh; ch < issued_sh; ++ch)
      mbar_wait(smem_u32(&full[ch % S]), static_cast<uint32_t>((ch / S) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
}

}  // namespace b2p
