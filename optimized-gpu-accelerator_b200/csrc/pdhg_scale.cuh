// Diagonal scaling of an LP's operators on the device: Ruiz equilibration
// and the Pock-Chambolle step (src/lp/scaling.cpp:97-139), then the scaled
// operators value * (R_i * Cs_j) (scaling.cpp:28-32).  Used by the single-LP
// engine and, over the block-diagonal operator of a batch (whose LPs' rows and
// columns never meet), by the multi-LP engine.
//
// Each row / column quantity is the host's expression in the host's order --
// (|a| * Cs_j) * R_i; maxima are order-free; the 1-norms are summed by one
// thread in the row's or column's entry order (A's rows by increasing column,
// A^T's rows in the CSC order) -- so the factors are bit-identical to
// ruiz_impl in pdhg_prepare.cpp.  The power-of-two rounding of the factors
// and the rescaling constants stay on the host (finish_scaling).
#pragma once

#include <cstdint>
#include <vector>

#include "pdhg_host_common.h"
#include "pdhg_kernels.cuh"

namespace b2p {

// Per row r of a CSR operator: the maximum (SUM false) or the in-order sum
// (SUM true) over its entries of (|a| * Cs_j) * R_i.  For A's rows own is R
// (own_is_row) and other is Cs; for A^T's rows own is Cs and other is R; the
// product keeps the host's order in both.
template <bool SUM>
__global__ void k_ruiz_rows(int32_t rows, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            const double* __restrict__ val, const double* __restrict__ own,
                            const double* __restrict__ other, bool own_is_row, double* __restrict__ out) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const double so = own[r];
  double acc = 0.0;
  for (int32_t q = ptr[r]; q < ptr[r + 1]; ++q) {
    const double a = fabs(val[q]);
    // host order: (|a| * cs[j]) * rs[i]
    const double t = own_is_row ? __dmul_rn(__dmul_rn(a, other[idx[q]]), so) : __dmul_rn(__dmul_rn(a, so), other[idx[q]]);
    if (SUM)
      acc = __dadd_rn(acc, t);
    else
      acc = (acc < t) ? t : acc;
  }
  out[r] = acc;
}

// s[i] /= sqrt(q[i]) where q[i] > 0.
static __global__ void k_ruiz_update(int32_t len, const double* __restrict__ q, double* __restrict__ s) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < len && q[i] > 0) s[i] = __ddiv_rn(s[i], __dsqrt_rn(q[i]));
}

// a = a * (own[r] * other[idx]) for the entries of row r: the scaled operator
// value[q] * (R[i] * Cs[j]) (src/lp/scaling.cpp:28-32); for A^T, own = Cs and
// other = R, and the factor is still R[i] * Cs[j].
static __global__ void k_scale_rows(int32_t rows, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                             const double* __restrict__ own, const double* __restrict__ other,
                             double* __restrict__ val) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const double so = own[r];
  for (int32_t q = ptr[r]; q < ptr[r + 1]; ++q) val[q] = __dmul_rn(val[q], __dmul_rn(so, other[idx[q]]));
}

// Unrounded factors (rs over A's rows, cs over A^T's rows = A's columns) of
// the operators A and A^T with raw values: `iterations` equilibration passes,
// then the Pock-Chambolle pass.  rs and cs carry the starting factors in and
// the result out; temporaries come from the device's stream-ordered pool.
inline void device_ruiz_factors(cudaStream_t stream, int dev, const CsrView& A, const CsrView& AT, int iterations,
                                bool pock_chambolle, std::vector<double>& rs, std::vector<double>& cs) {
  const int32_t m = A.rows, n = AT.rows;
  const cudaMemPool_t pool = device_pool(dev);
  double *d_rs = nullptr, *d_cs = nullptr, *d_rq = nullptr, *d_cq = nullptr;
  B2P_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_rs), sizeof(double) * (m ? m : 1), pool, stream));
  B2P_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_rq), sizeof(double) * (m ? m : 1), pool, stream));
  B2P_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_cs), sizeof(double) * (n ? n : 1), pool, stream));
  B2P_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_cq), sizeof(double) * (n ? n : 1), pool, stream));
  if (m) B2P_CUDA(cudaMemcpyAsync(d_rs, rs.data(), sizeof(double) * m, cudaMemcpyHostToDevice, stream));
  if (n) B2P_CUDA(cudaMemcpyAsync(d_cs, cs.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream));
  const unsigned gm = static_cast<unsigned>((m + kBlock - 1) / kBlock), gn = static_cast<unsigned>((n + kBlock - 1) / kBlock);
  auto pass = [&](bool sum) {
    if (n) {
      if (sum)
        k_ruiz_rows<true><<<gn, kBlock, 0, stream>>>(n, AT.ptr, AT.idx, AT.val, d_cs, d_rs, false, d_cq);
      else
        k_ruiz_rows<false><<<gn, kBlock, 0, stream>>>(n, AT.ptr, AT.idx, AT.val, d_cs, d_rs, false, d_cq);
    }
    if (m) {
      if (sum)
        k_ruiz_rows<true><<<gm, kBlock, 0, stream>>>(m, A.ptr, A.idx, A.val, d_rs, d_cs, true, d_rq);
      else
        k_ruiz_rows<false><<<gm, kBlock, 0, stream>>>(m, A.ptr, A.idx, A.val, d_rs, d_cs, true, d_rq);
      k_ruiz_update<<<gm, kBlock, 0, stream>>>(m, d_rq, d_rs);
    }
    if (n) k_ruiz_update<<<gn, kBlock, 0, stream>>>(n, d_cq, d_cs);
  };
  for (int it = 0; it < iterations; ++it) pass(false);
  if (pock_chambolle) pass(true);
  B2P_CUDA(cudaGetLastError());
  if (m) B2P_CUDA(cudaMemcpyAsync(rs.data(), d_rs, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
  if (n) B2P_CUDA(cudaMemcpyAsync(cs.data(), d_cs, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
  for (double* p : {d_rs, d_cs, d_rq, d_cq}) cudaFreeAsync(p, stream);
  B2P_CUDA(cudaStreamSynchronize(stream));
}

// A.val and AT.val (raw, in place) <- value * (R_i * Cs_j) with the rounded
// factors R (rows of A) and Cs (columns).
inline void device_scale_operators(cudaStream_t stream, int dev, const CsrView& A, const CsrView& AT, double* a_val,
                                   double* t_val, const std::vector<double>& R, const std::vector<double>& Cs) {
  const int32_t m = A.rows, n = AT.rows;
  const cudaMemPool_t pool = device_pool(dev);
  double *dR = nullptr, *dC = nullptr;
  B2P_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dR), sizeof(double) * (m ? m : 1), pool, stream));
  B2P_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dC), sizeof(double) * (n ? n : 1), pool, stream));
  if (m) B2P_CUDA(cudaMemcpyAsync(dR, R.data(), sizeof(double) * m, cudaMemcpyHostToDevice, stream));
  if (n) B2P_CUDA(cudaMemcpyAsync(dC, Cs.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream));
  if (m) k_scale_rows<<<static_cast<unsigned>((m + kBlock - 1) / kBlock), kBlock, 0, stream>>>(m, A.ptr, A.idx, dR, dC, a_val);
  if (n) k_scale_rows<<<static_cast<unsigned>((n + kBlock - 1) / kBlock), kBlock, 0, stream>>>(n, AT.ptr, AT.idx, dC, dR, t_val);
  B2P_CUDA(cudaGetLastError());
  cudaFreeAsync(dR, stream);
  cudaFreeAsync(dC, stream);
  // the host vectors R and Cs must outlive the copies
  B2P_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace b2p
