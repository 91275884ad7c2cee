// Device-side pieces of the certifier shared between translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "pdhg_kernels.cuh"

namespace b2p {

// Enqueues the outward-rounded Neumaier-Shcherbina bound of k cases on `s`
// (pdhg_certify.cu).  Device arrays, case-major: y (k x m), c, lo, up
// (k x n), rl, ru (k x m); AT is A in CSC form read as the CSR of A^T.
// Work: yp (k x m), terms (k x (m + n)), stats (k x 4), inf_terms (k).
// Out: bound (k), -inf where a column forces it; stats[4b + {0, 1, 2}] =
// row projection, largest clipped reduced cost, cost perturbation.
void enqueue_safe_bound(cudaStream_t s, int32_t m, int32_t n, int32_t k, CsrView AT, const double* y, const double* c,
                        const double* lo, const double* up, const double* rl, const double* ru, double* yp,
                        double* terms, double* stats, int32_t* inf_terms, double* bound);

}  // namespace b2p
