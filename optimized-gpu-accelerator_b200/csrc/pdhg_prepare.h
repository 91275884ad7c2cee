// Host-side problem preparation for the PDHG engine: diagonal scaling,
// objective/bound rescaling, the two CSR operators and the spectral-norm
// estimate.  Follows PRAMANA's prepare() (src/pdhg/pdhg.cpp:394-459) and
// ruizScaling() (src/lp/scaling.cpp:97-139) with the same floating-point
// evaluation order, so that the scaled problem is bit-identical.
#pragma once

#include <cstdint>
#include <vector>

namespace b2p {

constexpr double kInfBoundThreshold = 1e20;  // src/util/common.h:14
inline bool finite_bound(double v) { return v < kInfBoundThreshold && v > -kInfBoundThreshold; }
// std::max / std::min semantics (the reference uses them throughout).
inline double smax(double a, double b) { return (a < b) ? b : a; }
inline double smin(double a, double b) { return (b < a) ? b : a; }

struct HostCsr {
  int32_t rows = 0, cols = 0;
  std::vector<int32_t> ptr, idx;
  std::vector<double> val;
};

struct Prepared {
  int32_t n = 0, m = 0;
  HostCsr A, AT;                // A (m x n) and A^T (n x m), both row-major
  std::vector<double> R, Cs;    // power-of-two row / column factors
  double beta = 1, gamma = 1;   // bound / objective rescaling
  std::vector<double> rfac, cfac;
  double normA = 1;             // 1.01 x power-iteration estimate of ||A||_2
  double offset = 0;
};

struct PrepareOptions {
  int ruiz_iterations = 10;
  bool pock_chambolle = true;
  bool rescale = true;
  bool norm_on_host = true;  // false: normA is left 0 for the caller to estimate (on the device)
  // run the element-wise passes on host threads (OpenMP); every result is
  // the same as the sequential passes' (maxima are order-free, every sum
  // keeps its order).  Off when the caller already prepares LPs in parallel.
  bool parallel = true;
};

// A given in CSC (start/index/value) with m rows and n columns.
Prepared prepare(int32_t m, int32_t n, const int32_t* start, const int32_t* index, const double* value,
                 const double* cost, const double* row_lower, const double* row_upper, double offset,
                 const PrepareOptions& opt);

// Structure-only preparation (scaling done elsewhere, e.g. on the device):
// A (CSR, from the same stable counting sort) and A^T (= the CSC) with the
// raw values, R = Cs = 1, no rescaling constants yet.
Prepared prepare_structure(int32_t m, int32_t n, const int32_t* start, const int32_t* index, const double* value,
                           double offset, bool parallel);

// Completes a structure-only preparation from the unrounded Ruiz factors
// (rs, cs): their power-of-two rounding (src/lp/scaling.cpp:9-14), beta and
// gamma (src/pdhg/pdhg.cpp:440-452) and the factors of the check.  The
// operators' values are left to the caller.
void finish_scaling(Prepared& P, const double* rs, const double* cs, const double* cost, const double* row_lower,
                    const double* row_upper, bool rescale);

double pow2_round(double v);

double power_iteration(int32_t m, int32_t n, const int32_t* start, const int32_t* index, const double* value,
                       int iters);

}  // namespace b2p
