#include "pdhg_prepare.h"

#include <omp.h>

#include <algorithm>
#include <cmath>

namespace b2p {

// Power-of-two rounding of a scale factor (src/lp/scaling.cpp:9-14): the
// nearest 2^e with |e| <= 60, so that scaling and unscaling are exact.
double pow2_round(double v) {
  if (!(v > 0) || !std::isfinite(v)) return 1.0;
  int e = static_cast<int>(std::lround(std::log2(v)));
  e = e < -60 ? -60 : (e > 60 ? 60 : e);
  return std::ldexp(1.0, e);
}

namespace {

// Row-major view of a CSC matrix: for every row, its entries by increasing
// column -- the order SparseMatrix::transpose produces
// (src/core/sparse.cpp:49-65) and hence the order of every row sum -- as
// (column, CSC position) pairs.
struct RowMap {
  std::vector<int32_t> ptr, col, pos;
};

RowMap row_map(int32_t m, int32_t n, const int32_t* start, const int32_t* index, bool par) {
  RowMap r;
  const int32_t nnz = start[n];
  r.ptr.assign(static_cast<size_t>(m) + 1, 0);
  r.col.resize(nnz);
  r.pos.resize(nnz);
  int T = par ? omp_get_max_threads() : 1;
  // per-thread row counters: T x m integers, capped at 2^26
  if (T > 1 && static_cast<int64_t>(T) * m > (int64_t(1) << 26))
    T = static_cast<int>(std::max<int64_t>(1, (int64_t(1) << 26) / std::max<int32_t>(m, 1)));
  if (T <= 1 || m == 0) {
    for (int32_t q = 0; q < nnz; ++q) r.ptr[index[q] + 1]++;
    for (int32_t i = 0; i < m; ++i) r.ptr[i + 1] += r.ptr[i];
    std::vector<int32_t> next(r.ptr.begin(), r.ptr.end() - 1);
    for (int32_t j = 0; j < n; ++j)
      for (int32_t q = start[j]; q < start[j + 1]; ++q) {
        const int32_t e = next[index[q]]++;
        r.col[e] = j;
        r.pos[e] = q;
      }
    return r;
  }
  // Parallel stable counting sort: thread t takes a run of whole columns
  // (balanced by entries); its entries of row i go after those of threads
  // < t, in column order, so the result equals the sequential one.
  std::vector<int32_t> cbeg(static_cast<size_t>(T) + 1);
  for (int t = 0; t <= T; ++t) {
    const int64_t target = static_cast<int64_t>(nnz) * t / T;
    cbeg[t] = static_cast<int32_t>(std::lower_bound(start, start + n, target) - start);
  }
  cbeg[T] = n;
  std::vector<int32_t> cnt(static_cast<size_t>(T) * m, 0);
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    int32_t* c = cnt.data() + static_cast<size_t>(t) * m;
    for (int32_t q = start[cbeg[t]]; q < start[cbeg[t + 1]]; ++q) c[index[q]]++;
  }
#pragma omp parallel for schedule(static) num_threads(T)
  for (int32_t i = 0; i < m; ++i) {
    int32_t tot = 0;
    for (int t = 0; t < T; ++t) tot += cnt[static_cast<size_t>(t) * m + i];
    r.ptr[i + 1] = tot;
  }
  for (int32_t i = 0; i < m; ++i) r.ptr[i + 1] += r.ptr[i];
#pragma omp parallel for schedule(static) num_threads(T)
  for (int32_t i = 0; i < m; ++i) {
    int32_t off = r.ptr[i];
    for (int t = 0; t < T; ++t) {
      int32_t& c = cnt[static_cast<size_t>(t) * m + i];
      const int32_t k = c;
      c = off;
      off += k;
    }
  }
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    int32_t* cur = cnt.data() + static_cast<size_t>(t) * m;
    for (int32_t j = cbeg[t]; j < cbeg[t + 1]; ++j)
      for (int32_t q = start[j]; q < start[j + 1]; ++q) {
        const int32_t e = cur[index[q]]++;
        r.col[e] = j;
        r.pos[e] = q;
      }
  }
  return r;
}

// OpenMP only above this many nonzeros (the team's start-up costs more below)
constexpr int32_t kParallelNnz = 1 << 15;

}  // namespace

// Each pass computes every row and column quantity with the same expression
// and, for the Pock-Chambolle sums, in the same order as the reference's
// column sweep (a row's terms by increasing column), so the result does not
// depend on `parallel`.
namespace {

void ruiz_impl(int32_t m, int32_t n, const int32_t* start, const int32_t* index, const double* value,
               int iterations, bool pock_chambolle, std::vector<double>& rs, std::vector<double>& cs, const RowMap& R,
               bool par) {
  rs.assign(m, 1.0);
  cs.assign(n, 1.0);
  std::vector<double> rmax(m), cmax(n);
  // |A| in row order, once: the row passes then read it sequentially
  const int32_t nnz = start[n];
  std::vector<double> rabs(nnz);
#pragma omp parallel for schedule(static) if (par)
  for (int32_t e = 0; e < nnz; ++e) rabs[e] = std::fabs(value[R.pos[e]]);
  // Infinity-norm equilibration passes.
  for (int it = 0; it < iterations; ++it) {
#pragma omp parallel for schedule(static) if (par)
    for (int32_t j = 0; j < n; ++j) {
      double c = 0;
      for (int32_t q = start[j]; q < start[j + 1]; ++q) c = smax(c, std::fabs(value[q]) * cs[j] * rs[index[q]]);
      cmax[j] = c;
    }
#pragma omp parallel for schedule(static) if (par)
    for (int32_t i = 0; i < m; ++i) {
      double r = 0;
      for (int32_t e = R.ptr[i]; e < R.ptr[i + 1]; ++e) r = smax(r, rabs[e] * cs[R.col[e]] * rs[i]);
      rmax[i] = r;
    }
#pragma omp parallel for schedule(static) if (par)
    for (int32_t i = 0; i < m; ++i)
      if (rmax[i] > 0) rs[i] /= std::sqrt(rmax[i]);
#pragma omp parallel for schedule(static) if (par)
    for (int32_t j = 0; j < n; ++j)
      if (cmax[j] > 0) cs[j] /= std::sqrt(cmax[j]);
  }
  // Pock-Chambolle step with alpha = 1 (row / column 1-norms).
  if (pock_chambolle) {
    std::vector<double> rsum(m, 0.0), csum(n, 0.0);
#pragma omp parallel for schedule(static) if (par)
    for (int32_t j = 0; j < n; ++j) {
      double c = 0.0;
      for (int32_t q = start[j]; q < start[j + 1]; ++q) c += std::fabs(value[q]) * cs[j] * rs[index[q]];
      csum[j] = c;
    }
#pragma omp parallel for schedule(static) if (par)
    for (int32_t i = 0; i < m; ++i) {
      double r = 0.0;
      for (int32_t e = R.ptr[i]; e < R.ptr[i + 1]; ++e) r += rabs[e] * cs[R.col[e]] * rs[i];
      rsum[i] = r;
    }
#pragma omp parallel for schedule(static) if (par)
    for (int32_t i = 0; i < m; ++i)
      if (rsum[i] > 0) rs[i] /= std::sqrt(rsum[i]);
#pragma omp parallel for schedule(static) if (par)
    for (int32_t j = 0; j < n; ++j)
      if (csum[j] > 0) cs[j] /= std::sqrt(csum[j]);
  }
  for (auto& v : rs) v = pow2_round(v);
  for (auto& v : cs) v = pow2_round(v);
}

}  // namespace

// ||A||_2 estimate: 40 steps of x <- A^T A x / ||A^T A x|| and sqrt of the
// last norm (src/pdhg/pdhg.cpp:404-422), with the scatter-order products of
// SparseMatrix::multiply / multiplyTranspose (src/core/sparse.cpp:67-82).
double power_iteration(int32_t m, int32_t n, const int32_t* start, const int32_t* index, const double* value,
                       int iters) {
  if (start[n] == 0) return 1.0;
  std::vector<double> x(n, 1.0 / std::sqrt(static_cast<double>(n > 1 ? n : 1))), y(m), z(n);
  double s = 1;
  for (int it = 0; it < iters; ++it) {
    std::fill(y.begin(), y.end(), 0.0);
    for (int32_t j = 0; j < n; ++j) {
      const double xj = x[j];
      if (xj == 0.0) continue;
      for (int32_t q = start[j]; q < start[j + 1]; ++q) y[index[q]] += value[q] * xj;
    }
    for (int32_t j = 0; j < n; ++j) {
      double t = 0;
      for (int32_t q = start[j]; q < start[j + 1]; ++q) t += value[q] * y[index[q]];
      z[j] = t;
    }
    double nz = 0;
    for (int32_t j = 0; j < n; ++j) nz += z[j] * z[j];
    nz = std::sqrt(nz);
    if (nz == 0) return 1.0;
    s = std::sqrt(nz);
    for (int32_t j = 0; j < n; ++j) x[j] = z[j] / nz;
  }
  return s;
}

Prepared prepare(int32_t m, int32_t n, const int32_t* start, const int32_t* index, const double* value,
                 const double* cost, const double* row_lower, const double* row_upper, double offset,
                 const PrepareOptions& opt) {
  Prepared P;
  P.n = n;
  P.m = m;
  P.offset = offset;
  const int32_t nnz = start[n];
  const bool par = opt.parallel && nnz >= kParallelNnz;
  RowMap rm = row_map(m, n, start, index, par);
  if (opt.ruiz_iterations > 0 && nnz > 0) {
    ruiz_impl(m, n, start, index, value, opt.ruiz_iterations, opt.pock_chambolle, P.R, P.Cs, rm, par);
  } else {
    P.R.assign(m, 1.0);
    P.Cs.assign(n, 1.0);
  }
  // A <- diag(R) A diag(Cs) (src/lp/scaling.cpp:28-32); exact, the factors are powers of two.
  std::vector<double> sval(nnz);
#pragma omp parallel for schedule(static) if (par)
  for (int32_t j = 0; j < n; ++j)
    for (int32_t q = start[j]; q < start[j + 1]; ++q) sval[q] = value[q] * (P.R[index[q]] * P.Cs[j]);
  if (opt.rescale) {
    double cn = 0, bn = 0;
    for (int32_t j = 0; j < n; ++j) {
      const double t = cost[j] * P.Cs[j];
      cn += t * t;
    }
    for (int32_t i = 0; i < m; ++i) {
      if (finite_bound(row_lower[i])) {
        const double t = row_lower[i] * P.R[i];
        bn += t * t;
      }
      if (finite_bound(row_upper[i]) && row_upper[i] != row_lower[i]) {
        const double t = row_upper[i] * P.R[i];
        bn += t * t;
      }
    }
    P.gamma = 1.0 + std::sqrt(cn);
    P.beta = 1.0 + std::sqrt(bn);
  }
  {
    P.A.rows = m;
    P.A.cols = n;
    P.A.val.resize(nnz);
#pragma omp parallel for schedule(static) if (par)
    for (int32_t e = 0; e < nnz; ++e) P.A.val[e] = sval[rm.pos[e]];
    P.A.ptr = std::move(rm.ptr);
    P.A.idx = std::move(rm.col);
  }
  // CSR of A^T is the (scaled) CSC of A.
  P.AT.rows = n;
  P.AT.cols = m;
  P.AT.ptr.resize(static_cast<size_t>(n) + 1);
  P.AT.idx.resize(nnz);
#pragma omp parallel for schedule(static) if (par)
  for (int32_t j = 0; j <= n; ++j) P.AT.ptr[j] = start[j];
#pragma omp parallel for schedule(static) if (par)
  for (int32_t q = 0; q < nnz; ++q) P.AT.idx[q] = index[q];
  P.AT.val = std::move(sval);
  P.rfac.resize(m);
  P.cfac.resize(n);
  for (int32_t i = 0; i < m; ++i) P.rfac[i] = P.beta / P.R[i];
  for (int32_t j = 0; j < n; ++j) P.cfac[j] = P.gamma / P.Cs[j];
  if (opt.norm_on_host) P.normA = power_iteration(m, n, start, index, P.AT.val.data(), 40) * 1.01;
  return P;
}

Prepared prepare_structure(int32_t m, int32_t n, const int32_t* start, const int32_t* index, const double* value,
                           double offset, bool parallel) {
  Prepared P;
  P.n = n;
  P.m = m;
  P.offset = offset;
  const int32_t nnz = start[n];
  const bool par = parallel && nnz >= kParallelNnz;
  RowMap rm = row_map(m, n, start, index, par);
  P.R.assign(m, 1.0);
  P.Cs.assign(n, 1.0);
  P.A.rows = m;
  P.A.cols = n;
  P.A.val.resize(nnz);
#pragma omp parallel for schedule(static) if (par)
  for (int32_t e = 0; e < nnz; ++e) P.A.val[e] = value[rm.pos[e]];
  P.A.ptr = std::move(rm.ptr);
  P.A.idx = std::move(rm.col);
  P.AT.rows = n;
  P.AT.cols = m;
  P.AT.ptr.assign(start, start + n + 1);
  P.AT.idx.assign(index, index + nnz);
  P.AT.val.assign(value, value + nnz);
  return P;
}

void finish_scaling(Prepared& P, const double* rs, const double* cs, const double* cost, const double* row_lower,
                    const double* row_upper, bool rescale) {
  const int32_t m = P.m, n = P.n;
  for (int32_t i = 0; i < m; ++i) P.R[i] = pow2_round(rs[i]);
  for (int32_t j = 0; j < n; ++j) P.Cs[j] = pow2_round(cs[j]);
  P.beta = P.gamma = 1.0;
  if (rescale) {
    double cn = 0, bn = 0;
    for (int32_t j = 0; j < n; ++j) {
      const double t = cost[j] * P.Cs[j];
      cn += t * t;
    }
    for (int32_t i = 0; i < m; ++i) {
      if (finite_bound(row_lower[i])) {
        const double t = row_lower[i] * P.R[i];
        bn += t * t;
      }
      if (finite_bound(row_upper[i]) && row_upper[i] != row_lower[i]) {
        const double t = row_upper[i] * P.R[i];
        bn += t * t;
      }
    }
    P.gamma = 1.0 + std::sqrt(cn);
    P.beta = 1.0 + std::sqrt(bn);
  }
  P.rfac.resize(m);
  P.cfac.resize(n);
  for (int32_t i = 0; i < m; ++i) P.rfac[i] = P.beta / P.R[i];
  for (int32_t j = 0; j < n; ++j) P.cfac[j] = P.gamma / P.Cs[j];
}

}  // namespace b2p
