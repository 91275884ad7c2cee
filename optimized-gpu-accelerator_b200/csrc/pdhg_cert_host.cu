// Host side of the certifier: constraint-implied column bounds and the
// verdict on an OPTIMAL claim, batched over cases of one LP.
//
// * propagate(): activity-based bound propagation as the reference's
//   Propagator::propagate (src/mip/propagate.cpp:23-138) runs it for
//   continuous columns -- rows visited in queue order, bounds updated in
//   place, a tightening only when significant (1e-3 of the range) and relaxed
//   by 1e-7 (1 + |bound|), rows of changed columns queued for the next round,
//   activities not refreshed within a row, early return on a detected
//   infeasibility;
// * implied_bounds(): 30 rounds, then every tightened bound relaxed by
//   1e-6 (1 + |bound|) and the others restored (certifier.cpp:340-356);
// * certify(): the certifier's LP branch (certifier.cpp:218-262, 311-380):
//   relative column violations, Neumaier-compensated row activities summed
//   column by column, the objective summed from the offset, the safe dual
//   bound (the GPU kernel of pdhg_certify.cu), its implied-bounds retry, and
//   the gap/acceptance rules.
// Compiled with -ffp-contract=off like the reference, every operation is the
// same IEEE operation in the same order, so results are bit-identical.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "pdhg_host_common.h"
#include "pdhg_sched.h"

namespace b2p {
namespace {

constexpr double kInfD = std::numeric_limits<double>::infinity();
inline bool fin(double v) { return std::fabs(v) < 1e20; }

// Row-major copy of A in the reference's transpose order (columns ascending within a row).
struct RowMajor {
  std::vector<int32_t> ptr, idx;
  std::vector<double> val;
};

RowMajor row_major(const b2p_lp* lp) {
  const int32_t m = lp->num_rows, n = lp->num_cols, nnz = lp->start[n];
  RowMajor r;
  r.ptr.assign(static_cast<size_t>(m) + 1, 0);
  for (int32_t k = 0; k < nnz; ++k) r.ptr[lp->index[k] + 1]++;
  for (int32_t i = 0; i < m; ++i) r.ptr[i + 1] += r.ptr[i];
  r.idx.resize(nnz);
  r.val.resize(nnz);
  std::vector<int32_t> pos(r.ptr.begin(), r.ptr.end() - 1);
  for (int32_t j = 0; j < n; ++j)
    for (int32_t k = lp->start[j]; k < lp->start[j + 1]; ++k) {
      const int32_t p = pos[lp->index[k]]++;
      r.idx[p] = j;
      r.val[p] = lp->value[k];
    }
  return r;
}

// One case's vectors: the case's override, else the base model's.
struct CaseView {
  const double *c, *lo, *up, *rl, *ru;
};

CaseView case_view(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, int b) {
  const b2p_case* cs = num_cases > 0 ? &cases[b] : nullptr;
  auto pick = [&](const double* v, const double* base) { return (cs && v) ? v : base; };
  return CaseView{pick(cs ? cs->cost : nullptr, lp->col_cost), pick(cs ? cs->col_lower : nullptr, lp->col_lower),
                  pick(cs ? cs->col_upper : nullptr, lp->col_upper), pick(cs ? cs->row_lower : nullptr, lp->row_lower),
                  pick(cs ? cs->row_upper : nullptr, lp->row_upper)};
}

// Propagator::propagate for continuous columns; false = infeasibility detected
// (the bounds keep what was tightened before it, as in the reference).
bool propagate(const b2p_lp* lp, const RowMajor& R, const double* rl, const double* ru, std::vector<double>& lo,
               std::vector<double>& up, int max_rounds) {
  const int32_t m = lp->num_rows;
  std::vector<char> in_queue(m, 1);
  std::vector<int32_t> queue(m);
  for (int32_t i = 0; i < m; ++i) queue[i] = i;
  for (int round = 0; round < max_rounds && !queue.empty(); ++round) {
    std::vector<int32_t> next;
    for (int32_t i : queue) {
      in_queue[i] = 0;
      double minFin = 0, maxFin = 0;
      int minInf = 0, maxInf = 0;
      for (int32_t e = R.ptr[i]; e < R.ptr[i + 1]; ++e) {
        const int32_t j = R.idx[e];
        const double a = R.val[e];
        const double bmin = a > 0 ? lo[j] : up[j];
        const double bmax = a > 0 ? up[j] : lo[j];
        if (fin(bmin)) minFin += a * bmin;
        else ++minInf;
        if (fin(bmax)) maxFin += a * bmax;
        else ++maxInf;
      }
      const double L = rl[i], U = ru[i];
      const double scale = 1.0 + std::max(fin(L) ? std::fabs(L) : 0.0, fin(U) ? std::fabs(U) : 0.0);
      if (minInf == 0 && fin(U) && minFin > U + 1e-6 * scale) return false;
      if (maxInf == 0 && fin(L) && maxFin < L - 1e-6 * scale) return false;
      for (int32_t e = R.ptr[i]; e < R.ptr[i + 1]; ++e) {
        const int32_t j = R.idx[e];
        const double a = R.val[e];
        const double bmin = a > 0 ? lo[j] : up[j];
        const double bmax = a > 0 ? up[j] : lo[j];
        double resMin, resMax;
        bool resMinOk, resMaxOk;
        if (fin(bmin)) {
          resMinOk = minInf == 0;
          resMin = minFin - a * bmin;
        } else {
          resMinOk = minInf == 1;
          resMin = minFin;
        }
        if (fin(bmax)) {
          resMaxOk = maxInf == 0;
          resMax = maxFin - a * bmax;
        } else {
          resMaxOk = maxInf == 1;
          resMax = maxFin;
        }
        double newLo = -kInfD, newUp = kInfD;
        if (fin(U) && resMinOk) {
          const double lim = (U - resMin) / a;
          if (a > 0) newUp = lim;
          else newLo = lim;
        }
        if (fin(L) && resMaxOk) {
          const double lim = (L - resMax) / a;
          if (a > 0) newLo = std::max(newLo, lim);
          else newUp = std::min(newUp, lim);
        }
        bool changed = false;
        const double range = (fin(lo[j]) && fin(up[j])) ? up[j] - lo[j] : kInfD;
        if (fin(newLo)) {
          const double margin = 1e-7 * (1 + std::fabs(newLo));
          const double cand = newLo - margin;
          if (cand > lo[j] + 1e-3 * std::min(range, 1.0 + std::fabs(cand))) {
            lo[j] = cand;
            changed = true;
          }
        }
        if (fin(newUp)) {
          const double margin = 1e-7 * (1 + std::fabs(newUp));
          const double cand = newUp + margin;
          const double r2 = (fin(lo[j]) && fin(up[j])) ? up[j] - lo[j] : kInfD;
          if (cand < up[j] - 1e-3 * std::min(r2, 1.0 + std::fabs(cand))) {
            up[j] = cand;
            changed = true;
          }
        }
        if (lo[j] > up[j] + 1e-6 * (1 + std::fabs(lo[j]))) return false;
        if (lo[j] > up[j]) lo[j] = up[j];
        if (changed) {
          for (int32_t k = lp->start[j]; k < lp->start[j + 1]; ++k) {
            const int32_t r = lp->index[k];
            if (r != i && !in_queue[r]) {
              in_queue[r] = 1;
              next.push_back(r);
            }
          }
        }
      }
    }
    queue.swap(next);
  }
  return true;
}

// Constraint-implied bounds of one case, relaxed as the certifier relaxes them.
void implied_bounds(const b2p_lp* lp, const RowMajor& R, const CaseView& v, double* lo_out, double* up_out) {
  const int32_t n = lp->num_cols;
  std::vector<double> lo(v.lo, v.lo + n), up(v.up, v.up + n);
  propagate(lp, R, v.rl, v.ru, lo, up, 30);
  for (int32_t j = 0; j < n; ++j) {
    if (fin(lo[j]) && (!fin(v.lo[j]) || lo[j] > v.lo[j])) lo[j] -= 1e-6 * (1 + std::fabs(lo[j]));
    else lo[j] = v.lo[j];
    if (fin(up[j]) && (!fin(v.up[j]) || up[j] < v.up[j])) up[j] += 1e-6 * (1 + std::fabs(up[j]));
    else up[j] = v.up[j];
  }
  std::memcpy(lo_out, lo.data(), sizeof(double) * n);
  std::memcpy(up_out, up.data(), sizeof(double) * n);
}

// Lower bound of the exact a + b (interval.h:30-35 of the reference).
double add_down(double a, double b) {
  const double s = a + b;
  if (std::isinf(s) || std::isnan(s)) return s;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return e < 0 ? std::nextafter(s, -kInfD) : s;
}

// Neumaier / Kahan-Babuska compensated sum (CompensatedSum, interval.h:94-103).
struct CompSum {
  double sum = 0, comp = 0;
  void add(double v) {
    const double t = sum + v;
    if (std::fabs(sum) >= std::fabs(v)) comp += (sum - t) + v;
    else comp += (v - t) + sum;
    sum = t;
  }
  double value() const { return sum + comp; }
};

// checkPrimal (certifier.cpp:218-262) and the objective (core/model.cpp:74-84).
void check_primal(const b2p_lp* lp, const CaseView& v, const double* x, b2p_certificate& c) {
  const int32_t m = lp->num_rows, n = lp->num_cols;
  double colViol = 0, rowViol = 0;
  int32_t worst = -1;
  for (int32_t j = 0; j < n; ++j) {
    double q = 0;
    if (!std::isfinite(x[j])) {
      colViol = kInfD;
      continue;
    }
    if (fin(v.lo[j]) && x[j] < v.lo[j]) q = (v.lo[j] - x[j]) / (1 + std::fabs(v.lo[j]));
    if (fin(v.up[j]) && x[j] > v.up[j]) q = std::max(q, (x[j] - v.up[j]) / (1 + std::fabs(v.up[j])));
    colViol = std::max(colViol, q);
  }
  std::vector<CompSum> act(m);
  for (int32_t j = 0; j < n; ++j)
    for (int32_t k = lp->start[j]; k < lp->start[j + 1]; ++k) act[lp->index[k]].add(lp->value[k] * x[j]);
  for (int32_t i = 0; i < m; ++i) {
    const double r = act[i].value();
    double q = std::isfinite(r) ? 0.0 : kInfD;
    if (fin(v.rl[i]) && r < v.rl[i]) q = (v.rl[i] - r) / (1 + std::fabs(v.rl[i]));
    if (fin(v.ru[i]) && r > v.ru[i]) q = std::max(q, (r - v.ru[i]) / (1 + std::fabs(v.ru[i])));
    if (q > rowViol) {
      rowViol = q;
      worst = i;
    }
  }
  c.max_col_violation = colViol;
  c.max_row_violation = rowViol;
  c.max_primal_violation = std::max(colViol, rowViol);
  c.worst_row = worst;
  double f = lp->obj_offset;
  for (int32_t j = 0; j < n; ++j) f += v.c[j] * x[j];
  c.primal_objective = f;
}

template <class F>
void parallel_cases(int k, F&& f) {
  const int threads = std::max(1, std::min<int>(k, static_cast<int>(std::thread::hardware_concurrency())));
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  std::vector<std::exception_ptr> err(threads);
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      try {
        for (int b = next++; b < k; b = next++) f(b);
      } catch (...) {
        err[t] = std::current_exception();
      }
    });
  for (auto& th : pool) th.join();
  for (auto& e : err)
    if (e) std::rethrow_exception(e);
}

}  // namespace
}  // namespace b2p

using namespace b2p;

extern "C" int b2p_implied_bounds(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, double* col_lower_out,
                                  double* col_upper_out) {
  return guarded([&] {
    check_lp(lp);
    if (!col_lower_out || !col_upper_out) throw Error(B2P_ERR_INVALID, "NULL output");
    if (num_cases > 0 && !cases) throw Error(B2P_ERR_INVALID, "cases is NULL");
    const int k = num_cases > 0 ? num_cases : 1;
    const RowMajor R = row_major(lp);
    const size_t n = static_cast<size_t>(lp->num_cols);
    parallel_cases(k, [&](int b) {
      implied_bounds(lp, R, case_view(lp, cases, num_cases, b), col_lower_out + b * n, col_upper_out + b * n);
    });
  });
}

extern "C" int b2p_certify_lp(const b2p_lp* lp, const b2p_case* cases, int32_t num_cases, const double* x,
                              const double* row_dual, const b2p_cert_tolerances* tol, b2p_certificate* out) {
  return guarded([&] {
    check_lp(lp);
    if (!x || !row_dual || !out) throw Error(B2P_ERR_INVALID, "NULL argument");
    if (num_cases > 0 && !cases) throw Error(B2P_ERR_INVALID, "cases is NULL");
    const b2p_cert_tolerances t = tol ? *tol : b2p_cert_tolerances{1e-6, 1e-6, 1e-6};
    const int k = num_cases > 0 ? num_cases : 1;
    const size_t n = static_cast<size_t>(lp->num_cols);
    std::vector<b2p_certificate> cert(k);
    parallel_cases(k, [&](int b) {
      std::memset(&cert[b], 0, sizeof(b2p_certificate));
      check_primal(lp, case_view(lp, cases, num_cases, b), x + b * n, cert[b]);
    });
    std::vector<b2p_safe_bound> sb(k);
    const int rc = b2p_safe_dual_bound(lp, cases, num_cases, row_dual, sb.data());
    if (rc != B2P_OK) throw Error(rc, last_error());
    // retry with constraint-implied column bounds where the bound is -inf
    std::vector<int> retry;
    for (int b = 0; b < k; ++b)
      if (std::isinf(sb[b].bound)) retry.push_back(b);
    std::vector<char> used(k, 0);
    if (!retry.empty()) {
      const RowMajor R = row_major(lp);
      const size_t m = static_cast<size_t>(lp->num_rows);
      const int r = static_cast<int>(retry.size());
      std::vector<double> lo(r * n), up(r * n), y(r * m);
      std::vector<b2p_case> rc_cases(r);
      parallel_cases(r, [&](int q) {
        const int b = retry[q];
        const CaseView v = case_view(lp, cases, num_cases, b);
        implied_bounds(lp, R, v, lo.data() + q * n, up.data() + q * n);
        if (m) std::memcpy(y.data() + q * m, row_dual + b * m, sizeof(double) * m);
        rc_cases[q] = b2p_case{v.c, lo.data() + q * n, up.data() + q * n, v.rl, v.ru};
      });
      std::vector<b2p_safe_bound> sb2(r);
      const int rc2 = b2p_safe_dual_bound(lp, rc_cases.data(), r, y.data(), sb2.data());
      if (rc2 != B2P_OK) throw Error(rc2, last_error());
      for (int q = 0; q < r; ++q)
        if (!std::isinf(sb2[q].bound)) {
          sb[retry[q]] = sb2[q];
          used[retry[q]] = 1;
        }
    }
    for (int b = 0; b < k; ++b) {
      b2p_certificate& c = cert[b];
      const bool primal_ok = c.max_col_violation <= t.primal_feasibility && c.max_row_violation <= t.primal_feasibility;
      const double lb = std::isinf(sb[b].bound) ? -kInfD : add_down(add_down(sb[b].bound, 0.0), lp->obj_offset);
      c.used_implied_bounds = used[b];
      c.max_dual_violation = sb[b].max_dual_infeasibility;
      c.cost_perturbation = sb[b].cost_perturbation;
      c.infinite_terms = sb[b].infinite_terms;
      c.certified_gap = std::isinf(lb) ? kInfD : (c.primal_objective - lb) / std::max(1.0, std::fabs(c.primal_objective));
      c.safe_dual_bound = std::isinf(lb) ? -kInfD : lb;
      const bool rigorous = !std::isinf(lb);
      const bool dual_ok = rigorous ? c.certified_gap <= t.relative_gap
                                    : sb[b].max_dual_infeasibility <= t.dual_feasibility;
      c.accepted = primal_ok && dual_ok;
      out[b] = c;
    }
  });
}
