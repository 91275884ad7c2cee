/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the restarted-Halpern PDHG
 * path.  Nothing in the product links, loads or calls this file; the parity
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it as the
 * checker.
 *
 * A single-threaded C restatement of the reference's PDHG (PRAMANA,
 * src/pdhg/pdhg.cpp) with the same floating-point evaluation order, so that a
 * run of it is bit-for-bit the reference CpuBackend run on the same LP:
 *   - Ruiz + Pock-Chambolle scaling, power-of-two factors   src/lp/scaling.cpp:9-14, 97-139
 *   - applyScaling                                          src/lp/scaling.cpp:28-32
 *   - CSR of A / CSR of A^T                                  src/pdhg/pdhg.cpp:25-43, src/core/sparse.cpp:49-65
 *   - prepare (beta/gamma rescale, rfac/cfac, ||A||)        src/pdhg/pdhg.cpp:424-459
 *   - powerIteration (40 steps, x1.01)                      src/pdhg/pdhg.cpp:404-422
 *   - caseVectors                                           src/pdhg/pdhg.cpp:466-481
 *   - runPdhg: case setup, loop, check, restart, omega      src/pdhg/pdhg.cpp:483-687
 *   - CpuBackend ops mult/primal/dual/halpern/restart/kkt/diff2   src/pdhg/pdhg.cpp:93-205
 * The reference's CpuBackend splits rows/elements over threads but every
 * output element and every reduction is computed in the same order as here
 * (row sums are left to right; kkt and diff2 are sequential), so the results
 * do not depend on the thread count.
 *
 * Build: gcc -O2 -ffp-contract=off (oracle/Makefile); the reference is built
 * with -ffp-contract=off as well (CMakeLists.txt:17), so no FMA contraction.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define INF_BOUND_THRESHOLD 1e20 /* src/util/common.h:14 */

/* std::max / std::min semantics: max(a,b) = (a<b)?b:a, min(a,b) = (b<a)?b:a */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline int fin(double v) { return fabs(v) < INF_BOUND_THRESHOLD; }
static inline double sqr(double v) { return v * v; }

typedef struct {
  double tolerance;
  int64_t max_iterations;
  int32_t check_every;
  int32_t ruiz_iterations;
  int32_t pock_chambolle;
  int32_t rescale;
  double reflection;
  double time_limit; /* ignored by the oracle (no clock); kept for layout parity */
  /* > 0 and finite: every case's initial primal weight, in original-space
   * units (scaled weight = w beta / gamma).  No counterpart in the reference
   * (its weight starts at ||c|| / ||b||); it checks the engine's primal-weight
   * warm start.  The reference shim ignores it. */
  double primal_weight_start;
} oracle_options;

typedef struct {
  int32_t status; /* 1 Optimal, 5 TimeLimit, 6 IterationLimit (src/util/common.h:27-39) */
  int32_t pad;
  int64_t iterations;
  double objective;
  double dual_objective;
  double relative_kkt;
} oracle_case_result;

typedef struct {
  int64_t iterations;
  int32_t restarts;
  int32_t threads;
  double primal_weight;
  double spectral_norm;
  double setup_seconds;
  double solve_seconds;
  double primal_residual, dual_residual, gap;
} oracle_stats;

enum { ST_OPTIMAL = 1, ST_TIME_LIMIT = 5, ST_ITERATION_LIMIT = 6 };

typedef struct {
  int rows, cols;
  int *ptr, *idx;
  double* val;
} csr_t;

/* CSR of the matrix whose CSC (start/index/value) is given: the reference
 * builds it with SparseMatrix::transpose (src/core/sparse.cpp:49-65), which
 * lists each row's entries in increasing column order. */
static void csr_of_csc(int m, int n, const int* start, const int* index, const double* value, csr_t* out) {
  const int nnz = start[n];
  out->rows = m;
  out->cols = n;
  out->ptr = (int*)calloc((size_t)m + 1, sizeof(int));
  out->idx = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  out->val = (double*)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  for (int k = 0; k < nnz; ++k) out->ptr[index[k] + 1]++;
  for (int i = 0; i < m; ++i) out->ptr[i + 1] += out->ptr[i];
  int* pos = (int*)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  for (int i = 0; i < m; ++i) pos[i] = out->ptr[i];
  for (int j = 0; j < n; ++j)
    for (int k = start[j]; k < start[j + 1]; ++k) {
      int p = pos[index[k]]++;
      out->idx[p] = j;
      out->val[p] = value[k];
    }
  free(pos);
}

static void csr_free(csr_t* c) {
  free(c->ptr);
  free(c->idx);
  free(c->val);
}

/* pow2Round, src/lp/scaling.cpp:9-14 */
static double pow2_round(double v) {
  if (!(v > 0) || !isfinite(v)) return 1.0;
  int e = (int)lround(log2(v));
  if (e < -60) e = -60;
  if (e > 60) e = 60;
  return ldexp(1.0, e);
}

/* ruizScaling, src/lp/scaling.cpp:97-139 (rangeBefore/After are not needed). */
int oracle_ruiz_scaling(int m, int n, const int* start, const int* index, const double* value, int iterations,
                        int pock_chambolle, double* rs, double* cs) {
  for (int i = 0; i < m; ++i) rs[i] = 1.0;
  for (int j = 0; j < n; ++j) cs[j] = 1.0;
  double* rmax = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  double* cmax = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int it = 0; it < iterations; ++it) {
    for (int i = 0; i < m; ++i) rmax[i] = 0.0;
    for (int j = 0; j < n; ++j) {
      double c = 0;
      for (int k = start[j]; k < start[j + 1]; ++k) {
        double a = fabs(value[k]) * cs[j] * rs[index[k]];
        c = smax(c, a);
        rmax[index[k]] = smax(rmax[index[k]], a);
      }
      cmax[j] = c;
    }
    for (int i = 0; i < m; ++i)
      if (rmax[i] > 0) rs[i] /= sqrt(rmax[i]);
    for (int j = 0; j < n; ++j)
      if (cmax[j] > 0) cs[j] /= sqrt(cmax[j]);
  }
  if (pock_chambolle) {
    double* rsum = (double*)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
    double* csum = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int j = 0; j < n; ++j)
      for (int k = start[j]; k < start[j + 1]; ++k) {
        double a = fabs(value[k]) * cs[j] * rs[index[k]];
        csum[j] += a;
        rsum[index[k]] += a;
      }
    for (int i = 0; i < m; ++i)
      if (rsum[i] > 0) rs[i] /= sqrt(rsum[i]);
    for (int j = 0; j < n; ++j)
      if (csum[j] > 0) cs[j] /= sqrt(csum[j]);
    free(rsum);
    free(csum);
  }
  for (int i = 0; i < m; ++i) rs[i] = pow2_round(rs[i]);
  for (int j = 0; j < n; ++j) cs[j] = pow2_round(cs[j]);
  free(rmax);
  free(cmax);
  return 0;
}

/* powerIteration, src/pdhg/pdhg.cpp:404-422, with SparseMatrix::multiply and
 * multiplyTranspose (src/core/sparse.cpp:67-82) on the scaled CSC. */
double oracle_power_iteration(int m, int n, const int* start, const int* index, const double* value, int iters) {
  if (start[n] == 0) return 1.0;
  double* x = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double* y = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  double* z = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  const double x0 = 1.0 / sqrt((double)(n > 1 ? n : 1));
  for (int j = 0; j < n; ++j) x[j] = x0;
  double s = 1;
  for (int it = 0; it < iters; ++it) {
    for (int i = 0; i < m; ++i) y[i] = 0.0;
    for (int j = 0; j < n; ++j) {
      double xj = x[j];
      if (xj == 0.0) continue;
      xj *= 1.0;
      for (int k = start[j]; k < start[j + 1]; ++k) y[index[k]] += value[k] * xj;
    }
    for (int j = 0; j < n; ++j) z[j] = 0.0;
    for (int j = 0; j < n; ++j) {
      double t = 0;
      for (int k = start[j]; k < start[j + 1]; ++k) t += value[k] * y[index[k]];
      z[j] += 1.0 * t;
    }
    double nz = 0;
    for (int j = 0; j < n; ++j) nz += z[j] * z[j];
    nz = sqrt(nz);
    if (nz == 0) {
      s = 1.0;
      break;
    }
    s = sqrt(nz);
    for (int j = 0; j < n; ++j) x[j] = z[j] / nz;
  }
  free(x);
  free(y);
  free(z);
  return s;
}

/* CpuBackend::mult, src/pdhg/pdhg.cpp:93-103: out(i,q) = sum_p val[p]*in(idx[p],q), left to right. */
void oracle_csr_mult(int rows, int k, const int* ptr, const int* idx, const double* val, const double* in,
                     double* out) {
  for (int i = 0; i < rows; ++i)
    for (int q = 0; q < k; ++q) {
      double s = 0;
      for (int p = ptr[i]; p < ptr[i + 1]; ++p) s += val[p] * in[(size_t)idx[p] * k + q];
      out[(size_t)i * k + q] = s;
    }
}

/* Vector slots, src/pdhg/pdhg.cpp:45 */
enum { X, XP, X0, ATY, ATYP, C, LO, UP, Y, YP, Y0, AX, AXP, AX0, RL, RU, NV };

typedef struct {
  int n, m, k;
  csr_t A, AT;
  double *rfac, *cfac;
  double* v[NV];
  int* iter;
  double *tau, *sigma;
} backend_t;

static void be_primal(backend_t* be) {
  const int k = be->k;
  double *x = be->v[X], *aty = be->v[ATY], *c = be->v[C], *lo = be->v[LO], *up = be->v[UP], *xp = be->v[XP];
  const size_t len = (size_t)be->n * k;
  for (size_t t = 0; t < len; ++t) {
    double v = x[t] - be->tau[t % k] * (c[t] - aty[t]);
    v = smax(v, lo[t]);
    v = smin(v, up[t]);
    xp[t] = v;
  }
}

static void be_dual(backend_t* be) {
  const int k = be->k;
  double *y = be->v[Y], *axp = be->v[AXP], *ax = be->v[AX], *rl = be->v[RL], *ru = be->v[RU], *yp = be->v[YP];
  const size_t len = (size_t)be->m * k;
  for (size_t t = 0; t < len; ++t) {
    double s = be->sigma[t % k];
    double v = y[t] - s * (2.0 * axp[t] - ax[t]);
    double w = -v / s;
    w = smax(w, rl[t]);
    w = smin(w, ru[t]);
    yp[t] = v + s * w;
  }
}

static void be_halpern_one(backend_t* be, int z, int zp, int z0, size_t len, double rho) {
  const int k = be->k;
  double *a = be->v[z], *p = be->v[zp], *o = be->v[z0];
  for (size_t t = 0; t < len; ++t) {
    double kk2 = (double)be->iter[t % k];
    double lam = (kk2 + 1.0) / (kk2 + 2.0);
    a[t] = lam * ((1.0 + rho) * p[t] - rho * a[t]) + (1.0 - lam) * o[t];
  }
}

static void be_halpern(backend_t* be, double rho) {
  be_halpern_one(be, X, XP, X0, (size_t)be->n * be->k, rho);
  be_halpern_one(be, Y, YP, Y0, (size_t)be->m * be->k, rho);
  be_halpern_one(be, AX, AXP, AX0, (size_t)be->m * be->k, rho);
  for (int b = 0; b < be->k; ++b) be->iter[b]++;
}

static void be_restart(backend_t* be, const int* mask) {
  const int k = be->k;
  const int src[3] = {XP, YP, AXP}, d1[3] = {X, Y, AX}, d2[3] = {X0, Y0, AX0};
  const size_t len[3] = {(size_t)be->n * k, (size_t)be->m * k, (size_t)be->m * k};
  for (int q = 0; q < 3; ++q) {
    double *s = be->v[src[q]], *a = be->v[d1[q]], *b = be->v[d2[q]];
    for (size_t t = 0; t < len[q]; ++t)
      if (mask[t % k]) a[t] = b[t] = s[t];
  }
  for (int b = 0; b < k; ++b)
    if (mask[b]) be->iter[b] = 0;
}

/* CpuBackend::kkt, src/pdhg/pdhg.cpp:166-197 */
static void be_kkt(backend_t* be, double* r3, double* c3) {
  const int k = be->k, m = be->m, n = be->n;
  for (int q = 0; q < 3 * k; ++q) r3[q] = c3[q] = 0.0;
  double *axp = be->v[AXP], *rl = be->v[RL], *ru = be->v[RU], *yp = be->v[YP];
  for (int i = 0; i < m; ++i)
    for (int b = 0; b < k; ++b) {
      size_t t = (size_t)i * k + b;
      double a = axp[t];
      double res = (smax(rl[t] - a, 0.0) + smax(a - ru[t], 0.0)) * be->rfac[i];
      r3[3 * b] += res * res;
      double y = yp[t];
      if (y > 0 && rl[t] > -1e300)
        r3[3 * b + 1] += y * rl[t];
      else if (y < 0 && ru[t] < 1e300)
        r3[3 * b + 1] += y * ru[t];
      r3[3 * b + 2] += y * y;
    }
  double *xp = be->v[XP], *c = be->v[C], *atyp = be->v[ATYP], *lo = be->v[LO], *up = be->v[UP];
  for (int j = 0; j < n; ++j)
    for (int b = 0; b < k; ++b) {
      size_t t = (size_t)j * k + b;
      double d = c[t] - atyp[t];
      int hl = lo[t] > -1e300, hu = up[t] < 1e300;
      double res = 0;
      if (!hl && !hu)
        res = fabs(d);
      else if (!hl)
        res = smax(d, 0.0);
      else if (!hu)
        res = smax(-d, 0.0);
      res *= be->cfac[j];
      c3[3 * b] += res * res;
      c3[3 * b + 1] += c[t] * xp[t];
      if (d > 0 && hl)
        c3[3 * b + 2] += d * lo[t];
      else if (d < 0 && hu)
        c3[3 * b + 2] += d * up[t];
    }
}

/* CpuBackend::diff2, src/pdhg/pdhg.cpp:198-205 */
static void be_diff2(backend_t* be, int a, int b, double* out) {
  const int k = be->k;
  const size_t len = (size_t)(a >= Y ? be->m : be->n) * k;
  for (int q = 0; q < k; ++q) out[q] = 0.0;
  double *va = be->v[a], *vb = be->v[b];
  for (size_t t = 0; t < len; ++t) {
    double d = va[t] - vb[t];
    out[t % k] += d * d;
  }
}

static const double* pick(const double* const* arr, int b, const double* base) {
  return (arr && arr[b]) ? arr[b] : base;
}

/* runPdhg + solvePdhg / solvePdhgBatch, src/pdhg/pdhg.cpp:483-728.
 * k <= 0 means a single solve of the base model (solvePdhg). */
int oracle_pdhg_solve(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                      const double* colLower, const double* colUpper, const double* rowLower,
                      const double* rowUpper, double offset, int kIn, const double* const* caseCost,
                      const double* const* caseColLower, const double* const* caseColUpper,
                      const double* const* caseRowLower, const double* const* caseRowUpper,
                      const oracle_options* o, double* xOut, double* yOut, oracle_case_result* res,
                      oracle_stats* st) {
  const int k = kIn <= 0 ? 1 : kIn;
  const int nnz = start[n];
  memset(st, 0, sizeof(*st));
  st->threads = 1;

  /* ---- prepare (src/pdhg/pdhg.cpp:424-459) ---- */
  double* R = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  double* Cs = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  if (o->ruiz_iterations > 0 && nnz > 0) {
    oracle_ruiz_scaling(m, n, start, index, value, o->ruiz_iterations, o->pock_chambolle, R, Cs);
  } else {
    for (int i = 0; i < m; ++i) R[i] = 1.0;
    for (int j = 0; j < n; ++j) Cs[j] = 1.0;
  }
  double* sval = (double*)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  for (int j = 0; j < n; ++j)
    for (int q = start[j]; q < start[j + 1]; ++q) sval[q] = value[q] * (R[index[q]] * Cs[j]);
  double beta = 1, gamma = 1;
  if (o->rescale) {
    double cn = 0, bn = 0;
    for (int j = 0; j < n; ++j) cn += sqr(cost[j] * Cs[j]);
    for (int i = 0; i < m; ++i) {
      if (fin(rowLower[i])) bn += sqr(rowLower[i] * R[i]);
      if (fin(rowUpper[i]) && rowUpper[i] != rowLower[i]) bn += sqr(rowUpper[i] * R[i]);
    }
    gamma = 1.0 + sqrt(cn);
    beta = 1.0 + sqrt(bn);
  }
  backend_t be;
  memset(&be, 0, sizeof(be));
  be.n = n;
  be.m = m;
  be.k = k;
  csr_of_csc(m, n, start, index, sval, &be.A);
  /* CSR of A^T == CSC of A (pdhg.cpp:35-43) */
  be.AT.rows = n;
  be.AT.cols = m;
  be.AT.ptr = (int*)malloc(sizeof(int) * ((size_t)n + 1));
  memcpy(be.AT.ptr, start, sizeof(int) * ((size_t)n + 1));
  be.AT.idx = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  memcpy(be.AT.idx, index, sizeof(int) * (size_t)nnz);
  be.AT.val = sval;
  be.rfac = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  be.cfac = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < m; ++i) be.rfac[i] = beta / R[i];
  for (int j = 0; j < n; ++j) be.cfac[j] = gamma / Cs[j];
  const double normA = oracle_power_iteration(m, n, start, index, sval, 40) * 1.01;

  for (int v = 0; v < NV; ++v) be.v[v] = (double*)calloc((size_t)(v >= Y ? m : n) * k + 1, sizeof(double));
  be.iter = (int*)calloc((size_t)k, sizeof(int));
  be.tau = (double*)calloc((size_t)k, sizeof(double));
  be.sigma = (double*)calloc((size_t)k, sizeof(double));

  /* ---- case data in scaled space, k-interleaved (pdhg.cpp:506-545) ---- */
  double* omega = (double*)malloc(sizeof(double) * (size_t)k);
  double* cNorm = (double*)malloc(sizeof(double) * (size_t)k);
  double* rhsNorm = (double*)malloc(sizeof(double) * (size_t)k);
  for (int b = 0; b < k; ++b) {
    const int useCase = kIn > 0;
    const double* cc = useCase ? pick(caseCost, b, cost) : cost;
    const double* cl = useCase ? pick(caseColLower, b, colLower) : colLower;
    const double* cu = useCase ? pick(caseColUpper, b, colUpper) : colUpper;
    const double* rl = useCase ? pick(caseRowLower, b, rowLower) : rowLower;
    const double* ru = useCase ? pick(caseRowUpper, b, rowUpper) : rowUpper;
    double s = 0;
    for (int j = 0; j < n; ++j) s += cc[j] * cc[j];
    cNorm[b] = sqrt(s);
    s = 0;
    for (int i = 0; i < m; ++i) {
      if (fin(rl[i])) s += rl[i] * rl[i];
      if (fin(ru[i]) && ru[i] != rl[i]) s += ru[i] * ru[i];
    }
    rhsNorm[b] = sqrt(s);
    omega[b] = 1.0;
    double cn = 0, bn = 0;
    for (int j = 0; j < n; ++j) {
      size_t t = (size_t)j * k + b;
      be.v[C][t] = cc[j] * Cs[j] / gamma;
      be.v[LO][t] = fin(cl[j]) ? cl[j] / Cs[j] / beta : -HUGE_VAL;
      be.v[UP][t] = fin(cu[j]) ? cu[j] / Cs[j] / beta : HUGE_VAL;
      be.v[X][t] = smin(smax(0.0, be.v[LO][t]), be.v[UP][t]);
      cn += be.v[C][t] * be.v[C][t];
    }
    for (int i = 0; i < m; ++i) {
      size_t t = (size_t)i * k + b;
      be.v[RL][t] = fin(rl[i]) ? rl[i] * R[i] / beta : -HUGE_VAL;
      be.v[RU][t] = fin(ru[i]) ? ru[i] * R[i] / beta : HUGE_VAL;
      if (fin(be.v[RL][t])) bn += be.v[RL][t] * be.v[RL][t];
      if (fin(be.v[RU][t]) && be.v[RU][t] != be.v[RL][t]) bn += be.v[RU][t] * be.v[RU][t];
    }
    if (cn > 1e-20 && bn > 1e-20) omega[b] = sqrt(cn) / sqrt(bn);
    if (isfinite(o->primal_weight_start) && o->primal_weight_start > 0) omega[b] = o->primal_weight_start * beta / gamma;
  }
  memcpy(be.v[X0], be.v[X], sizeof(double) * (size_t)n * k);
  oracle_csr_mult(m, k, be.A.ptr, be.A.idx, be.A.val, be.v[X], be.v[AX]);
  memcpy(be.v[AX0], be.v[AX], sizeof(double) * (size_t)m * k);
  const double eta = 0.998 / normA;
  st->spectral_norm = normA;
  for (int b = 0; b < k; ++b) {
    be.tau[b] = eta / omega[b];
    be.sigma[b] = eta * omega[b];
  }

  /* ---- iterations (pdhg.cpp:560-662) ---- */
  char* done = (char*)calloc((size_t)k, 1);
  double* fpRestart = (double*)malloc(sizeof(double) * (size_t)k);
  double* fpPrev = (double*)malloc(sizeof(double) * (size_t)k);
  int64_t* sinceRestart = (int64_t*)calloc((size_t)k, sizeof(int64_t));
  for (int b = 0; b < k; ++b) fpRestart[b] = fpPrev[b] = INFINITY;
  int remaining = k;
  int64_t it = 0;
  double* r3 = (double*)calloc((size_t)3 * k, sizeof(double));
  double* c3 = (double*)calloc((size_t)3 * k, sizeof(double));
  double* dx2 = (double*)calloc((size_t)k, sizeof(double));
  double* dy2 = (double*)calloc((size_t)k, sizeof(double));
  double* ax2 = (double*)calloc((size_t)k, sizeof(double));
  double* ay2 = (double*)calloc((size_t)k, sizeof(double));
  int* mask = (int*)calloc((size_t)k, sizeof(int));
  const double scaleObj = beta * gamma;

#define EXTRACT(b_, status_, kkt_, pobj_, dobj_)                                               \
  do {                                                                                       \
    const int bb = (b_);                                                                     \
    for (int j = 0; j < n; ++j) xOut[(size_t)bb * n + j] = be.v[XP][(size_t)j * k + bb] * Cs[j] * beta; \
    for (int i = 0; i < m; ++i) yOut[(size_t)bb * m + i] = be.v[YP][(size_t)i * k + bb] * R[i] * gamma; \
    res[bb].status = (status_);                                                              \
    res[bb].iterations = it;                                                                 \
    res[bb].relative_kkt = (kkt_);                                                           \
    res[bb].objective = (pobj_) + offset;                                                    \
    res[bb].dual_objective = (dobj_) + offset;                                               \
  } while (0)

  for (; it < o->max_iterations; ++it) {
    oracle_csr_mult(n, k, be.AT.ptr, be.AT.idx, be.AT.val, be.v[Y], be.v[ATY]);
    be_primal(&be);
    oracle_csr_mult(m, k, be.A.ptr, be.A.idx, be.A.val, be.v[XP], be.v[AXP]);
    be_dual(&be);
    const int check = ((it + 1) % o->check_every) == 0 || it + 1 == o->max_iterations;
    int anyRestart = 0;
    if (check) {
      oracle_csr_mult(n, k, be.AT.ptr, be.AT.idx, be.AT.val, be.v[YP], be.v[ATYP]);
      be_kkt(&be, r3, c3);
      be_diff2(&be, X, XP, dx2);
      be_diff2(&be, Y, YP, dy2);
      for (int b = 0; b < k; ++b) mask[b] = 0;
      for (int b = 0; b < k; ++b) {
        if (done[b]) continue;
        double pobj = c3[3 * b + 1] * scaleObj;
        double dobj = (r3[3 * b + 1] + c3[3 * b + 2]) * scaleObj;
        double pres = sqrt(r3[3 * b]), dres = sqrt(c3[3 * b]);
        double relP = pres / (1.0 + rhsNorm[b]);
        double relD = dres / (1.0 + cNorm[b]);
        double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
        double kktErr = smax(relP, smax(relD, gap));
        if (k == 1) {
          st->primal_residual = relP;
          st->dual_residual = relD;
          st->gap = gap;
        }
        if (relP <= o->tolerance && relD <= o->tolerance && gap <= o->tolerance) {
          EXTRACT(b, ST_OPTIMAL, kktErr, pobj, dobj);
          done[b] = 1;
          --remaining;
          continue;
        }
        sinceRestart[b] += o->check_every;
        double fp = sqrt(omega[b] * dx2[b] + dy2[b] / omega[b]);
        if (fpRestart[b] == INFINITY) fpRestart[b] = fp;
        int restart = fp <= 0.2 * fpRestart[b] || (fp <= 0.8 * fpRestart[b] && fp > fpPrev[b]) ||
                      sinceRestart[b] >= (int64_t)(0.36 * (double)(it + 1));
        fpPrev[b] = fp;
        if (restart) {
          mask[b] = 1;
          anyRestart = 1;
        }
      }
      if (anyRestart) {
        be_diff2(&be, XP, X0, ax2);
        be_diff2(&be, YP, Y0, ay2);
        for (int b = 0; b < k; ++b) {
          if (!mask[b]) continue;
          double dxn = sqrt(ax2[b]), dyn = sqrt(ay2[b]);
          if (dxn > 1e-10 && dyn > 1e-10) omega[b] = exp(0.5 * log(dyn / dxn) + 0.5 * log(omega[b]));
          fpRestart[b] = sqrt(omega[b] * dx2[b] + dy2[b] / omega[b]);
          fpPrev[b] = INFINITY;
          sinceRestart[b] = 0;
          st->restarts++;
        }
        for (int b = 0; b < k; ++b) {
          be.tau[b] = eta / omega[b];
          be.sigma[b] = eta * omega[b];
        }
      }
      if (remaining == 0) break;
    }
    be_halpern(&be, o->reflection);
    if (check && anyRestart) be_restart(&be, mask);
  }
  st->iterations = it + (remaining == 0 ? 1 : 0);
  st->primal_weight = omega[0];
  if (remaining > 0) {
    oracle_csr_mult(n, k, be.AT.ptr, be.AT.idx, be.AT.val, be.v[YP], be.v[ATYP]);
    be_kkt(&be, r3, c3);
    for (int b = 0; b < k; ++b) {
      if (done[b]) continue;
      double pobj = c3[3 * b + 1] * scaleObj, dobj = (r3[3 * b + 1] + c3[3 * b + 2]) * scaleObj;
      double relP = sqrt(r3[3 * b]) / (1 + rhsNorm[b]), relD = sqrt(c3[3 * b]) / (1 + cNorm[b]);
      double gap = fabs(pobj - dobj) / (1 + fabs(pobj) + fabs(dobj));
      EXTRACT(b, ST_ITERATION_LIMIT, smax(relP, smax(relD, gap)), pobj, dobj);
    }
  }
#undef EXTRACT

  for (int v = 0; v < NV; ++v) free(be.v[v]);
  free(be.iter);
  free(be.tau);
  free(be.sigma);
  csr_free(&be.A);
  free(be.AT.ptr);
  free(be.AT.idx); /* AT.val == sval */
  free(sval);
  free(be.rfac);
  free(be.cfac);
  free(R);
  free(Cs);
  free(omega);
  free(cNorm);
  free(rhsNorm);
  free(done);
  free(fpRestart);
  free(fpPrev);
  free(sinceRestart);
  free(r3);
  free(c3);
  free(dx2);
  free(dy2);
  free(ax2);
  free(ay2);
  free(mask);
  return 0;
}
