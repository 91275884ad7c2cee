// TEST INFRASTRUCTURE ONLY (the oracle). Never linked into the product.
//
// C-ABI shim over the reference's own CPU PDHG, compiled together with the
// reference's unmodified sources (see oracle/Makefile) into
// oracle/_ref/libpramana_ref.so.  It lets the parity tests and the CPU
// baseline call, through ctypes:
//   - pramana::solvePdhg / solvePdhgBatch with useGpu=false, i.e. the
//     multithreaded CpuBackend            (src/pdhg/pdhg.cpp:712-728, 75-214)
//   - pramana::safeDualBound, the outward-rounded Neumaier-Shcherbina bound
//                                          (src/cert/certifier.h:93)
//   - pramana::ruizScaling                 (src/lp/scaling.cpp:97-139)
//   - pramana::crossover (src/lp/crossover.cpp) from a primal-dual point, and
//     the dual simplex from scratch (src/lp/simplex.cpp), for the handoff
//   - pramana::certify of an OPTIMAL LP claim (src/cert/certifier.cpp:208-380)
//     and its constraint-implied column bounds (Propagator, src/mip/propagate.cpp)
//   - the router's features and decision (src/router/router.cpp) and timed
//     solves by the dual simplex and the interior-point method (src/ipm/ipm.cpp),
//     the CPU engines a router calibration compares the GPU engine with
//   - the LP that solve() hands to its LP engines for an MPS file: readMps
//     (src/io/mps.cpp), minimisation form, Presolver (src/presolve/presolve.cpp),
//     the inputs of the reference's published PDHG runs
// The GPU path of the reference is switched off (PRAMANA_DISABLE_GPU) so that
// loading this library never brings up a CUDA context or NVRTC.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "cert/certifier.h"
#include "core/model.h"
#include "io/mps.h"
#include "ipm/ipm.h"
#include "lp/crossover.h"
#include "lp/scaling.h"
#include "lp/simplex.h"
#include "mip/propagate.h"
#include "pdhg/pdhg.h"
#include "presolve/presolve.h"
#include "router/router.h"
#include "util/log.h"
#include "util/parallel.h"
#include "util/timer.h"

using namespace pramana;

namespace {
std::string gErr;

Model buildModel(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                 const double* colLower, const double* colUpper, const double* rowLower, const double* rowUpper,
                 double offset) {
  Model lp;
  lp.objOffset = offset;
  lp.A.numRows = m;
  lp.A.numCols = n;
  lp.A.start.assign(start, start + n + 1);
  const int nnz = start[n];
  lp.A.index.assign(index, index + nnz);
  lp.A.value.assign(value, value + nnz);
  lp.colCost.assign(cost, cost + n);
  lp.colLower.assign(colLower, colLower + n);
  lp.colUpper.assign(colUpper, colUpper + n);
  lp.rowLower.assign(rowLower, rowLower + m);
  lp.rowUpper.assign(rowUpper, rowUpper + m);
  lp.colType.assign(n, VarType::Continuous);
  return lp;
}

Model gLoaded;          // the model of the last ref_load_mps, until ref_model_arrays copies it out
bool gLoadedMax = false;  // whether that file's objective sense was maximise

std::vector<double> vecOrEmpty(const double* p, int len) {
  return p ? std::vector<double>(p, p + len) : std::vector<double>();
}
}  // namespace

extern "C" {

struct ref_options {
  double tolerance;
  int64_t max_iterations;
  int32_t check_every;
  int32_t ruiz_iterations;
  int32_t pock_chambolle;
  int32_t rescale;
  double reflection;
  double time_limit;  // <= 0: no limit
};

struct ref_case_result {
  int32_t status;  // pramana::Status numbering (src/util/common.h:27-39)
  int32_t pad;
  int64_t iterations;
  double objective;
  double dual_objective;
  double relative_kkt;
};

struct ref_stats {
  int64_t iterations;
  int32_t restarts;
  int32_t threads;
  double primal_weight;
  double spectral_norm;
  double setup_seconds;
  double solve_seconds;
  double primal_residual, dual_residual, gap;
};

const char* ref_last_error() { return gErr.c_str(); }

void ref_set_threads(int n) {
  ThreadPool::setThreads(n);
  Log::setLevel(LogLevel::Error);
}

int ref_threads() { return ThreadPool::instance().threads(); }

// cost/colLower/... of case b: cases_x[b] (NULL = base model's vector).
}  // extern "C"

namespace {
std::string gBackend;        // backend of the last solve ("cpu" / "gpu")
double gKernelSeconds = 0;   // its PdhgStats::kernelSeconds

int solve_impl(bool gpu, int m, int n, const int* start, const int* index, const double* value, const double* cost,
               const double* colLower, const double* colUpper, const double* rowLower, const double* rowUpper,
               double offset, int k, const double* const* caseCost, const double* const* caseColLower,
               const double* const* caseColUpper, const double* const* caseRowLower,
               const double* const* caseRowUpper, const ref_options* o, double* xOut, double* yOut,
               ref_case_result* res, ref_stats* st) {
  try {
    if (gpu)
      unsetenv("PRAMANA_DISABLE_GPU");
    else
      setenv("PRAMANA_DISABLE_GPU", "1", 1);
    Log::setLevel(LogLevel::Error);
    Model lp = buildModel(m, n, start, index, value, cost, colLower, colUpper, rowLower, rowUpper, offset);
    PdhgOptions po;
    po.tolerance = o->tolerance;
    po.maxIterations = o->max_iterations;
    po.checkEvery = o->check_every;
    po.ruizIterations = o->ruiz_iterations;
    po.pockChambolle = o->pock_chambolle != 0;
    po.rescaleObjectiveAndBounds = o->rescale != 0;
    po.reflection = o->reflection;
    po.useGpu = gpu;
    Deadline dl(o->time_limit);
    std::vector<PdhgResult> rr;
    PdhgStats bst;
    if (k <= 0) {
      rr.push_back(solvePdhg(lp, po, o->time_limit > 0 ? &dl : nullptr));
      bst = rr[0].stats;
    } else {
      std::vector<LpCase> cases(k);
      for (int b = 0; b < k; ++b) {
        cases[b].cost = vecOrEmpty(caseCost ? caseCost[b] : nullptr, n);
        cases[b].colLower = vecOrEmpty(caseColLower ? caseColLower[b] : nullptr, n);
        cases[b].colUpper = vecOrEmpty(caseColUpper ? caseColUpper[b] : nullptr, n);
        cases[b].rowLower = vecOrEmpty(caseRowLower ? caseRowLower[b] : nullptr, m);
        cases[b].rowUpper = vecOrEmpty(caseRowUpper ? caseRowUpper[b] : nullptr, m);
      }
      rr = solvePdhgBatch(lp, cases, po, o->time_limit > 0 ? &dl : nullptr, &bst);
    }
    for (size_t b = 0; b < rr.size(); ++b) {
      const PdhgResult& r = rr[b];
      res[b].status = static_cast<int32_t>(r.status);
      res[b].iterations = r.iterations;
      res[b].objective = r.objective;
      res[b].dual_objective = r.dualObjective;
      res[b].relative_kkt = r.relativeKkt;
      if (xOut) std::memcpy(xOut + b * static_cast<size_t>(n), r.x.data(), sizeof(double) * n);
      if (yOut) std::memcpy(yOut + b * static_cast<size_t>(m), r.rowDual.data(), sizeof(double) * m);
    }
    if (st) {
      st->iterations = bst.iterations;
      st->restarts = bst.restarts;
      st->threads = ThreadPool::instance().threads();
      st->primal_weight = bst.primalWeight;
      st->spectral_norm = bst.spectralNorm;
      st->setup_seconds = bst.setupSeconds;
      st->solve_seconds = bst.solveSeconds;
      st->primal_residual = bst.primalResidual;
      st->dual_residual = bst.dualResidual;
      st->gap = bst.gap;
    }
    gBackend = bst.backend;
    gKernelSeconds = bst.kernelSeconds;
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}
}  // namespace

extern "C" {

// solvePdhg / solvePdhgBatch on the reference's multithreaded CpuBackend.
int ref_pdhg_solve(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                   const double* colLower, const double* colUpper, const double* rowLower, const double* rowUpper,
                   double offset, int k, const double* const* caseCost, const double* const* caseColLower,
                   const double* const* caseColUpper, const double* const* caseRowLower,
                   const double* const* caseRowUpper, const ref_options* o, double* xOut, double* yOut,
                   ref_case_result* res, ref_stats* st) {
  return solve_impl(false, m, n, start, index, value, cost, colLower, colUpper, rowLower, rowUpper, offset, k,
                    caseCost, caseColLower, caseColUpper, caseRowLower, caseRowUpper, o, xOut, yOut, res, st);
}

// The same on the reference's own GpuBackend (its NVRTC-compiled kernels,
// src/pdhg/kernels.cpp, through its driver-API context), where a GPU and
// NVRTC are present; the reference falls back to its CPU backend otherwise,
// which ref_last_backend reports.
int ref_pdhg_solve_gpu(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                       const double* colLower, const double* colUpper, const double* rowLower,
                       const double* rowUpper, double offset, int k, const double* const* caseCost,
                       const double* const* caseColLower, const double* const* caseColUpper,
                       const double* const* caseRowLower, const double* const* caseRowUpper, const ref_options* o,
                       double* xOut, double* yOut, ref_case_result* res, ref_stats* st) {
  return solve_impl(true, m, n, start, index, value, cost, colLower, colUpper, rowLower, rowUpper, offset, k,
                    caseCost, caseColLower, caseColUpper, caseRowLower, caseRowUpper, o, xOut, yOut, res, st);
}

const char* ref_last_backend() { return gBackend.c_str(); }
double ref_last_kernel_seconds() { return gKernelSeconds; }

// Outward-rounded lower bound on min c^T x over the given boxes, valid for any y.
// extra (optional): maxDualInfeasibility, rowProjection, costPerturbation
int ref_safe_dual_bound(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                        const double* colLower, const double* colUpper, const double* rowLower,
                        const double* rowUpper, const double* y, double* bound, int* infiniteTerms, double* extra) {
  try {
    SparseMatrix A(m, n);
    A.start.assign(start, start + n + 1);
    A.index.assign(index, index + start[n]);
    A.value.assign(value, value + start[n]);
    SafeBoundResult sb = safeDualBound(A, std::vector<double>(cost, cost + n),
                                       std::vector<double>(colLower, colLower + n),
                                       std::vector<double>(colUpper, colUpper + n),
                                       std::vector<double>(rowLower, rowLower + m),
                                       std::vector<double>(rowUpper, rowUpper + m), std::vector<double>(y, y + m));
    *bound = sb.bound;
    if (infiniteTerms) *infiniteTerms = sb.infiniteTerms;
    if (extra) {
      extra[0] = sb.maxDualInfeasibility;
      extra[1] = sb.rowProjection;
      extra[2] = sb.costPerturbation;
    }
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

// The certifier's constraint-implied column bounds (certifier.cpp:346-356):
// Propagator on the continuous relaxation, 30 rounds, tightened bounds relaxed.
int ref_implied_bounds(int m, int n, const int* start, const int* index, const double* value,
                       const double* colLower, const double* colUpper, const double* rowLower, const double* rowUpper,
                       double* loOut, double* upOut) {
  try {
    std::vector<double> zero(n, 0.0);
    Model relaxed = buildModel(m, n, start, index, value, zero.data(), colLower, colUpper, rowLower, rowUpper, 0.0);
    Propagator prop;
    prop.setup(relaxed);
    std::vector<double> lo = relaxed.colLower, up = relaxed.colUpper;
    prop.propagate(lo, up, 30);
    for (int j = 0; j < n; ++j) {
      if (std::fabs(lo[j]) < kInfBoundThreshold &&
          (!(std::fabs(relaxed.colLower[j]) < kInfBoundThreshold) || lo[j] > relaxed.colLower[j]))
        lo[j] -= 1e-6 * (1 + std::fabs(lo[j]));
      else lo[j] = relaxed.colLower[j];
      if (std::fabs(up[j]) < kInfBoundThreshold &&
          (!(std::fabs(relaxed.colUpper[j]) < kInfBoundThreshold) || up[j] < relaxed.colUpper[j]))
        up[j] += 1e-6 * (1 + std::fabs(up[j]));
      else up[j] = relaxed.colUpper[j];
    }
    std::memcpy(loOut, lo.data(), sizeof(double) * n);
    std::memcpy(upOut, up.data(), sizeof(double) * n);
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

// pramana::certify of an OPTIMAL claim (x, y) on a min-form LP.
// out: accepted, primalObjective, safeDualBound, certifiedGap, maxPrimalViolation,
//      column violation, row violation, maxDualViolation, costPerturbation,
//      used implied bounds (0/1)
int ref_certify_lp(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                   const double* colLower, const double* colUpper, const double* rowLower, const double* rowUpper,
                   double offset, const double* x, const double* y, const double* tol3, double* out) {
  try {
    Model lp = buildModel(m, n, start, index, value, cost, colLower, colUpper, rowLower, rowUpper, offset);
    SolutionClaim claim;
    claim.status = Status::Optimal;
    claim.x.assign(x, x + n);
    claim.rowDual.assign(y, y + m);
    CertTolerances tol;
    if (tol3) {
      tol.primalFeas = tol3[0];
      tol.dualFeas = tol3[1];
      tol.relGap = tol3[2];
    }
    Certificate c = certify(lp, claim, tol);
    out[0] = c.accepted ? 1.0 : 0.0;
    out[1] = c.primalObjective;
    out[2] = c.safeDualBound;
    out[3] = c.certifiedGap;
    out[4] = c.maxPrimalViolation;
    out[5] = out[6] = 0.0;
    out[9] = 0.0;
    for (const CertCheck& k : c.checks) {
      if (k.name == "primal_bound_violation") out[5] = k.value;
      if (k.name == "primal_row_violation") out[6] = k.value;
      if (k.name == "safe_dual_bound_gap" && k.detail.find("constraint-implied") != std::string::npos) out[9] = 1.0;
    }
    out[7] = c.maxDualViolation;
    out[8] = c.costPerturbation;
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

// Simplex from a basis guessed at (x, y) (crossover) when x != NULL, else from
// scratch.  out: status, objective (incl. offset), simplex iterations.
int ref_simplex(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                const double* colLower, const double* colUpper, const double* rowLower, const double* rowUpper,
                double offset, const double* x, const double* y, double* out) {
  try {
    Log::setLevel(LogLevel::Error);
    Model lp = buildModel(m, n, start, index, value, cost, colLower, colUpper, rowLower, rowUpper, offset);
    SimplexOptions so;
    LpResult r = x ? crossover(lp, std::vector<double>(x, x + n), std::vector<double>(y, y + m), so, nullptr)
                   : solveLpSimplex(lp, so, nullptr);
    out[0] = static_cast<double>(r.status);
    out[1] = r.objective;
    out[2] = static_cast<double>(r.stats.iterations);
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

int ref_ruiz_scaling(int m, int n, const int* start, const int* index, const double* value, int iterations,
                     int pockChambolle, double* rowScale, double* colScale) {
  try {
    SparseMatrix A(m, n);
    A.start.assign(start, start + n + 1);
    A.index.assign(index, index + start[n]);
    A.value.assign(value, value + start[n]);
    ScalingResult s = ruizScaling(A, iterations, pockChambolle != 0);
    std::memcpy(rowScale, s.rowScale.data(), sizeof(double) * m);
    std::memcpy(colScale, s.colScale.data(), sizeof(double) * n);
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

// computeFeatures (src/router/router.cpp:64-95): out = m, n, nnz, avg row nnz,
// max row nnz, coefficient range, equality-row fraction, free-column
// fraction, is_mip, is_qp.
int ref_router_features(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                        const double* colLower, const double* colUpper, const double* rowLower,
                        const double* rowUpper, double* out) {
  try {
    Model lp = buildModel(m, n, start, index, value, cost, colLower, colUpper, rowLower, rowUpper, 0.0);
    const RouterFeatures f = computeFeatures(lp);
    const double v[10] = {f.m, f.n, f.nnz, f.avgRowNnz, f.maxRowNnz, f.coeffRange, f.eqFraction, f.freeFraction,
                          f.isMip ? 1.0 : 0.0, f.isQp ? 1.0 : 0.0};
    std::memcpy(out, v, sizeof(v));
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

// Router::decide (src/router/router.cpp:163-207) with the weights of
// `model_path` (Router::load) or, when it is NULL or does not load, the
// built-in priors.  engine = index into dual, ipm, pdhg-cpu, pdhg-gpu;
// pred = the four predicted seconds; loaded = whether the file loaded.
int ref_router_decide(int m, int n, const int* start, const int* index, const double* value, const double* cost,
                      const double* colLower, const double* colUpper, const double* rowLower,
                      const double* rowUpper, const char* model_path, int gpu, double tolerance, int* engine,
                      double* pred, int* loaded) {
  try {
    Log::setLevel(LogLevel::Error);
    Model lp = buildModel(m, n, start, index, value, cost, colLower, colUpper, rowLower, rowUpper, 0.0);
    Router r;
    *loaded = model_path ? (r.load(model_path) ? 1 : 0) : 0;
    const RouterDecision d = r.decide(lp, gpu != 0, tolerance);
    const auto& names = Router::engines();
    *engine = -1;
    for (size_t e = 0; e < names.size(); ++e)
      if (names[e] == d.engine) *engine = static_cast<int>(e);
    pred[0] = d.predictedDual;
    pred[1] = d.predictedIpm;
    pred[2] = d.predictedPdhgCpu;
    pred[3] = d.predictedPdhgGpu;
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

// A timed solve from scratch by the reference's dual simplex (engine 0) or
// interior-point method with crossover (engine 1) under a time limit:
// out = status, objective, seconds, iterations.
int ref_timed_solve(int engine, int m, int n, const int* start, const int* index, const double* value,
                    const double* cost, const double* colLower, const double* colUpper, const double* rowLower,
                    const double* rowUpper, double offset, double time_limit, double* out) {
  try {
    Log::setLevel(LogLevel::Error);
    Model lp = buildModel(m, n, start, index, value, cost, colLower, colUpper, rowLower, rowUpper, offset);
    Deadline dl(time_limit);
    Timer t;
    if (engine == 0) {
      const LpResult r = solveLpSimplex(lp, SimplexOptions{}, time_limit > 0 ? &dl : nullptr);
      out[0] = static_cast<double>(r.status);
      out[1] = r.objective;
      out[3] = static_cast<double>(r.stats.iterations);
    } else {
      const IpmResult r = solveIpm(lp, IpmOptions{}, time_limit > 0 ? &dl : nullptr);
      out[0] = static_cast<double>(r.status);
      out[1] = r.objective;
      out[3] = static_cast<double>(r.stats.iterations);
    }
    out[2] = t.seconds();
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

// The LP that pramana::solve hands to an LP engine for the MPS file at
// `path` (src/api/solver.cpp:251, 302-333): readMps, Model::toMinimization
// and, when `presolve` is set, Presolver::run(minModel, mip) whose reduced
// model is used when the status is Reduced or Empty.  dims = m, n, nnz,
// rows removed, columns removed; the arrays follow from ref_model_arrays.
int ref_load_mps(const char* path, int presolve, int* dims, double* offset) {
  try {
    Log::setLevel(LogLevel::Error);
    const Model input = readMps(path);
    input.validate();
    const Model minModel = input.toMinimization();
    gLoaded = minModel;
    gLoadedMax = input.sense == ObjSense::Maximize;
    dims[3] = dims[4] = 0;
    if (presolve) {
      Presolver pre;
      const PresolveStatus ps = pre.run(minModel, input.isMip());
      if (ps == PresolveStatus::Reduced || ps == PresolveStatus::Empty) {
        gLoaded = pre.reduced();
        dims[3] = pre.stats().rowsRemoved;
        dims[4] = pre.stats().colsRemoved;
      }
    }
    dims[0] = gLoaded.numRows();
    dims[1] = gLoaded.numCols();
    dims[2] = gLoaded.A.nnz();
    *offset = gLoaded.objOffset;
    return 0;
  } catch (std::exception& e) {
    gErr = e.what();
    return 1;
  }
}

// Column of the last loaded model named `name` (-1 if none) and whether the
// file was a maximisation (its costs are negated in the loaded model).
int ref_loaded_column(const char* name, int* was_max) {
  *was_max = gLoadedMax ? 1 : 0;
  for (size_t j = 0; j < gLoaded.colNames.size(); ++j)
    if (gLoaded.colNames[j] == name) return static_cast<int>(j);
  return -1;
}

int ref_model_arrays(int* start, int* index, double* value, double* cost, double* colLower, double* colUpper,
                     double* rowLower, double* rowUpper) {
  const Model& lp = gLoaded;
  std::memcpy(start, lp.A.start.data(), sizeof(int) * lp.A.start.size());
  std::memcpy(index, lp.A.index.data(), sizeof(int) * lp.A.index.size());
  std::memcpy(value, lp.A.value.data(), sizeof(double) * lp.A.value.size());
  std::memcpy(cost, lp.colCost.data(), sizeof(double) * lp.colCost.size());
  std::memcpy(colLower, lp.colLower.data(), sizeof(double) * lp.colLower.size());
  std::memcpy(colUpper, lp.colUpper.data(), sizeof(double) * lp.colUpper.size());
  std::memcpy(rowLower, lp.rowLower.data(), sizeof(double) * lp.rowLower.size());
  std::memcpy(rowUpper, lp.rowUpper.data(), sizeof(double) * lp.rowUpper.size());
  return 0;
}

}  // extern "C"
