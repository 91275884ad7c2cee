// src/pdhg/pdhg_b200.cpp -- PRAMANA's PDHG entry points on the B200 engine.
//
// The file a maintainer adds to the reference: solvePdhg / solvePdhgBatch /
// gpuAvailable / gpuInfoJson (src/pdhg/pdhg.h:73-80) keep their signatures;
// with opts.useGpu and a usable B200 they run on libb2p_pdhg.so through its
// C ABI (include/b2p_pdhg.h), otherwise on the reference's own code.  In the
// reference itself the routing goes at the top of the existing functions in
// src/pdhg/pdhg.cpp; built beside an unmodified tree (tests/dropin/Makefile)
// that file is compiled with its four entry points renamed to
// reference_cpu_*, which the routing below falls back on.
#include <atomic>
#include <chrono>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "b2p_pdhg.h"
#include "pdhg/pdhg.h"
#include "util/common.h"

namespace pramana {

// The reference's own entry points (src/pdhg/pdhg.cpp:712-746), renamed.
PdhgResult reference_cpu_solvePdhg(const Model& lp, const PdhgOptions& opts, const Deadline* deadline);
std::vector<PdhgResult> reference_cpu_solvePdhgBatch(const Model& base, const std::vector<LpCase>& cases,
                                                     const PdhgOptions& opts, const Deadline* deadline,
                                                     PdhgStats* batchStats);

namespace b200 {

inline void check(int rc) {
  if (rc != B2P_OK) throw PramanaError(std::string("B200 PDHG engine: ") + b2p_last_error());
}

inline b2p_lp view(const Model& lp) {  // borrows the model's arrays (CSC A, bounds, costs)
  b2p_lp s{};
  s.num_rows = lp.numRows();
  s.num_cols = lp.numCols();
  s.start = lp.A.start.data();
  s.index = lp.A.index.data();
  s.value = lp.A.value.data();
  s.col_cost = lp.colCost.data();
  s.col_lower = lp.colLower.data();
  s.col_upper = lp.colUpper.data();
  s.row_lower = lp.rowLower.data();
  s.row_upper = lp.rowUpper.data();
  s.obj_offset = lp.objOffset;
  return s;
}

inline b2p_options options(const PdhgOptions& o, const Deadline* dl, const volatile int32_t* cancel) {
  b2p_options b;
  b2p_default_options(&b);
  b.tolerance = o.tolerance;
  b.max_iterations = o.maxIterations;
  b.check_every = o.checkEvery;
  b.ruiz_iterations = o.ruizIterations;
  b.pock_chambolle = o.pockChambolle ? 1 : 0;
  b.rescale_objective_and_bounds = o.rescaleObjectiveAndBounds ? 1 : 0;
  b.reflection = o.reflection;
  b.log_interval = o.logInterval;
  if (dl && dl->limit() > 0) b.time_limit = dl->remaining();
  b.cancel_flag = cancel;
  return b;
}

// Race mode cancels through Deadline::setCancelFlag; the engine polls a plain
// int at every check, so the flag is relayed while a solve runs.
struct CancelRelay {
  volatile int32_t flag = 0;
  std::atomic<bool> done{false};
  std::thread relay;
  explicit CancelRelay(const Deadline* dl) {
    if (dl)
      relay = std::thread([this, dl] {
        while (!done.load()) {
          if (dl->cancelled()) flag = 1;
          std::this_thread::sleep_for(std::chrono::milliseconds(1));
        }
      });
  }
  ~CancelRelay() {
    done = true;
    if (relay.joinable()) relay.join();
  }
};

inline PdhgStats stats(const b2p_stats& s) {
  PdhgStats t;
  t.iterations = s.iterations;
  t.restarts = s.restarts;
  t.primalResidual = s.primal_residual;
  t.dualResidual = s.dual_residual;
  t.gap = s.gap;
  t.primalWeight = s.primal_weight;
  t.setupSeconds = s.setup_seconds;
  t.solveSeconds = s.solve_seconds;
  t.kernelSeconds = s.kernel_seconds;
  t.transferSeconds = s.transfer_seconds;
  t.bytesUploaded = s.bytes_uploaded;
  t.bytesDownloaded = s.bytes_downloaded;
  t.kernelLaunches = s.kernel_launches;
  t.spectralNorm = s.spectral_norm;
  t.backend = "gpu";
  t.device = "B200 (sm_100a)";
  return t;
}

// One solve (cases == nullptr) or a batch over a shared A; external linkage,
// so that the routing may sit in src/pdhg/pdhg.cpp.
std::vector<PdhgResult> solve(const Model& lp, const std::vector<LpCase>* cases, const PdhgOptions& o,
                              const Deadline* dl, PdhgStats* batchStats) {
  const int n = lp.numCols(), m = lp.numRows();
  const int k = cases ? static_cast<int>(cases->size()) : 1;
  CancelRelay cancel(dl);
  const b2p_lp a = view(lp);
  const b2p_options bo = options(o, dl, &cancel.flag);
  std::vector<double> x(static_cast<size_t>(k) * n), y(static_cast<size_t>(k) * m);
  std::vector<b2p_result> r(k);
  b2p_stats st{};
  if (cases) {
    std::vector<b2p_case> cs(k);
    for (int b = 0; b < k; ++b) {
      const LpCase& c = (*cases)[b];
      cs[b].cost = c.cost.empty() ? nullptr : c.cost.data();
      cs[b].col_lower = c.colLower.empty() ? nullptr : c.colLower.data();
      cs[b].col_upper = c.colUpper.empty() ? nullptr : c.colUpper.data();
      cs[b].row_lower = c.rowLower.empty() ? nullptr : c.rowLower.data();
      cs[b].row_upper = c.rowUpper.empty() ? nullptr : c.rowUpper.data();
    }
    check(b2p_solve_pdhg_batch(&a, cs.data(), k, &bo, x.data(), y.data(), r.data(), &st));
  } else {
    check(b2p_solve_pdhg(&a, &bo, x.data(), y.data(), r.data(), &st));
  }
  std::vector<PdhgResult> out(k);
  for (int b = 0; b < k; ++b) {
    out[b].status = static_cast<Status>(r[b].status);  // same numbering as pramana::Status
    out[b].objective = r[b].objective;
    out[b].dualObjective = r[b].dual_objective;
    out[b].iterations = r[b].iterations;
    out[b].relativeKkt = r[b].relative_kkt;
    out[b].x.assign(x.begin() + static_cast<size_t>(b) * n, x.begin() + static_cast<size_t>(b + 1) * n);
    out[b].rowDual.assign(y.begin() + static_cast<size_t>(b) * m, y.begin() + static_cast<size_t>(b + 1) * m);
    out[b].stats = stats(st);
  }
  if (batchStats) *batchStats = stats(st);
  return out;
}

}  // namespace b200

PdhgResult solvePdhg(const Model& lp, const PdhgOptions& opts, const Deadline* deadline) {
  if (opts.useGpu && b2p_gpu_available()) return b200::solve(lp, nullptr, opts, deadline, nullptr)[0];
  return reference_cpu_solvePdhg(lp, opts, deadline);
}

std::vector<PdhgResult> solvePdhgBatch(const Model& base, const std::vector<LpCase>& cases, const PdhgOptions& opts,
                                       const Deadline* deadline, PdhgStats* batchStats) {
  if (cases.empty()) return {};
  if (opts.useGpu && b2p_gpu_available()) return b200::solve(base, &cases, opts, deadline, batchStats);
  return reference_cpu_solvePdhgBatch(base, cases, opts, deadline, batchStats);
}

bool gpuAvailable() { return b2p_gpu_available() != 0; }

Json gpuInfoJson() {  // the engine's keys; "nvrtc" no longer applies
  std::string s(static_cast<size_t>(b2p_gpu_info_json(nullptr, 0)) + 1, '\0');
  b2p_gpu_info_json(s.data(), s.size());
  return Json::parse(s.c_str());
}

}  // namespace pramana
