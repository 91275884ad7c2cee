// Restart bookkeeping of one PDHG case between checks, on the host.
//
// Restarted Halpern PDHG restarts a case from its current point when a
// merit -- the weighted fixed-point residual sqrt(w |x - x+|^2 + |y - y+|^2 / w)
// measured at the check -- has decayed enough since the last restart: by a
// factor 0.2 (sufficient decay), or by 0.8 while it grew since the previous
// check (necessary decay without progress), or when 36% of all iterations so
// far have passed since the last restart (the artificial restart).  At a
// restart the primal weight w moves to the geometric mean of itself and the
// ratio |dy| / |dx| of the movement since the last restart, when both
// movements are measurable (> 1e-10).  These rules and constants are the
// method's (src/pdhg/pdhg.cpp:631-656) and are kept for iterate parity.
#pragma once

#include <cmath>
#include <cstdint>

#include "pdhg_kernels.cuh"

namespace b2p {

class RestartTracker {
 public:
  // The merit of a check's sums under primal weight w.
  static double merit(double w, const double* sums) { return std::sqrt(w * sums[CS_DX2] + sums[CS_DY2] / w); }

  // At a check of iteration `iter` that did not terminate, `interval`
  // iterations after the previous one: whether the case restarts now.
  bool due(double w, const double* sums, int64_t iter, int interval) {
    elapsed_ += interval;
    const double now = merit(w, sums);
    if (std::isinf(reference_)) reference_ = now;
    const bool decayed = now <= 0.2 * reference_;
    const bool stalled = now <= 0.8 * reference_ && now > previous_;
    const bool overdue = elapsed_ >= static_cast<int64_t>(0.36 * static_cast<double>(iter + 1));
    previous_ = now;
    return decayed || stalled || overdue;
  }

  // The restart itself: the new primal weight (updated in place) from the
  // movement since the last restart, and the merit the next test compares with.
  void restart(double& w, const double* sums) {
    const double moved_x = std::sqrt(sums[CS_AX2]), moved_y = std::sqrt(sums[CS_AY2]);
    if (moved_x > 1e-10 && moved_y > 1e-10) w = std::exp(0.5 * std::log(moved_y / moved_x) + 0.5 * std::log(w));
    reference_ = merit(w, sums);
    previous_ = INFINITY;
    elapsed_ = 0;
  }

  // Forget the history (a new phase starts from the current point).
  void reset() {
    reference_ = previous_ = INFINITY;
    elapsed_ = 0;
  }

 private:
  double reference_ = INFINITY;  // merit right after the last restart (or at the first check)
  double previous_ = INFINITY;   // merit at the previous check
  int64_t elapsed_ = 0;          // iterations since the last restart
};

}  // namespace b2p
