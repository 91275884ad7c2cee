// Checks that the host preparation's parallel passes (OpenMP) give exactly
// the sequential result: scaled operators, factors and rescaling constants.
// Built and run by tests/test_prepare_parallel.py.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "pdhg_prepare.h"

using namespace b2p;

template <class T>
static bool same(const std::vector<T>& a, const std::vector<T>& b) {
  return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(T)) == 0);
}

int main() {
  int failures = 0;
  for (int seed = 0; seed < 6; ++seed) {
    std::mt19937 rng(seed);
    const int m = 2000 + 7919 * seed, n = 2 * m + 13;
    std::vector<int32_t> start(n + 1, 0), index;
    std::vector<double> value;
    std::normal_distribution<double> nd;
    for (int j = 0; j < n; ++j) {
      const int len = (seed % 3 == 0 && j % 97 == 0) ? 0 : 1 + static_cast<int>(rng() % 12);
      std::vector<int> rows;
      for (int q = 0; q < len; ++q) rows.push_back(static_cast<int>(rng() % (seed == 5 ? 7 : m)));
      std::sort(rows.begin(), rows.end());
      rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
      for (int r : rows) {
        index.push_back(r);
        value.push_back(nd(rng) * std::pow(10.0, static_cast<int>(rng() % 7) - 3));
      }
      start[j + 1] = static_cast<int32_t>(index.size());
    }
    std::vector<double> cost(n), rl(m), ru(m);
    for (auto& c : cost) c = nd(rng);
    for (int i = 0; i < m; ++i) {
      rl[i] = (i % 3 == 0) ? -1e30 : nd(rng);
      ru[i] = (i % 5 == 0) ? 1e30 : rl[i] + 1.0;
    }
    PrepareOptions seq, par;
    seq.parallel = false;
    par.parallel = true;
    const Prepared a = prepare(m, n, start.data(), index.data(), value.data(), cost.data(), rl.data(), ru.data(), 0.5,
                               seq);
    const Prepared b = prepare(m, n, start.data(), index.data(), value.data(), cost.data(), rl.data(), ru.data(), 0.5,
                               par);
    const bool ok = same(a.A.ptr, b.A.ptr) && same(a.A.idx, b.A.idx) && same(a.A.val, b.A.val) &&
                    same(a.AT.ptr, b.AT.ptr) && same(a.AT.idx, b.AT.idx) && same(a.AT.val, b.AT.val) &&
                    same(a.R, b.R) && same(a.Cs, b.Cs) && same(a.rfac, b.rfac) && same(a.cfac, b.cfac) &&
                    a.beta == b.beta && a.gamma == b.gamma && a.normA == b.normA;
    std::printf("seed %d m %d n %d nnz %d: %s\n", seed, m, n, start[n], ok ? "identical" : "DIFFERENT");
    failures += !ok;
  }
  return failures;
}
