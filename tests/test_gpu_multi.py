"""Independent LPs of different sizes solved together (b2p_solve_pdhg_multi):
every instance must follow the reference algorithm as if solved alone --
checked against the oracle at fixed iteration counts and to convergence."""
import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200 import pdhg
from pramana_b200.model import Model
from test_gpu_parity import _host_kkt, assert_close, opts

pytestmark = pytest.mark.gpu


def family():
    lps = [G.random_lp(m, 2 * m, 4.0, int(0.6 * m), 100 + i) for i, m in enumerate([50, 300, 120, 1000, 10])]
    lps.append(G.random_lp(2000, 4000, 6.4, 1200, 7, heavy_row_frac=0.01, heavy_nnz_frac=0.1))
    lps.append(lp_cases.edge_lp(5))
    n = 5
    lps.append(Model(num_rows=0, num_cols=n, start=np.zeros(n + 1), index=[], value=[], col_cost=[1, -1, 2, 0, 3],
                     col_lower=np.zeros(n), col_upper=np.full(n, 4.0), row_lower=[], row_upper=[]))
    return lps


@pytest.mark.parametrize("iters", [1, 64, 1000])
def test_multi_fixed_iterations_vs_oracle(oracle_mod, iters):
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=iters))
    for lp, r in zip(lps, rs):
        assert_close(r, oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters))


def test_multi_converged_vs_oracle(oracle_mod):
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, maxIterations=200000))
    for lp, r in zip(lps, rs):
        o = oracle_mod.solve(lp, "oracle", tolerance=1e-6, max_iterations=200000)
        assert r.status == "Optimal" and o.status == 1
        assert abs(r.iterations - o.iterations) <= 4 * 64
        assert abs(r.objective - o.objective) <= 1e-5 * (1 + abs(o.objective))
        if lp.num_rows:
            assert max(_host_kkt(lp, r.x, r.rowDual)) <= 1e-6 * (1 + 1e-6)


def test_multi_iteration_limit_reports_every_instance(oracle_mod):
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=100))
    for lp, r in zip(lps, rs):
        o = oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=100)
        assert r.status == {1: "Optimal", 6: "IterationLimit"}[o.status] and r.iterations == o.iterations


def test_multi_warm_start():
    lps = family()[:6]
    cold = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6))
    starts = [(r.x, r.rowDual) if b % 2 == 0 else None for b, r in enumerate(cold)]
    warm = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6), starts=starts)
    for b, (c, w) in enumerate(zip(cold, warm)):
        assert w.status == "Optimal"
        if b % 2 == 0:
            assert w.iterations <= 64
        else:
            assert w.iterations == c.iterations


# ---- SpMV schedules of the multi-LP engine: warp tiles and the autotuner ----

from pramana_b200 import _lib  # noqa: E402


@pytest.mark.parametrize("sched", [_lib.SCHEDULE_TILED, _lib.SCHEDULE_TUNED])
@pytest.mark.parametrize("iters", [1, 64, 1000])
def test_multi_schedules_fixed_iterations_vs_oracle(oracle_mod, sched, iters):
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=iters, spmvSchedule=sched))
    st = pdhg.solvePdhgMulti.last_stats
    if sched == _lib.SCHEDULE_TILED:
        assert st.schedule_a == _lib.SCHEDULE_TILED and st.schedule_at == _lib.SCHEDULE_TILED
    else:
        assert st.autotune_seconds > 0
    for lp, r in zip(lps, rs):
        assert_close(r, oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters))


@pytest.mark.parametrize("iters", [1, 2, 63])
def test_tiled_rows_sum_in_reference_order(oracle_mod, iters):
    """Every row and column of config-1 has at most 32 entries, so the tiled
    kernels sum every row left to right exactly as the reference does: before
    the first check the iterates are bit-identical to the oracle's."""
    lp = G.config1(1)
    assert np.diff(lp.start).max() <= 32 and np.bincount(lp.index).max() <= 32
    r = pdhg.solvePdhgMulti([lp], opts(tolerance=1e-30, maxIterations=iters,
                                       spmvSchedule=_lib.SCHEDULE_TILED))[0]
    o = oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters)
    assert np.array_equal(r.x, o.x) and np.array_equal(r.rowDual, o.y)


def test_tiled_many_tiles_per_cta_matches_binned():
    """~3M nonzeros: many warp tiles per launch, long rows on the binned
    path as leading blocks of the same launch."""
    lps = G.uneven_family(8, 2e5, 6e5, seed=11)
    kw = dict(tolerance=1e-30, maxIterations=200)
    rb = pdhg.solvePdhgMulti(lps, opts(spmvSchedule=_lib.SCHEDULE_BINNED, **kw))
    rt = pdhg.solvePdhgMulti(lps, opts(spmvSchedule=_lib.SCHEDULE_TILED, **kw))
    for a, b in zip(rb, rt):
        assert np.linalg.norm(a.x - b.x) <= 1e-9 * np.linalg.norm(a.x)
        assert np.linalg.norm(a.rowDual - b.rowDual) <= 1e-9 * np.linalg.norm(a.rowDual)


def test_tiled_converged_and_compacted(oracle_mod):
    lps = family() + [G.random_lp(3000, 6000, 6.4, 1800, 21, heavy_row_frac=0.01, heavy_nnz_frac=0.1)]
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, maxIterations=200000, spmvSchedule=_lib.SCHEDULE_TILED))
    for lp, r in zip(lps, rs):
        o = oracle_mod.solve(lp, "oracle", tolerance=1e-6, max_iterations=200000)
        assert r.status == "Optimal" and o.status == 1
        assert abs(r.iterations - o.iterations) <= 4 * 64
        assert max(_host_kkt(lp, r.x, r.rowDual)) <= 1.5e-6
