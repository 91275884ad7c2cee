"""The engine on the reference's published PDHG runs: its refinery planning
models (data/gen/plan_*.mps) presolved as solve() hands them to solvePdhg,
with the telemetry it published for `--algo pdhg-cpu|pdhg-gpu --pdhg-tol
1e-4|1e-6` (results/gpu/plan_*.json; fixtures by
tests/golden/make_plan_golden.py).  The reference's CPU and GPU runs agree on
every iteration and restart count; so must this engine, in the plain FP64
form, alone and batched."""
import numpy as np
import pytest

import lp_cases
from pramana_b200 import _lib, pdhg
from test_gpu_parity import _host_kkt, opts

pytestmark = pytest.mark.gpu

RUNS = ("pdhg-cpu_raw1e-4", "pdhg-gpu_raw1e-6")


@pytest.mark.parametrize("run", RUNS)
@pytest.mark.parametrize("plan", lp_cases.PLANS)
def test_engine_reproduces_published_plan_runs(plan, run):
    """Iterations, restarts and the spectral-norm estimate exactly as
    published; relative KKT within 1e-6 and objective within 1e-9 relative
    (the engine's row sums are split across lanes for long rows, so its
    rounding differs from both published runs in the last bits)."""
    lp, pub = lp_cases.load_plan(plan)
    p = pub[run]
    r = pdhg.solvePdhg(lp, opts(tolerance=p["tolerance"]))
    st = r.stats
    assert r.status == "Optimal"
    assert (st.iterations, st.restarts) == (p["iterations"], p["restarts"])
    assert st.spectralNorm == p["spectral_norm_estimate"]
    assert abs(r.relativeKkt - p["relative_kkt"]) <= 1e-6 * p["relative_kkt"]
    assert abs(r.objective - p["objective"]) <= 1e-9 * abs(p["objective"])


@pytest.mark.parametrize("tol,run", [(1e-4, "pdhg-cpu_raw1e-4"), (1e-6, "pdhg-gpu_raw1e-6")])
def test_multi_engine_reproduces_published_plan_runs(tol, run):
    """All six plans in one batched solve: each LP terminates at its
    published iteration (the result counts the check iteration, the
    published telemetry one more, src/pdhg/pdhg.cpp:583, 665)."""
    plans = [lp_cases.load_plan(p) for p in lp_cases.PLANS]
    rs = pdhg.solvePdhgMulti([lp for lp, _ in plans], opts(tolerance=tol))
    for (lp, pub), r in zip(plans, rs):
        p = pub[run]
        assert r.status == "Optimal"
        assert r.iterations + 1 == p["iterations"], lp.name
        assert abs(r.objective - p["objective"]) <= 1e-9 * abs(p["objective"])


@pytest.mark.parametrize("plan", lp_cases.PLANS)
def test_mixed_form_on_published_plans(plan):
    """The mixed-precision form meets 1e-6 in FP64 terms on every plan and
    lands within 1e-5 relative of the published 1e-6 objective."""
    lp, pub = lp_cases.load_plan(plan)
    p = pub["pdhg-gpu_raw1e-6"]
    r = pdhg.solvePdhg(lp, opts(tolerance=1e-6, precision=_lib.PRECISION_MIXED))
    assert r.status == "Optimal" and r.relativeKkt <= 1e-6
    assert abs(r.objective - p["objective"]) <= 1e-5 * abs(p["objective"])
    assert max(_host_kkt(lp, r.x, r.rowDual)) <= 1.5e-6
    assert np.all(r.x >= lp.col_lower - 1e-9) and np.all(r.x <= lp.col_upper + 1e-9)
