"""The shared-A batch engine on the reference's published repeated-solve
experiment (results/family/*.json): K crude-price or crude-availability cases
of a refinery plan in one solvePdhgBatch call at 1e-6 with at most 200,000
iterations, certified by the outward-rounded dual bound over
constraint-implied column bounds (src/parametric/parametric.cpp:483-527).
The batch must end at the published iteration, solve and certify the
published number of cases, and land on the published objective error against
the exact optima (the reference's dual simplex)."""
import numpy as np
import pytest

import lp_cases
from pramana_b200 import pdhg
from test_gpu_parity import opts

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fam", lp_cases.FAMILIES)
def test_batch_reproduces_published_family(fam):
    lp, cases, exact, pub = lp_cases.load_family(fam)
    p = pub["gpu"]
    st = pdhg.PdhgStats()
    rs = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-6, maxIterations=200000), batchStats=st)
    assert st.iterations == p["iterations"]
    solved = [b for b, r in enumerate(rs) if r.status == "Optimal"]
    assert len(solved) == p["solved"]
    assert lp_cases.family_certified(lp, cases, rs, pdhg.safeDualBound, pdhg.impliedBounds) == p["certified"]
    if solved:
        err = max(abs(rs[b].objective - exact[b]) / max(1.0, abs(exact[b])) for b in solved)
        assert abs(err - p["max_relative_error"]) <= 1e-3 * p["max_relative_error"]
    else:
        assert all(r.status == "IterationLimit" for r in rs)
