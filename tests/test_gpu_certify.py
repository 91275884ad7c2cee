"""b2p_safe_dual_bound against the reference's own safeDualBound
(src/cert/certifier.cpp:58-118, built into oracle/_ref): every field must be
bit-identical, for solved duals, for duals whose wrong-signed reduced costs
on infinite bounds are clipped (finite bound, cost perturbation recorded) or
make the bound -inf, and for batches of cases."""
import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200 import pdhg
from pramana_b200.model import Model

pytestmark = pytest.mark.gpu

FIELDS = ("bound", "infinite_terms", "max_dual_infeasibility", "row_projection", "cost_perturbation")


def assert_same(got: dict, want: dict):
    for f in FIELDS:
        g, w = got[f], want[f]
        assert g == w or (np.isnan(g) and np.isnan(w)), (f, g, w)


@pytest.mark.parametrize("which", ["c1", "c2", "edge_solved", "edge_tight", "edge_random"])
def test_safe_bound_bitexact_vs_reference(oracle_mod, which):
    if which == "c1":
        lp = G.config1(1)
        y = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-4)).rowDual
    elif which == "c2":
        lp = G.config2(2)
        y = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-6)).rowDual
    elif which == "edge_solved":
        lp = lp_cases.edge_lp(5)
        y = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-6)).rowDual
    elif which == "edge_tight":
        lp = lp_cases.edge_lp(5)
        y = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-12, maxIterations=200000)).rowDual
    else:
        lp = lp_cases.edge_lp(6)
        y = np.random.default_rng(4).normal(size=lp.num_rows)
    got = pdhg.safeDualBound(lp, y)[0]
    want = oracle_mod.safe_dual_bound(lp, y, full=True)
    assert_same(got, want)
    if which in ("c1", "c2"):
        assert np.isfinite(got["bound"])
    if which == "edge_random":
        assert got["bound"] == -np.inf and got["infinite_terms"] > 0


def test_safe_bound_clipping_path_is_exercised(oracle_mod):
    """A dual accurate to ~1e-12 leaves tiny wrong-signed reduced costs on
    free columns: they are clipped and the bound stays finite."""
    lp = lp_cases.edge_lp(5)
    y = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-12, maxIterations=200000)).rowDual
    got = pdhg.safeDualBound(lp, y)[0]
    if got["cost_perturbation"] > 0:
        assert np.isfinite(got["bound"]) or got["cost_perturbation"] > 1e-9
    assert_same(got, oracle_mod.safe_dual_bound(lp, y, full=True))


def test_safe_bound_batch_bitexact(oracle_mod):
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    cases = lp_cases.mixed_cases(lp, 6)
    rs = pdhg.solvePdhgBatch(lp, cases, pdhg.PdhgOptions(tolerance=1e-6))
    y = np.concatenate([r.rowDual for r in rs])
    got = pdhg.safeDualBound(lp, y, cases)
    for b, cs in enumerate(cases):
        one = Model(**{**lp.__dict__, **{f: getattr(cs, f) for f in ("row_lower", "row_upper", "col_lower",
                                                                      "col_upper") if getattr(cs, f) is not None},
                       "col_cost": cs.cost if cs.cost is not None else lp.col_cost})
        assert_same(got[b], oracle_mod.safe_dual_bound(one, rs[b].rowDual, full=True))
        # certified in the family sense: a finite safe bound within 1e-4 of the objective
        assert abs(rs[b].objective - (got[b]["bound"] + lp.obj_offset)) <= 1e-4 * (1 + abs(rs[b].objective))
