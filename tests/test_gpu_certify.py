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


CERT_FIELDS = ("accepted", "primal_objective", "safe_dual_bound", "certified_gap", "max_primal_violation",
               "max_col_violation", "max_row_violation", "max_dual_violation", "cost_perturbation",
               "used_implied_bounds")


def assert_same_cert(got: dict, want: dict):
    for f in CERT_FIELDS:
        g, w = got[f], want[f]
        assert g == w or (np.isnan(g) and np.isnan(w)), (f, g, w)


def _refinery():
    from pramana_b200 import warmstart as W
    return W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)


@pytest.mark.parametrize("which", ["c1", "edge", "refinery", "refinery_perturbed", "random_dual"])
def test_certify_bitexact_vs_reference(oracle_mod, which):
    """b2p_certify_lp against the reference's certify() on OPTIMAL claims:
    accepted claims, a bound that needs the implied-bounds retry, a perturbed
    (rejected) point, and a random dual (no rigorous bound)."""
    if which == "c1":
        lp = G.config1(1)
        r = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-8))
        x, y = r.x, r.rowDual
    elif which == "edge":
        lp = lp_cases.edge_lp(5)
        r = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-8, maxIterations=200000))
        x, y = r.x, r.rowDual
    elif which.startswith("refinery"):
        fam = _refinery()
        lp = fam.instance(fam.sample(1, 8)[0])
        r = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-6, maxIterations=200000))
        x, y = r.x.copy(), r.rowDual
        if which == "refinery_perturbed":
            x *= 1.01
    else:
        lp = G.config1(2)
        x = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-4)).x
        y = np.random.default_rng(5).normal(size=lp.num_rows)
    got = pdhg.certifyLp(lp, x, y)[0]
    want = oracle_mod.certify(lp, x, y)
    assert_same_cert(got, want)
    if which == "c1":
        assert got["accepted"] == 1
    if which == "refinery_perturbed":
        assert got["accepted"] == 0
    if which == "refinery":
        assert got["used_implied_bounds"] == 1 and np.isfinite(got["safe_dual_bound"])


def test_certify_family_batch_bitexact(oracle_mod):
    fam = _refinery()
    params = fam.sample(6, 9)
    cases = [fam.case(p) for p in params]
    rs = pdhg.solvePdhgBatch(fam.base, cases, pdhg.PdhgOptions(tolerance=1e-6, maxIterations=200000))
    X = np.concatenate([r.x for r in rs])
    Y = np.concatenate([r.rowDual for r in rs])
    got = pdhg.certifyLp(fam.base, X, Y, cases)
    for b, p in enumerate(params):
        assert_same_cert(got[b], oracle_mod.certify(fam.instance(p), rs[b].x, rs[b].rowDual))
