"""b2p_safe_dual_bound against the reference's own safeDualBound
(src/cert/certifier.cpp:58-118, built into oracle/_ref): every field must be
bit-identical, for solved duals, for duals whose wrong-signed reduced costs
on infinite bounds are clipped (finite bound, cost perturbation recorded) or
make the bound -inf, and for batches of cases.  b2p_certify_lp against the
reference's certify(): the same verdicts, primal figures equal to rounding,
and valid bounds over the implied column bounds."""
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


def assert_agrees_with_reference_certificate(got: dict, want: dict, lp, exact_opt=None):
    """The verdict is the reference's; the primal figures agree to rounding
    (compensated sums in a different order); the bound over the given column
    bounds is bit-identical, and one over implied bounds is valid (at most the
    exact optimum) and no weaker than the reference's beyond its relaxation."""
    assert got["accepted"] == want["accepted"]
    assert got["used_implied_bounds"] == want["used_implied_bounds"]
    po, pw = got["primal_objective"], want["primal_objective"]
    assert abs(po - pw) <= 1e-13 * (1 + abs(pw)), (po, pw)
    # the row activities: compensated dot products here (product errors kept),
    # Kahan-Babuska sums of rounded products in the reference
    for f in ("max_primal_violation", "max_col_violation", "max_row_violation"):
        g, w = got[f], want[f]
        assert g == w or abs(g - w) <= 1e-9 * (1 + abs(w)), (f, g, w)
    if "worst_row" in want and want["max_row_violation"] > 1e-9:
        assert got["worst_row"] == want["worst_row"]
    if not got["used_implied_bounds"]:
        for f in ("safe_dual_bound", "max_dual_violation", "cost_perturbation"):
            assert got[f] == want[f] or (np.isnan(got[f]) and np.isnan(want[f])), (f, got[f], want[f])
        g, w = got["certified_gap"], want["certified_gap"]
        assert g == w or abs(g - w) <= 1e-13, (g, w)
    else:
        lb, lw = got["safe_dual_bound"], want["safe_dual_bound"]
        assert np.isfinite(lb) == np.isfinite(lw)
        if np.isfinite(lw):
            assert lb >= lw - 1e-6 * (1 + abs(pw)), (lb, lw)
        if exact_opt is not None and np.isfinite(lb):
            assert lb <= exact_opt + 1e-12 * (1 + abs(exact_opt)), (lb, exact_opt)


def _refinery():
    from pramana_b200 import warmstart as W
    return W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)


@pytest.mark.parametrize("which", ["c1", "edge", "refinery", "refinery_perturbed", "random_dual"])
def test_certify_agrees_with_reference(oracle_mod, which):
    """b2p_certify_lp against the reference's certify() on OPTIMAL claims:
    accepted claims, a bound that needs the implied-bounds retry, a perturbed
    (rejected) point, and a random dual (no rigorous bound)."""
    exact = None
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
        exact = oracle_mod.simplex(lp)["objective"]
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
    assert_agrees_with_reference_certificate(got, want, lp, exact)
    if which == "c1":
        assert got["accepted"] == 1
    if which == "refinery_perturbed":
        assert got["accepted"] == 0
    if which == "refinery":
        assert got["used_implied_bounds"] == 1 and np.isfinite(got["safe_dual_bound"])


def test_certify_family_batch_agrees_with_reference(oracle_mod):
    fam = _refinery()
    params = fam.sample(6, 9)
    cases = [fam.case(p) for p in params]
    rs = pdhg.solvePdhgBatch(fam.base, cases, pdhg.PdhgOptions(tolerance=1e-6, maxIterations=200000))
    X = np.concatenate([r.x for r in rs])
    Y = np.concatenate([r.rowDual for r in rs])
    got = pdhg.certifyLp(fam.base, X, Y, cases)
    for b, p in enumerate(params):
        inst = fam.instance(p)
        assert_agrees_with_reference_certificate(got[b], oracle_mod.certify(inst, rs[b].x, rs[b].rowDual), inst,
                                                 oracle_mod.simplex(inst)["objective"])
