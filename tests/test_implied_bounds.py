"""b2p_implied_bounds: constraint-implied column bounds on the GPU (Jacobi
rounds of activity-based tightening, rounded outward).

The bounds are judged by what a certificate needs from them:
  * validity -- they contain the LP's feasible points: a point solved to rel
    KKT 1e-10 lies inside them (to its own residual), and the outward-rounded
    dual bound over them stays at or below the exact optimum of the
    reference's simplex;
  * tightness -- every column the reference's own propagation bounds
    (oracle/_ref, Propagator::propagate through the certifier's relaxation)
    is bounded here too, at least as tightly up to that relaxation, and the
    dual bound over them is finite wherever the reference's is.
Cases of a family with overridden bounds, and empty boxes, are covered."""
import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200 import pdhg, warmstart as W
from pramana_b200.model import LpCase, Model

pytestmark = pytest.mark.gpu


def _with_bounds(lp, lo, up):
    return Model(**{**lp.__dict__, "col_lower": lo, "col_upper": up})


def _lp(which):
    if which == "refinery":
        return G.refinery_lp(periods=2, regions=1, units=4, pools=10, streams=4, properties=2, seed=5,
                             scale_exponent=0.0)
    if which == "refinery_scaled":
        return G.refinery_lp(periods=3, regions=2, units=5, pools=10, streams=6, properties=3, seed=7)
    if which == "edge":
        return lp_cases.edge_lp(5)
    if which == "c1":
        return G.config1(1)
    if which == "plan_10x12":
        return lp_cases.load_plan("plan_10x12")[0]
    lp = G.random_lp(200, 400, 3.0, 120, 21)
    rng = np.random.default_rng(2)
    lo, up = lp.col_lower.copy(), lp.col_upper.copy()
    free = rng.random(lp.num_cols) < 0.3
    lo[free], up[free] = -np.inf, np.inf
    return _with_bounds(lp, lo, up)


def _finite(v):
    return np.abs(v) < 1e20


def assert_as_tight_as_reference(lo, up, ref_lo, ref_up):
    """Every bound the reference tightened is here too, no looser than the
    reference's (whose tightened bounds carry a 1e-6 (1 + |b|) relaxation)."""
    for mine, ref, sign in ((lo, ref_lo, 1.0), (up, ref_up, -1.0)):
        fr = _finite(ref)
        assert np.all(_finite(mine[fr])), "a bound the reference finds is missing"
        slack = 2e-6 * (1.0 + np.abs(ref[fr]))
        assert np.all(sign * (mine[fr] - ref[fr]) >= -slack), np.max(sign * (ref[fr] - mine[fr]) / slack)


@pytest.mark.parametrize("which", ["refinery", "refinery_scaled", "edge", "c1", "random_free", "plan_10x12"])
def test_implied_bounds_valid_and_as_tight_as_reference(oracle_mod, which):
    lp = _lp(which)
    lo, up = pdhg.impliedBounds(lp)
    lo, up = lo[0], up[0]
    # never looser than the model's own bounds
    assert np.all(lo >= np.where(_finite(lp.col_lower), lp.col_lower, -np.inf))
    assert np.all(up <= np.where(_finite(lp.col_upper), lp.col_upper, np.inf))
    want_lo, want_up = oracle_mod.implied_bounds(lp)
    assert_as_tight_as_reference(lo, up, want_lo, want_up)
    # a tightly solved point lies inside them, to its own residual
    r = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-10, maxIterations=400000))
    if r.status == "Optimal":
        scale = 1e-6 * (1.0 + np.abs(r.x))
        assert np.all(r.x >= lo - scale) and np.all(r.x <= up + scale)
    if which.startswith("refinery") or which == "plan_10x12":
        # the balances bound the otherwise unbounded flows
        assert _finite(up).sum() > _finite(lp.col_upper).sum()


@pytest.mark.parametrize("which", ["refinery", "plan_10x12"])
def test_dual_bound_over_implied_bounds_is_below_the_exact_optimum(oracle_mod, which):
    """The reason the bounds exist: PDHG's duals leave wrong-signed reduced
    costs on free columns, which make the plain bound -inf; over the implied
    bounds it is finite, at most the exact optimum, and within the
    reference's family rule 1e-4 (1 + |obj|) of it."""
    lp = _lp(which)
    exact = oracle_mod.simplex(lp)
    assert exact["status"] == "Optimal"
    opt = exact["objective"]
    r = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-6, maxIterations=400000))
    lo, up = pdhg.impliedBounds(lp)
    sb = pdhg.safeDualBound(lp, r.rowDual, [LpCase(col_lower=lo[0], col_upper=up[0])])[0]
    lb = sb["bound"] + lp.obj_offset
    assert np.isfinite(lb)
    assert lb <= opt + 1e-12 * (1 + abs(opt))
    assert opt - lb <= 1e-4 * (1 + abs(opt))
    ref_lo, ref_up = oracle_mod.implied_bounds(lp)
    ref = oracle_mod.safe_dual_bound(lp, r.rowDual, ref_lo, ref_up, full=True)
    assert lb >= ref["bound"] + lp.obj_offset - 1e-6 * (1 + abs(opt))


def test_implied_bounds_per_case(oracle_mod):
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    params = fam.sample(5, 3)
    cases = [fam.case(p) for p in params]
    lo, up = pdhg.impliedBounds(fam.base, cases)
    for b, p in enumerate(params):
        one_lo, one_up = pdhg.impliedBounds(fam.instance(p))
        # a case of the batch gets exactly what it gets alone
        assert np.array_equal(lo[b], one_lo[0]) and np.array_equal(up[b], one_up[0])
        want_lo, want_up = oracle_mod.implied_bounds(fam.instance(p))
        assert_as_tight_as_reference(lo[b], up[b], want_lo, want_up)


def test_empty_boxes_are_returned_valid(oracle_mod):
    """Columns whose upper bound lies below the lower one: the case is
    infeasible, and whatever comes back is no looser than the given bounds."""
    lp = lp_cases.edge_lp(6)
    up = lp.col_upper.copy()
    fin = np.isfinite(up)
    up[fin] = lp.col_lower[fin] - 1.0 * (lp.col_lower[fin] > -np.inf)  # empty boxes
    up[~np.isfinite(lp.col_lower)] = lp.col_upper[~np.isfinite(lp.col_lower)]
    lo_g, up_g = pdhg.impliedBounds(lp, [LpCase(col_upper=up)])
    assert np.all(lo_g[0] >= np.where(_finite(lp.col_lower), lp.col_lower, -np.inf))
    assert np.all(up_g[0] <= np.where(_finite(up), up, np.inf))
