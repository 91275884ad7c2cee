"""b2p_implied_bounds (host restatement of the certifier's bound propagation)
against the reference's own Propagator (oracle/_ref): bit-identical bounds
on refinery-planning LPs, random LPs with boxed / one-sided / free columns,
family cases with overridden bounds, and empty column boxes.  Host computation: no GPU."""
import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200 import pdhg, warmstart as W
from pramana_b200.model import LpCase, Model


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


def _with_bounds(lp, lo, up):
    return Model(**{**lp.__dict__, "col_lower": lo, "col_upper": up})


@pytest.mark.parametrize("which", ["refinery", "refinery_scaled", "edge", "c1", "random_free"])
def test_implied_bounds_bitexact(oracle_mod, which):
    if which == "refinery":
        lp = G.refinery_lp(periods=2, regions=1, units=4, pools=10, streams=4, properties=2, seed=5,
                           scale_exponent=0.0)
    elif which == "refinery_scaled":
        lp = G.refinery_lp(periods=3, regions=2, units=5, pools=10, streams=6, properties=3, seed=7)
    elif which == "edge":
        lp = lp_cases.edge_lp(5)
    elif which == "c1":
        lp = G.config1(1)
    else:
        lp = G.random_lp(200, 400, 3.0, 120, 21)
        rng = np.random.default_rng(2)
        lo, up = lp.col_lower.copy(), lp.col_upper.copy()
        free = rng.random(lp.num_cols) < 0.3
        lo[free], up[free] = -np.inf, np.inf
        lp = _with_bounds(lp, lo, up)
    lo, up = pdhg.impliedBounds(lp)
    want_lo, want_up = oracle_mod.implied_bounds(lp)
    assert _same(lo[0], want_lo) and _same(up[0], want_up)
    if which.startswith("refinery"):
        # the balances bound the otherwise unbounded flows
        assert np.isfinite(up[0]).sum() > np.isfinite(lp.col_upper).sum()


def test_implied_bounds_per_case_bitexact(oracle_mod):
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    params = fam.sample(5, 3)
    cases = [fam.case(p) for p in params]
    lo, up = pdhg.impliedBounds(fam.base, cases)
    for b, p in enumerate(params):
        want_lo, want_up = oracle_mod.implied_bounds(fam.instance(p))
        assert _same(lo[b], want_lo) and _same(up[b], want_up)


def test_empty_boxes_bitexact(oracle_mod):
    lp = lp_cases.edge_lp(6)
    up = lp.col_upper.copy()
    fin = np.isfinite(up)
    up[fin] = lp.col_lower[fin] - 1.0 * (lp.col_lower[fin] > -np.inf)  # empty boxes
    up[~np.isfinite(lp.col_lower)] = lp.col_upper[~np.isfinite(lp.col_lower)]
    bad = _with_bounds(lp, lp.col_lower, up)
    lo_g, up_g = pdhg.impliedBounds(lp, [LpCase(col_upper=up)])
    want_lo, want_up = oracle_mod.implied_bounds(bad)
    assert _same(lo_g[0], want_lo) and _same(up_g[0], want_up)
