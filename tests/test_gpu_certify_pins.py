"""The reference's own certifier tests (tests/cpp/test_core.cpp:175-218) on
this engine's batched entries: on min x + y s.t. x + 2y >= 4, 3x + y >= 6,
0 <= x, y <= 10 (optimum 2.8 at (1.6, 1.2), duals (0.4, 0.2)) the safe bound
of the optimal duals is 2.8 and that of 200 random duals (the reference's
SplitMix64 stream, seed 1) never exceeds it, bit-identical to the reference;
a true OPTIMAL claim is accepted, an infeasible, a suboptimal and a NaN one
are rejected."""
import numpy as np
import pytest

from pramana_b200 import generators as G
from pramana_b200 import pdhg
from pramana_b200.model import LpCase, Model

pytestmark = pytest.mark.gpu


def tiny():
    return Model(num_rows=2, num_cols=2, start=[0, 2, 4], index=[0, 1, 0, 1], value=[1.0, 3.0, 2.0, 1.0],
                 col_cost=[1.0, 1.0], col_lower=[0.0, 0.0], col_upper=[10.0, 10.0], row_lower=[4.0, 6.0],
                 row_upper=[np.inf, np.inf])


def test_safe_bound_valid_for_any_dual(oracle_mod):
    lp = tiny()
    b = pdhg.safeDualBound(lp, [0.4, 0.2])[0]["bound"]
    assert abs(b - 2.8) <= 1e-12 * (1 + 2.8) and b <= 2.8
    u = (G._splitmix64(1, 0, 400) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    ys = u * 2 - 0.5
    bounds = [r["bound"] for r in pdhg.safeDualBound(lp, ys, [LpCase() for _ in range(200)])]
    assert max(bounds) <= 2.8 + 1e-12
    if oracle_mod.available("ref"):
        ref = [oracle_mod.safe_dual_bound(lp, ys[2 * t:2 * t + 2], full=True)["bound"] for t in range(200)]
        assert bounds == ref


def test_certifier_rejects_false_claims():
    lp = tiny()
    xs = [[1.6, 1.2], [1.0, 1.0], [2.0, 2.0], [np.nan, 1.0]]
    out = pdhg.certifyLp(lp, np.array(xs).ravel(), np.tile([0.4, 0.2], 4), [LpCase() for _ in range(4)])
    assert [bool(c["accepted"]) for c in out] == [True, False, False, False]
