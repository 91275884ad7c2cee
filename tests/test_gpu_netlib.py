"""The reference's own GPU-path tests (tests/cpp/test_solvers.cpp:112-149),
run on this engine: SC50A to 1e-7 reaches the Netlib optimum within 1e-5,
its outward-rounded dual bound is valid, and the iteration count is within
the reference's GPU-vs-CPU window of its CPU run; AFIRO's four cost cases in
one batch each reach the simplex optimum within 1e-5.  Fixtures by
tests/golden/make_netlib_golden.py (the reference's MPS reader)."""
import os

import numpy as np
import pytest

from pramana_b200 import pdhg
from pramana_b200.model import LpCase, Model
from test_gpu_parity import opts

pytestmark = pytest.mark.gpu

NETLIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "netlib")
SC50A_OPT = -64.5750770585


def load(name):
    d = np.load(os.path.join(NETLIB, name + ".npz"))
    lp = Model(num_rows=int(d["num_rows"]), num_cols=int(d["num_cols"]), start=d["start"], index=d["index"],
               value=d["value"], col_cost=d["col_cost"], col_lower=d["col_lower"], col_upper=d["col_upper"],
               row_lower=d["row_lower"], row_upper=d["row_upper"], obj_offset=float(d["obj_offset"]), name=name)
    return lp, d


@pytest.mark.parametrize("precision", [0, 1])
def test_sc50a_optimum_bound_and_iteration_window(precision):
    lp, d = load("sc50a")
    r = pdhg.solvePdhg(lp, opts(tolerance=1e-7, precision=precision))
    assert r.status == "Optimal"
    assert abs(r.objective - SC50A_OPT) <= 1e-5
    assert pdhg.safeDualBound(lp, r.rowDual)[0]["bound"] + lp.obj_offset <= SC50A_OPT + 1e-9
    if precision == 0:
        assert abs(r.iterations - int(d["ref_iterations"])) <= 4 * 64
        assert abs(r.objective - float(d["ref_objective"])) <= 1e-5


def test_afiro_batch_matches_simplex():
    lp, d = load("afiro")
    cases = []
    for k in range(4):
        c = lp.col_cost.copy()
        c[1] = -0.4 + 0.1 * k
        cases.append(LpCase(cost=c))
    rs = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-7))
    for r, opt in zip(rs, d["case_optima"]):
        assert r.status == "Optimal"
        assert abs(r.objective - opt) <= 1e-5
