"""The oracle pinned against the reference: this project's C restatement
(oracle/pdhg_oracle.c) must reproduce the reference CPU PDHG bit for bit, the
reference's own known answers (Netlib SC50A / AFIRO pins of
tests/cpp/test_solvers.cpp:112-149) and the committed golden fixtures."""
import glob
import os

import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200.model import Model
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_DATA = os.path.join(O.REFERENCE_SRC, "data", "netlib")


def load_golden(path):
    d = np.load(path)
    lp = Model(num_rows=int(d["num_rows"]), num_cols=int(d["num_cols"]), start=d["start"], index=d["index"],
               value=d["value"], col_cost=d["col_cost"], col_lower=d["col_lower"], col_upper=d["col_upper"],
               row_lower=d["row_lower"], row_upper=d["row_upper"], obj_offset=float(d["obj_offset"]))
    return lp, d


def same(a, b):
    assert a.status == b.status
    assert a.iterations == b.iterations
    assert np.array_equal(a.x, b.x)
    assert np.array_equal(a.y, b.y)
    assert a.objective == b.objective and a.dual_objective == b.dual_objective
    assert a.relative_kkt == b.relative_kkt


@pytest.mark.parametrize("iters", [1, 2, 63, 64, 65, 1000])
def test_oracle_bitexact_vs_reference_fixed_iterations(oracle_mod, iters):
    lp = G.config1(1)
    same(oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters),
         oracle_mod.solve(lp, "ref", tolerance=1e-30, max_iterations=iters))


@pytest.mark.parametrize("seed", [5, 6, 7])
def test_oracle_bitexact_vs_reference_edge_bounds(oracle_mod, seed):
    lp = lp_cases.edge_lp(seed)
    for kw in (dict(tolerance=1e-30, max_iterations=500), dict(tolerance=1e-6, max_iterations=50000)):
        same(oracle_mod.solve(lp, "oracle", **kw), oracle_mod.solve(lp, "ref", **kw))


@pytest.mark.parametrize("kw", [dict(ruiz_iterations=0), dict(pock_chambolle=0), dict(rescale=0),
                                dict(reflection=0.5), dict(check_every=17)])
def test_oracle_bitexact_vs_reference_options(oracle_mod, kw):
    lp = G.random_lp(200, 400, 4.0, 120, 9)
    same(oracle_mod.solve(lp, "oracle", tolerance=1e-5, max_iterations=20000, **kw),
         oracle_mod.solve(lp, "ref", tolerance=1e-5, max_iterations=20000, **kw))


def test_oracle_bitexact_vs_reference_converged_c1(oracle_mod):
    lp = G.config1(1)
    a = oracle_mod.solve(lp, "oracle", tolerance=1e-4)
    same(a, oracle_mod.solve(lp, "ref", tolerance=1e-4))
    assert a.status == 1


def test_oracle_bitexact_vs_reference_batch(oracle_mod):
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    for cases in (lp_cases.cost_sweep_cases(lp, 4), lp_cases.mixed_cases(lp, 6)):
        ra = oracle_mod.solve(lp, "oracle", cases=cases, tolerance=1e-6, max_iterations=100000)
        rb = oracle_mod.solve(lp, "ref", cases=cases, tolerance=1e-6, max_iterations=100000)
        for a, b in zip(ra, rb):
            same(a, b)


def test_oracle_empty_and_degenerate(oracle_mod):
    # no rows at all, and an LP whose A has no nonzeros
    n = 5
    lp0 = Model(num_rows=0, num_cols=n, start=np.zeros(n + 1), index=[], value=[], col_cost=[1, -1, 2, 0, 3],
                col_lower=np.zeros(n), col_upper=np.full(n, 4.0), row_lower=[], row_upper=[])
    lp1 = Model(num_rows=3, num_cols=n, start=np.zeros(n + 1), index=[], value=[], col_cost=[1, -1, 2, 0, 3],
                col_lower=np.zeros(n), col_upper=np.full(n, 4.0), row_lower=[0, -np.inf, -1],
                row_upper=[0, 1, np.inf])
    for lp in (lp0, lp1):
        for kw in (dict(tolerance=1e-6, max_iterations=5000), dict(tolerance=1e-30, max_iterations=130)):
            same(oracle_mod.solve(lp, "oracle", **kw), oracle_mod.solve(lp, "ref", **kw))


def test_ruiz_matches_reference(oracle_mod):
    for lp in (G.config1(3), lp_cases.edge_lp(6)):
        for pc in (True, False):
            rs_a, cs_a = oracle_mod.ruiz(lp, "oracle", 10, pc)
            rs_b, cs_b = oracle_mod.ruiz(lp, "ref", 10, pc)
            assert np.array_equal(rs_a, rs_b) and np.array_equal(cs_a, cs_b)
            # factors are powers of two
            assert np.all(np.frexp(rs_a)[0] == 0.5) and np.all(np.frexp(cs_a)[0] == 0.5)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_oracle_matches_golden(oracle_mod, path):
    lp, d = load_golden(path)
    kw = dict(tolerance=float(d["tolerance"]), max_iterations=int(d["max_iterations"]))
    if bool(d["batch"]):
        from pramana_b200.model import LpCase
        cases = [LpCase(cost=c) for c in d["case_cost"]]
        rs = oracle_mod.solve(lp, "oracle", cases=cases, **kw)
    else:
        rs = [oracle_mod.solve(lp, "oracle", **kw)]
    for b, r in enumerate(rs):
        assert r.status == d["status"][b] and r.iterations == d["iterations"][b]
        assert np.array_equal(r.x, d["x"][b]) and np.array_equal(r.y, d["y"][b])
        assert r.relative_kkt == d["relative_kkt"][b] and r.objective == d["objective"][b]


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data not present")
def test_sc50a_pin(oracle_mod):
    """tests/cpp/test_solvers.cpp:112-122: objective within 1e-5 of the Netlib optimum
    and the safe dual bound from the PDHG duals below it."""
    lp = lp_cases.read_mps(os.path.join(REF_DATA, "sc50a.mps.gz"))
    r = oracle_mod.solve(lp, "oracle", tolerance=1e-7)
    assert r.status == 1
    assert abs(r.objective - (-64.5750770585)) <= 1e-5 * (1 + 64.5750770585)
    same(r, oracle_mod.solve(lp, "ref", tolerance=1e-7))
    assert oracle_mod.safe_dual_bound(lp, r.y) <= -64.5750770585 + 1e-9


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data not present")
def test_afiro_batch_pin(oracle_mod):
    """tests/cpp/test_solvers.cpp:132-149: four cost cases, each within 1e-5 of an exact re-solve."""
    from scipy.optimize import linprog
    lp = lp_cases.read_mps(os.path.join(REF_DATA, "afiro.mps.gz"))
    cases = lp_cases.cost_sweep_cases(lp, 4)
    rs = oracle_mod.solve(lp, "oracle", cases=cases, tolerance=1e-7)
    for cs, r in zip(cases, rs):
        A = np.zeros((lp.num_rows, lp.num_cols))
        for j in range(lp.num_cols):
            A[lp.index[lp.start[j]:lp.start[j + 1]], j] = lp.value[lp.start[j]:lp.start[j + 1]]
        eq = lp.row_lower == lp.row_upper
        ub_rows = ~eq & np.isfinite(lp.row_upper)
        lb_rows = ~eq & np.isfinite(lp.row_lower)
        A_ub = np.vstack([A[ub_rows], -A[lb_rows]])
        b_ub = np.concatenate([lp.row_upper[ub_rows], -lp.row_lower[lb_rows]])
        ref = linprog(cs.cost, A_ub=A_ub, b_ub=b_ub, A_eq=A[eq], b_eq=lp.row_lower[eq],
                      bounds=list(zip(lp.col_lower, [None if not np.isfinite(u) else u for u in lp.col_upper])),
                      method="highs")
        assert r.status == 1
        assert abs(r.objective - (ref.fun + lp.obj_offset)) <= 1e-5 * (1 + abs(ref.fun))


# ---- the reference's published PDHG runs on its refinery planning models ----
# (results/gpu/plan_*.pdhg-{cpu,gpu}_raw1e-{4,6}.json: solve() -> presolve ->
# solvePdhg on the reduced LP; fixtures by tests/golden/make_plan_golden.py)

PLAN_RUNS_CPU = [(p, "pdhg-cpu_raw1e-4") for p in lp_cases.PLANS[:5]] + \
                [(p, "pdhg-gpu_raw1e-6") for p in lp_cases.PLANS[:3]]


@pytest.mark.parametrize("plan,run", PLAN_RUNS_CPU)
def test_oracle_reproduces_published_plan_runs(oracle_mod, plan, run):
    """The C restatement reproduces the reference's published runs: the same
    iteration and restart counts (the reference's GPU and CPU runs agree on
    them) and the same spectral-norm estimate, bit for bit; against its
    published CPU runs (16 threads, whose chunked reductions round a few sums
    differently from one thread on the larger plans) the objective within
    1e-12 and the relative KKT within 1e-9 relative, bit-identical on the
    smaller plans; against its GPU runs (another summation order over 16k+
    iterations) within 1e-12 and 1e-7."""
    lp, pub = lp_cases.load_plan(plan)
    p = pub[run]
    r = oracle_mod.solve(lp, "oracle", tolerance=p["tolerance"])
    st = oracle_mod.solve.last_stats
    assert r.status == 1
    assert st["iterations"] == p["iterations"] and st["restarts"] == p["restarts"]
    assert st["spectral_norm"] == p["spectral_norm_estimate"]
    if "cpu" in run:
        assert abs(r.relative_kkt - p["relative_kkt"]) <= 1e-9 * p["relative_kkt"]
        assert abs(r.objective - p["objective"]) <= 1e-12 * abs(p["objective"])
        assert abs(st["primal_weight"] - p["primal_weight"]) <= 1e-12 * p["primal_weight"]
        if plan in ("plan_6x4", "plan_10x12", "plan_20x12"):
            assert r.objective == p["objective"] and r.relative_kkt == p["relative_kkt"]
    else:
        assert abs(r.relative_kkt - p["relative_kkt"]) <= 1e-7 * p["relative_kkt"]
        assert abs(r.objective - p["objective"]) <= 1e-12 * abs(p["objective"])


def test_oracle_reproduces_published_family_batch(oracle_mod):
    """The batched-PDHG leg of the reference's published repeated-solve
    experiment for plan_10x12's CR03 crude price (64 cases, 1e-6; 16 threads
    on the reference's CPU): the C restatement's batch ends at the published
    18,560 iterations with all 64 cases solved and certified, and the largest
    objective error against the exact optima equals the published one to
    rounding."""
    lp, cases, exact, pub = lp_cases.load_family("plan_10x12_BUY_CR03_0_cost")
    p = pub["cpu"]
    rs = oracle_mod.solve(lp, "oracle", cases=cases, tolerance=1e-6, max_iterations=200000)
    assert oracle_mod.solve.last_stats["iterations"] == p["iterations"]
    assert sum(r.status == 1 for r in rs) == p["solved"]
    err = max(abs(r.objective - e) / max(1.0, abs(e)) for r, e in zip(rs, exact))
    assert abs(err - p["max_relative_error"]) <= 1e-6 * p["max_relative_error"]

    def implied(lp_, cs):
        bounds = [oracle_mod.implied_bounds(lp_, lp_.col_lower, c.col_upper if c.col_upper is not None
                                            else lp_.col_upper) for c in cs]
        return np.stack([b[0] for b in bounds]), np.stack([b[1] for b in bounds])

    def safe(lp_, y, cs):
        out = []
        for b, c in enumerate(cs):
            case_lp = Model(num_rows=lp_.num_rows, num_cols=lp_.num_cols, start=lp_.start, index=lp_.index,
                            value=lp_.value, col_cost=c.cost if c.cost is not None else lp_.col_cost,
                            col_lower=c.col_lower, col_upper=c.col_upper, row_lower=lp_.row_lower,
                            row_upper=lp_.row_upper)
            out.append(oracle_mod.safe_dual_bound(case_lp, y[b * lp_.num_rows:(b + 1) * lp_.num_rows], full=True))
        return out

    class R:  # the oracle's results in the engine's result vocabulary
        def __init__(self, r):
            self.status = "Optimal" if r.status == 1 else "other"
            self.objective, self.rowDual = r.objective, r.y

    assert lp_cases.family_certified(lp, cases, [R(r) for r in rs], safe, implied) == p["certified"]
