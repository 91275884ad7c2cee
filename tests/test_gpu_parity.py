"""Parity of the sm_100a engine with the oracle (the reference PDHG restated,
bit-identical to the reference's CpuBackend) and with the golden fixtures
produced by the reference itself.

Bar: iterates within 1e-9 relative after a fixed number of
iterations, the same termination status, and on converged solves the
reference's own GPU-vs-CPU window of 4 * checkEvery iterations
(tests/cpp/test_solvers.cpp:128).  SpMV is bit-exact."""
import ctypes as C
import glob
import json
import os
import threading
import time

import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200 import pdhg
from pramana_b200.model import Model
from pramana_b200.model import LpCase, Model

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REL_TOL = 1e-9
STATUS = {1: "Optimal", 5: "TimeLimit", 6: "IterationLimit"}


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b))))) if len(b) else 0.0


def assert_close(g, o, exact_iters=True, window=0):
    assert g.status == STATUS[o.status], (g.status, o.status)
    if exact_iters:
        assert g.iterations == o.iterations
    else:
        assert abs(g.iterations - o.iterations) <= window, (g.iterations, o.iterations)
        return
    assert rel_err(g.x, o.x) <= REL_TOL, rel_err(g.x, o.x)
    assert rel_err(g.rowDual, o.y) <= REL_TOL, rel_err(g.rowDual, o.y)
    assert abs(g.relativeKkt - o.relative_kkt) <= REL_TOL * max(1.0, abs(o.relative_kkt))
    assert abs(g.objective - o.objective) <= REL_TOL * (1 + abs(o.objective))


FORMS = [1, 2]  # B2P_KERNELS_FUSED, B2P_KERNELS_RESIDENT


def opts(**kw):
    po = pdhg.PdhgOptions()
    for k, v in kw.items():
        setattr(po, k, v)
    return po


def test_gpu_info():
    assert pdhg.gpuAvailable()
    info = pdhg.gpuInfoJson()
    assert info["available"] is True
    assert info["compute_capability"].startswith("10.")
    assert info["kernel_binary_version"] == 100


@pytest.mark.parametrize("k", [1, 3, 8])
def test_spmv_bitexact(oracle_mod, k):
    rng = np.random.default_rng(k)
    rows, cols = 3000, 1700
    lens = rng.integers(0, 20, size=rows)
    lens[::97] = 0          # empty rows
    lens[5] = 1500          # a long row
    lens[17] = 700
    ptr = np.zeros(rows + 1, dtype=np.int32)
    np.cumsum(lens, out=ptr[1:])
    idx = np.concatenate([np.sort(rng.choice(cols, size=L, replace=False)) for L in lens]).astype(np.int32)
    val = rng.standard_normal(len(idx)) * 10.0 ** rng.uniform(-3, 3, len(idx))
    x = rng.standard_normal(cols * k)
    y = pdhg.csr_spmv(ptr, idx, val, x, rows, cols, k)
    assert np.array_equal(y, oracle_mod.csr_mult(ptr, idx, val, x, rows, k))


@pytest.mark.parametrize("mode", FORMS)
@pytest.mark.parametrize("iters", [1, 2, 63, 64, 65, 1000])
def test_fixed_iterations_c1(oracle_mod, iters, mode):
    lp = G.config1(1)
    g = pdhg.solvePdhg(lp, opts(tolerance=1e-30, maxIterations=iters, kernelMode=mode))
    assert_close(g, oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters))


@pytest.mark.parametrize("mode", FORMS)
def test_before_first_restart_rounding_level(oracle_mod, mode):
    """Before the first restart the iterates differ from the reference only by
    the rounding order of the row sums: far inside the 1e-9 bar."""
    lp = G.config2(2)
    g = pdhg.solvePdhg(lp, opts(tolerance=1e-30, maxIterations=64, kernelMode=mode))
    o = oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=64)
    assert rel_err(g.x, o.x) <= 1e-13 and rel_err(g.rowDual, o.y) <= 1e-13


@pytest.mark.parametrize("mode", FORMS)
def test_kernel_form_reported(mode):
    lp = G.config1(1)
    with pdhg.Engine(lp, opts(tolerance=1e-30, maxIterations=10, kernelMode=mode)) as e:
        e.solve()
        st = e.last_stats
    assert st.kernel_mode == mode
    if mode == 2:
        assert st.resident_blocks > 0 and 0 < st.resident_smem_bytes <= 232448


@pytest.mark.parametrize("mode", FORMS)
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_golden_fixtures(path, mode):
    d = np.load(path)
    lp = Model(num_rows=int(d["num_rows"]), num_cols=int(d["num_cols"]), start=d["start"], index=d["index"],
               value=d["value"], col_cost=d["col_cost"], col_lower=d["col_lower"], col_upper=d["col_upper"],
               row_lower=d["row_lower"], row_upper=d["row_upper"], obj_offset=float(d["obj_offset"]))
    po = opts(tolerance=float(d["tolerance"]), maxIterations=int(d["max_iterations"]), kernelMode=mode)
    if bool(d["batch"]):
        rs = pdhg.solvePdhgBatch(lp, [LpCase(cost=c) for c in d["case_cost"]], po)
    else:
        rs = [pdhg.solvePdhg(lp, po)]

    class Ref:
        pass

    for b, g in enumerate(rs):
        o = Ref()
        o.status, o.iterations = int(d["status"][b]), int(d["iterations"][b])
        o.x, o.y, o.relative_kkt, o.objective = d["x"][b], d["y"][b], float(d["relative_kkt"][b]), float(
            d["objective"][b])
        assert_close(g, o)


@pytest.mark.parametrize("mode", FORMS)
@pytest.mark.parametrize("seed", [5, 6, 7])
def test_edge_bounds(oracle_mod, seed, mode):
    lp = lp_cases.edge_lp(seed)
    for kw in (dict(tolerance=1e-30, max_iterations=500), dict(tolerance=1e-6, max_iterations=50000)):
        g = pdhg.solvePdhg(lp, opts(tolerance=kw["tolerance"], maxIterations=kw["max_iterations"], kernelMode=mode))
        assert_close(g, oracle_mod.solve(lp, "oracle", **kw))


@pytest.mark.parametrize("kw", [dict(ruizIterations=0), dict(pockChambolle=False),
                                dict(rescaleObjectiveAndBounds=False), dict(reflection=0.5), dict(checkEvery=17),
                                dict(maxIterations=1001), dict(useGraphs=False, kernelMode=1),
                                dict(checkEvery=17, kernelMode=2), dict(maxIterations=1001, kernelMode=2),
                                dict(reflection=0.5, kernelMode=2), dict(lanesPerRowA=8, lanesPerRowAT=4, kernelMode=1)])
def test_options(oracle_mod, kw):
    lp = G.random_lp(200, 400, 4.0, 120, 9)
    ok = dict(tolerance=1e-5, max_iterations=20000)
    m = {"ruizIterations": "ruiz_iterations", "pockChambolle": "pock_chambolle",
         "rescaleObjectiveAndBounds": "rescale", "reflection": "reflection", "checkEvery": "check_every",
         "maxIterations": "max_iterations"}
    for k, v in kw.items():
        if k in m:
            ok[m[k]] = int(v) if isinstance(v, bool) else v
    g = pdhg.solvePdhg(lp, opts(tolerance=ok["tolerance"], maxIterations=ok["max_iterations"], **{
        k: v for k, v in kw.items() if k != "maxIterations"}))
    assert_close(g, oracle_mod.solve(lp, "oracle", **ok))


def test_converged_c1_matches_reference_window(oracle_mod):
    lp = G.config1(1)
    g = pdhg.solvePdhg(lp, opts(tolerance=1e-4))
    o = oracle_mod.solve(lp, "oracle", tolerance=1e-4)
    assert g.status == "Optimal"
    assert abs(g.iterations - o.iterations) <= 4 * 64
    assert abs(g.objective - o.objective) <= 1e-5 * (1 + abs(o.objective))


@pytest.mark.parametrize("which", ["sweep", "mixed"])
def test_batch(oracle_mod, which):
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    cases = lp_cases.cost_sweep_cases(lp, 4) if which == "sweep" else lp_cases.mixed_cases(lp, 6)
    gs = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-6, maxIterations=100000))
    os_ = oracle_mod.solve(lp, "oracle", cases=cases, tolerance=1e-6, max_iterations=100000)
    for g, o in zip(gs, os_):
        assert_close(g, o)


def test_batch_equals_individual_solves():
    """Reference test pdhg_batch_equals_individual_solves, against this engine's own single solves."""
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    cases = lp_cases.cost_sweep_cases(lp, 4)
    rb = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-7))
    for cs, r in zip(cases, rb):
        one = Model(**{**lp.__dict__, "col_cost": cs.cost})
        s = pdhg.solvePdhg(one, opts(tolerance=1e-7))
        assert r.status == "Optimal" and s.status == "Optimal"
        assert abs(r.objective - s.objective) <= 1e-5 * (1 + abs(s.objective))


@pytest.mark.parametrize("mode", FORMS)
def test_resolve_is_deterministic(mode):
    lp = G.config1(2)
    with pdhg.Engine(lp, opts(tolerance=1e-4, kernelMode=mode)) as e:
        a = e.solve()[0]
        b = e.solve()[0]
    assert a.iterations == b.iterations and np.array_equal(a.x, b.x) and np.array_equal(a.rowDual, b.rowDual)


def test_time_limit_and_cancel():
    lp = G.config1(3)
    g = pdhg.solvePdhg(lp, opts(tolerance=1e-30, maxIterations=10_000_000, timeLimit=0.2))
    assert g.status == "TimeLimit"
    assert 0 < g.iterations < 10_000_000
    flag = (C.c_int32 * 1)(0)

    def cancel():
        time.sleep(0.2)
        flag[0] = 1

    th = threading.Thread(target=cancel)
    th.start()
    g = pdhg.solvePdhg(lp, opts(tolerance=1e-30, maxIterations=10_000_000), cancel_flag=flag)
    th.join()
    assert g.status == "TimeLimit"


def test_empty_rows_and_no_rows(oracle_mod):
    n = 5
    lp1 = Model(num_rows=3, num_cols=n, start=np.zeros(n + 1), index=[], value=[], col_cost=[1, -1, 2, 0, 3],
                col_lower=np.zeros(n), col_upper=np.full(n, 4.0), row_lower=[0, -np.inf, -1],
                row_upper=[0, 1, np.inf])
    lp0 = Model(num_rows=0, num_cols=n, start=np.zeros(n + 1), index=[], value=[], col_cost=[1, -1, 2, 0, 3],
                col_lower=np.zeros(n), col_upper=np.full(n, 4.0), row_lower=[], row_upper=[])
    for lp in (lp0, lp1):
        for kw in (dict(tolerance=1e-6, max_iterations=5000), dict(tolerance=1e-30, max_iterations=130)):
            g = pdhg.solvePdhg(lp, opts(tolerance=kw["tolerance"], maxIterations=kw["max_iterations"]))
            assert_close(g, oracle_mod.solve(lp, "oracle", **kw))


def _host_kkt(lp: Model, x, y):
    """Relative KKT of (x, y) in the original space, as runPdhg measures it (src/pdhg/pdhg.cpp:608-615)."""
    ax = lp.row_activity(x)
    res = np.maximum(lp.row_lower - ax, 0) + np.maximum(ax - lp.row_upper, 0)
    fin = lambda v: np.abs(v) < 1e20  # noqa: E731
    rhs = np.sqrt(np.sum(np.where(fin(lp.row_lower), lp.row_lower, 0) ** 2) + np.sum(
        np.where(fin(lp.row_upper) & (lp.row_upper != lp.row_lower), lp.row_upper, 0) ** 2))
    relP = np.linalg.norm(res) / (1 + rhs)
    cols = np.repeat(np.arange(lp.num_cols), np.diff(lp.start))
    aty = np.zeros(lp.num_cols)
    np.add.at(aty, cols, lp.value * y[lp.index])
    d = lp.col_cost - aty
    hl, hu = fin(lp.col_lower), fin(lp.col_upper)
    dres = np.where(~hl & ~hu, np.abs(d), np.where(~hl, np.maximum(d, 0), np.where(~hu, np.maximum(-d, 0), 0)))
    relD = np.linalg.norm(dres) / (1 + np.linalg.norm(lp.col_cost))
    pobj = lp.col_cost @ x
    dobj = np.sum(np.where((y > 0) & fin(lp.row_lower), y * np.where(fin(lp.row_lower), lp.row_lower, 0), 0)) + \
        np.sum(np.where((y < 0) & fin(lp.row_upper), y * np.where(fin(lp.row_upper), lp.row_upper, 0), 0)) + \
        np.sum(np.where((d > 0) & hl, d * np.where(hl, lp.col_lower, 0), 0)) + \
        np.sum(np.where((d < 0) & hu, d * np.where(hu, lp.col_upper, 0), 0))
    gap = abs(pobj - dobj) / (1 + abs(pobj) + abs(dobj))
    return relP, relD, gap


@pytest.mark.parametrize("mode", FORMS)
def test_c2_full_size_properties(oracle_mod, mode):
    """m=40k, n=80k, 512k nnz (skewed rows) to 1e-6: too long for the oracle at
    this size, so check size-independent properties: the returned point's KKT
    recomputed on the host meets the tolerance, the iteration count matches
    the reference run of the same LP (20,287 +- 4 checks), and the
    reference's outward-rounded dual bound is valid and tight."""
    lp = G.config2(2)
    g = pdhg.solvePdhg(lp, opts(tolerance=1e-6, kernelMode=mode))
    assert g.status == "Optimal"
    assert abs(g.iterations - 20287) <= 4 * 64
    relP, relD, gap = _host_kkt(lp, g.x, g.rowDual)
    assert max(relP, relD, gap) <= 1.000001e-6
    assert abs(max(relP, relD, gap) - g.relativeKkt) <= 1e-9
    lb = oracle_mod.safe_dual_bound(lp, g.rowDual)
    assert lb <= g.objective + 1e-9 * abs(g.objective)
    assert abs(g.objective - lb) <= 1e-4 * (1 + abs(g.objective))


@pytest.mark.parametrize("which", ["c1", "edge", "batch"])
def test_kkt_residual_matches_host(which):
    """b2p_kkt_residual against the same KKT formula evaluated on the host."""
    if which == "batch":
        lp = G.random_lp(150, 300, 4.0, 90, 13)
        cases = lp_cases.mixed_cases(lp, 5)
        rs = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-5))
        x = np.concatenate([r.x for r in rs])
        y = np.concatenate([r.rowDual for r in rs])
        got = pdhg.kktResidual(lp, x, y, cases)
        for b, cs in enumerate(cases):
            one = Model(**{**lp.__dict__, **{f: getattr(cs, f) for f in ("row_lower", "row_upper", "col_lower",
                                                                          "col_upper") if getattr(cs, f) is not None},
                           "col_cost": cs.cost if cs.cost is not None else lp.col_cost})
            want = _host_kkt(one, rs[b].x, rs[b].rowDual)
            assert np.allclose(got[b, :3], want, rtol=1e-9, atol=1e-15)
            assert abs(got[b, 3] - rs[b].relativeKkt) <= 1e-9 * max(1e-12, rs[b].relativeKkt) + 1e-15
        return
    lp = G.config1(1) if which == "c1" else lp_cases.edge_lp(6)
    r = pdhg.solvePdhg(lp, opts(tolerance=1e-6))
    got = pdhg.kktResidual(lp, r.x, r.rowDual)[0]
    want = _host_kkt(lp, r.x, r.rowDual)
    assert np.allclose(got[:3], want, rtol=1e-9, atol=1e-15)
    assert got[3] == max(got[:3])
    # the engine's own KKT at termination is the same quantity
    assert abs(got[3] - r.relativeKkt) <= 1e-9 * r.relativeKkt + 1e-15


@pytest.mark.parametrize("which", ["c1", "c2", "edge"])
def test_spectral_norm_bitexact(oracle_mod, which):
    """The ||A|| estimate (products on the device, norm on the host) is bit-identical to the reference's."""
    lp = {"c1": lambda: G.config1(1), "c2": lambda: G.config2(2), "edge": lambda: lp_cases.edge_lp(5)}[which]()
    g = pdhg.solvePdhg(lp, opts(tolerance=1e-30, maxIterations=1))
    oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=1)
    assert g.stats.spectralNorm == oracle_mod.solve.last_stats["spectral_norm"]


MIXED = 1  # B2P_PRECISION_MIXED


# Objective error of a mixed-form answer against the FP64 oracle's answer and
# against the exact optimum: both PDHG answers are tol-points of the LP, so
# they agree to a few tolerances, not to rounding.
MIXED_OBJ_FACTOR = 10


def _fp64_answers(oracle_mod, which, lp, tol):
    """(FP64 oracle objective, exact optimum) of the LP: the oracle and the
    reference's simplex run here for the small LPs; for config-2 the stored
    answers of one full run each (tests/golden/answers.json)."""
    if which == "c2":
        with open(os.path.join(os.path.dirname(__file__), "golden", "answers.json")) as f:
            a = json.load(f)["config2"]
        return a[f"{tol:g}"]["objective"], a["exact"]["objective"]
    o = oracle_mod.solve(lp, "oracle", tolerance=tol, max_iterations=400000)
    assert o.status == 1
    return o.objective, oracle_mod.simplex(lp)["objective"]


@pytest.mark.parametrize("which,tol", [("c1", 1e-4), ("c1", 1e-6), ("edge", 1e-6), ("c2", 1e-6), ("c2", 1e-8)])
def test_mixed_precision_meets_tolerance_in_fp64(oracle_mod, which, tol):
    """Mixed form: FP32 iterates, FP64 checks; the returned point's KKT,
    recomputed on the host in FP64, meets the tolerance, and its objective is
    within MIXED_OBJ_FACTOR tolerances of the FP64 oracle's answer and of the
    exact optimum."""
    lp = {"c1": lambda: G.config1(1), "c2": lambda: G.config2(2), "edge": lambda: lp_cases.edge_lp(6)}[which]()
    with pdhg.Engine(lp, opts(tolerance=tol, precision=MIXED)) as e:
        r = e.solve()[0]
        st = e.last_stats
    assert r.status == "Optimal"
    assert st.precision_used == MIXED and st.fp32_iterations > 0
    relP, relD, gap = _host_kkt(lp, r.x, r.rowDual)
    assert max(relP, relD, gap) <= tol * (1 + 1e-6)
    oracle_obj, exact = _fp64_answers(oracle_mod, which, lp, tol)
    assert abs(r.objective - oracle_obj) <= MIXED_OBJ_FACTOR * tol * (1 + abs(oracle_obj)), (r.objective, oracle_obj)
    assert abs(r.objective - exact) <= MIXED_OBJ_FACTOR * tol * (1 + abs(exact)), (r.objective, exact)


def _case_model(lp, cs):
    return Model(**{**lp.__dict__, **{f: getattr(cs, f) for f in ("row_lower", "row_upper", "col_lower", "col_upper")
                                      if getattr(cs, f) is not None},
                    "col_cost": cs.cost if cs.cost is not None else lp.col_cost})


@pytest.mark.parametrize("which", ["random", "family"])
def test_mixed_precision_batch_meets_tolerance_in_fp64(which):
    """Mixed form of a batch (k-interleaved FP32 kernels): every case returns
    Optimal, its KKT recomputed on the host in FP64 meets the tolerance, and
    its objective stays within a few tolerances of the plain FP64 batch's."""
    if which == "random":
        lp = G.random_lp(400, 800, 4.0, 240, 13)
        cases = lp_cases.mixed_cases(lp, 8)
    else:
        from pramana_b200 import warmstart as W
        fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
        lp = fam.base
        cases = [fam.case(p) for p in fam.sample(32, 4)]
    tol = 1e-6
    with pdhg.Engine(lp, opts(tolerance=tol, precision=MIXED, maxIterations=400000), cases) as e:
        rs = e.solve()
        st = e.last_stats
    assert st.precision_used == MIXED and st.fp32_iterations > 0
    ref = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=tol, maxIterations=400000))
    for cs, r, q in zip(cases, rs, ref):
        assert r.status == "Optimal" and q.status == "Optimal"
        relP, relD, gap = _host_kkt(_case_model(lp, cs), r.x, r.rowDual)
        assert max(relP, relD, gap) <= tol * (1 + 1e-6)
        assert abs(r.objective - q.objective) <= 10 * tol * (1 + abs(q.objective))


def test_mixed_batch_iteration_limit_returns_fp64_measure():
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    cases = lp_cases.cost_sweep_cases(lp, 3)
    rs = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-12, precision=MIXED, maxIterations=300))
    for cs, r in zip(cases, rs):
        assert r.status == "IterationLimit"
        assert abs(r.relativeKkt - max(_host_kkt(_case_model(lp, cs), r.x, r.rowDual))) <= 1e-6 * (1 + r.relativeKkt)


@pytest.mark.parametrize("mode", FORMS)
def test_warm_start_from_solution_and_back_to_cold(mode):
    lp = G.config1(1)
    with pdhg.Engine(lp, opts(tolerance=1e-6, kernelMode=mode)) as e:
        cold = e.solve()[0]
        e.set_start(cold.x, cold.rowDual, cold.stats.primalWeight)
        warm = e.solve()[0]
        e.set_start(None, None)
        cold2 = e.solve()[0]
    assert cold.status == warm.status == "Optimal"
    assert warm.iterations <= 64  # the first check already meets the tolerance
    assert abs(warm.objective - cold.objective) <= 1e-5 * (1 + abs(cold.objective))
    assert cold2.iterations == cold.iterations and np.array_equal(cold2.x, cold.x)
