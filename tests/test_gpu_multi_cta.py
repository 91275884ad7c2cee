"""The CTA form of the multi-LP engine (one thread block runs one LP's whole
PDHG loop, restart and termination decisions included): every LP must follow
the reference algorithm as if solved alone -- iterates against the oracle at
fixed iteration counts in each storage tier, and to convergence."""
import ctypes as C
import threading
import time

import numpy as np
import pytest

from pramana_b200 import _lib
from pramana_b200 import generators as G
from pramana_b200 import pdhg
from pramana_b200 import warmstart as W
from test_gpu_multi import family
from test_gpu_parity import _host_kkt, assert_close, opts

pytestmark = pytest.mark.gpu

CTA = dict(multiForm=_lib.MULTI_CTA)


def _stats():
    return pdhg.solvePdhgMulti.last_stats


@pytest.mark.parametrize("iters", [1, 64, 1000])
def test_cta_fixed_iterations_vs_oracle(oracle_mod, iters):
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=iters, **CTA))
    st = _stats()
    assert st.multi_form == _lib.MULTI_CTA and st.kernel_launches == 1
    for lp, r in zip(lps, rs):
        assert_close(r, oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters))


@pytest.mark.parametrize("limit,tiers", [(0, None), (64 * 1024, None), (1, (0, 0))])
def test_cta_storage_tiers_vs_oracle(oracle_mod, limit, tiers):
    """Shared-memory limits that move LPs between the three storage tiers
    (all in shared memory / iterates only / global memory)."""
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=300, ctaSmemLimit=limit, **CTA))
    st = _stats()
    if tiers is not None:
        assert (st.cta_lps_smem, st.cta_lps_vectors) == tiers
    else:
        assert st.cta_lps_smem >= 1
    for lp, r in zip(lps, rs):
        assert_close(r, oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=300))


def test_cta_mixed_tiers_counts():
    lps = family()
    pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=10, ctaSmemLimit=64 * 1024, **CTA))
    st = _stats()
    # the 2000 x 4000 LP (25.6k nonzeros) keeps only nothing / its iterates in 64 KB
    assert st.cta_lps_smem + st.cta_lps_vectors < len(lps)
    assert st.cta_smem_bytes <= 64 * 1024


def test_cta_converged_vs_oracle(oracle_mod):
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, maxIterations=200000, **CTA))
    for lp, r in zip(lps, rs):
        o = oracle_mod.solve(lp, "oracle", tolerance=1e-6, max_iterations=200000)
        assert r.status == "Optimal" and o.status == 1
        assert abs(r.iterations - o.iterations) <= 4 * 64
        assert abs(r.objective - o.objective) <= 1e-5 * (1 + abs(o.objective))
        if lp.num_rows:
            assert max(_host_kkt(lp, r.x, r.rowDual)) <= 1e-6 * (1 + 1e-6)


def test_cta_iteration_limit_reports_every_instance(oracle_mod):
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=100, **CTA))
    for lp, r in zip(lps, rs):
        o = oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=100)
        assert r.status == {1: "Optimal", 6: "IterationLimit"}[o.status] and r.iterations == o.iterations


def test_cta_matches_grid_form():
    """Both forms run the same algorithm; to 1e-6 they agree on status,
    iteration counts (within a few checks) and objectives."""
    lps = family()
    a = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, **CTA))
    b = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, multiForm=_lib.MULTI_GRID))
    assert _stats().multi_form == _lib.MULTI_GRID
    for ra, rb in zip(a, b):
        assert ra.status == rb.status == "Optimal"
        assert abs(ra.iterations - rb.iterations) <= 4 * 64
        assert abs(ra.objective - rb.objective) <= 1e-5 * (1 + abs(rb.objective))


def test_cta_warm_start():
    lps = family()[:6]
    cold = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, **CTA))
    starts = [(r.x, r.rowDual) if b % 2 == 0 else None for b, r in enumerate(cold)]
    warm = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, **CTA), starts=starts)
    for b, (c, w) in enumerate(zip(cold, warm)):
        assert w.status == "Optimal"
        if b % 2 == 0:
            assert w.iterations <= 64
        else:
            assert w.iterations == c.iterations


def test_cta_time_limit_and_cancel():
    lps = [G.random_lp(300, 600, 4.0, 180, 50 + i) for i in range(4)]
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=100_000_000, timeLimit=0.2, **CTA))
    assert all(r.status == "TimeLimit" and 0 < r.iterations < 100_000_000 for r in rs)
    flag = (C.c_int32 * 1)(0)

    def cancel():
        time.sleep(0.2)
        flag[0] = 1

    th = threading.Thread(target=cancel)
    th.start()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=100_000_000, **CTA), cancel_flag=flag)
    th.join()
    assert all(r.status == "TimeLimit" for r in rs)


def test_cta_auto_picks_cta_for_small_family():
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    params = fam.sample(64, seed=11)
    lps = [fam.instance(p) for p in params]
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6))
    st = _stats()
    assert st.multi_form == _lib.MULTI_CTA and st.cta_lps_smem == len(lps)
    assert st.cta_threads in (128, 256, 512)
    g = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, multiForm=_lib.MULTI_GRID))
    for lp, a, b in zip(lps, rs, g):
        assert a.status == b.status == "Optimal"
        assert max(_host_kkt(lp, a.x, a.rowDual)) <= 1e-6 * (1 + 1e-6)
        assert abs(a.objective - b.objective) <= 1e-5 * (1 + abs(b.objective))


def test_cta_uneven_batch_not_auto():
    """AUTO keeps the block-diagonal form when an LP does not fit in one
    block's shared memory."""
    lps = G.uneven_family(4, 1e4, 3e4, seed=3)
    pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=64))
    assert _stats().multi_form == _lib.MULTI_GRID


# ---- owner kernel (each thread owns 1 or 2 rows and columns) ----

def small_family():
    """LPs of at most 500 rows / columns, including one whose rows are all
    empty, one without rows and a refinery family member."""
    import lp_cases
    from pramana_b200.model import Model
    lps = [G.random_lp(m, 2 * m, 4.0, int(0.6 * m), 300 + i) for i, m in enumerate([40, 250, 120, 7])]
    lps.append(lp_cases.edge_lp(5))
    n = 5
    lps.append(Model(num_rows=0, num_cols=n, start=np.zeros(n + 1), index=[], value=[], col_cost=[1, -1, 2, 0, 3],
                     col_lower=np.zeros(n), col_upper=np.full(n, 4.0), row_lower=[], row_upper=[]))
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    lps.append(fam.instance(fam.sample(1, seed=3)[0]))
    return lps


@pytest.mark.parametrize("kernel,threads", [(_lib.CTA_OWNER1, 512), (_lib.CTA_OWNER2, 256), (_lib.CTA_OWNER2, 512),
                                            (_lib.CTA_GENERAL, 128)])
@pytest.mark.parametrize("iters", [1, 64, 1000])
def test_owner_kernel_fixed_iterations_vs_oracle(oracle_mod, kernel, threads, iters):
    lps = small_family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=iters, ctaKernel=kernel, ctaThreads=threads,
                                       **CTA))
    st = _stats()
    assert st.cta_threads == threads
    assert st.cta_owned_per_thread == {_lib.CTA_OWNER1: 1, _lib.CTA_OWNER2: 2, _lib.CTA_GENERAL: 0}[kernel]
    for lp, r in zip(lps, rs):
        assert_close(r, oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters))


def test_owner_and_general_kernels_agree_bitwise():
    """Same arithmetic element by element and the same reductions' inputs:
    the two kernels' answers are identical to convergence."""
    lps = small_family()
    a = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, ctaKernel=_lib.CTA_OWNER2, ctaThreads=256, **CTA))
    b = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, ctaKernel=_lib.CTA_GENERAL, ctaThreads=256, **CTA))
    for ra, rb in zip(a, b):
        assert ra.status == rb.status == "Optimal"
        assert ra.iterations == rb.iterations
        assert np.array_equal(ra.x, rb.x) and np.array_equal(ra.rowDual, rb.rowDual)


def test_owner_kernel_refused_when_too_large():
    lps = small_family()
    with pytest.raises(Exception):
        pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, ctaKernel=_lib.CTA_OWNER1, ctaThreads=128, **CTA))


def test_owner_kernel_converged_and_warm(oracle_mod):
    lps = small_family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, ctaKernel=_lib.CTA_OWNER2, **CTA))
    for lp, r in zip(lps, rs):
        o = oracle_mod.solve(lp, "oracle", tolerance=1e-6, max_iterations=200000)
        assert r.status == "Optimal" and o.status == 1
        assert abs(r.iterations - o.iterations) <= 4 * 64
        if lp.num_rows:
            assert max(_host_kkt(lp, r.x, r.rowDual)) <= 1e-6 * (1 + 1e-6)
    starts = [(r.x, r.rowDual) for r in rs]
    warm = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, ctaKernel=_lib.CTA_OWNER2, **CTA), starts=starts)
    ref = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, ctaKernel=_lib.CTA_GENERAL, **CTA), starts=starts)
    for r, w, g in zip(rs, warm, ref):
        assert w.status == "Optimal" and w.iterations <= r.iterations
        assert w.iterations == g.iterations and np.array_equal(w.x, g.x)


@pytest.mark.parametrize("iters", [1, 2, 63, 64])
@pytest.mark.parametrize("kernel", [_lib.CTA_GENERAL, _lib.CTA_OWNER2])
def test_cta_iterates_bit_identical_to_oracle(oracle_mod, iters, kernel):
    """The CTA kernels sum every row left to right, as the reference does, and
    each LP's ||A|| (the device power iteration over the whole batch) equals
    its own sequential estimate bit for bit: up to the first check (whose
    sums are reduced in another order) the iterates are the oracle's
    exactly, for every LP of the batch."""
    lps = [G.random_lp(m, 2 * m, 4.0, int(0.6 * m), 600 + i) for i, m in enumerate([30, 100, 250, 450])]
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    lps.append(fam.instance(fam.sample(1, seed=8)[0]))
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=iters, ctaKernel=kernel, **CTA))
    for lp, r in zip(lps, rs):
        o = oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters)
        assert np.array_equal(r.x, o.x) and np.array_equal(r.rowDual, o.y)


# ---- mixed precision in the CTA form -----------------------------------------

MIXED = dict(multiForm=_lib.MULTI_CTA, precision=_lib.PRECISION_MIXED)
# Objective error of a mixed-form answer against the FP64 oracle's answer at
# the same tolerance: both are 1e-6 points of the same LP, so they agree to
# the tolerance's order, not to rounding.
MIXED_OBJ_TOL = 1e-5


@pytest.mark.parametrize("limit", [0, 64 * 1024, 1])
def test_cta_mixed_converged_vs_fp64_oracle(oracle_mod, limit):
    """FP32 run, FP64 re-measure and FP64 continuation, in each storage tier
    of the FP32 run: every LP ends Optimal with its KKT recomputed in FP64 on
    the host <= tol, and its objective within MIXED_OBJ_TOL of the FP64
    oracle's."""
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, maxIterations=200000, ctaSmemLimit=limit, **MIXED))
    st = _stats()
    assert st.multi_form == _lib.MULTI_CTA and st.precision_used == _lib.PRECISION_MIXED
    assert st.fp32_iterations > 0
    for lp, r in zip(lps, rs):
        o = oracle_mod.solve(lp, "oracle", tolerance=1e-6, max_iterations=200000)
        assert r.status == "Optimal" and o.status == 1
        assert abs(r.objective - o.objective) <= MIXED_OBJ_TOL * (1 + abs(o.objective)), (r.objective, o.objective)
        if lp.num_rows:
            assert max(_host_kkt(lp, r.x, r.rowDual)) <= 1e-6 * (1 + 1e-6)
        # within the bounds up to the rounding of the unscaling x = x_scaled * C * beta
        slack = 1e-12 * (1 + np.abs(r.x))
        assert np.all(r.x >= lp.col_lower - slack) and np.all(r.x <= lp.col_upper + slack)


def test_cta_mixed_refinery_family_vs_fp64():
    """A refinery family: the mixed form's answers meet the tolerance in FP64
    and match the plain FP64 CTA form's objectives."""
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    lps = [fam.instance(p) for p in fam.sample(24, 11)]
    plain = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, maxIterations=400000, **CTA))
    mixed = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, maxIterations=400000, **MIXED))
    for lp, p, q in zip(lps, plain, mixed):
        assert p.status == q.status == "Optimal"
        assert max(_host_kkt(lp, q.x, q.rowDual)) <= 1e-6 * (1 + 1e-6)
        assert abs(p.objective - q.objective) <= MIXED_OBJ_TOL * (1 + abs(p.objective))


def test_cta_mixed_iteration_limit_and_time_limit():
    lps = family()
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-12, maxIterations=640, **MIXED))
    for r in rs:
        assert r.status in ("Optimal", "IterationLimit") and r.iterations <= 640
    # a time limit reaches the runs through the mapped stop flag
    lps = [G.random_lp(300, 600, 4.0, 180, 50 + i) for i in range(4)]
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=100_000_000, timeLimit=0.2, **MIXED))
    assert all(r.status == "TimeLimit" and 0 < r.iterations < 100_000_000 for r in rs)


@pytest.mark.parametrize("form", [_lib.MULTI_CTA, _lib.MULTI_GRID])
@pytest.mark.parametrize("iters", [1, 64, 1000])
def test_primal_weight_start_vs_oracle(oracle_mod, form, iters):
    """Starting primal weights (original-space units): every LP given one
    follows the oracle started from the same weight, iterate for iterate, in
    both forms; the others (weights 0, -1, nan) keep the default start."""
    lps = family()
    w = [0.37, 0.0, 2.5, -1.0, 11.0, np.nan, 0.05, 1.0]
    rs = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-30, maxIterations=iters, multiForm=form), primalWeights=w)
    for lp, r, wb in zip(lps, rs, w):
        start = wb if np.isfinite(wb) and wb > 0 else 0.0
        assert_close(r, oracle_mod.solve(lp, "oracle", tolerance=1e-30, max_iterations=iters,
                                         primal_weight_start=start))
        assert np.isfinite(r.primalWeight) and r.primalWeight > 0


def test_primal_weight_round_trip():
    """Each LP's final weight comes back finite and positive, and a solve
    restarted from the cold solve's point and final weight converges to the
    same objective."""
    lps = family()[:6]
    cold = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, **CTA))
    w = [r.primalWeight for r in cold]
    assert all(np.isfinite(x) and x > 0 for x in w)
    warm = pdhg.solvePdhgMulti(lps, opts(tolerance=1e-6, **CTA), starts=[(r.x, r.rowDual) for r in cold],
                               primalWeights=w)
    for c, r in zip(cold, warm):
        assert r.status == "Optimal"
        assert abs(r.objective - c.objective) <= 1e-5 * (1 + abs(c.objective))


def _vectors_ptr_bytes(lp):
    """Shared memory of an LP whose iterates and row pointers are in shared
    memory and whose operators are not (FP64)."""
    m, n = lp.num_rows, lp.num_cols
    return 8 * (3 * n + 6 * m) + (4 * ((m + 1) + (n + 1)) + 7) // 8 * 8


@pytest.mark.parametrize("precision", [_lib.PRECISION_FP64, _lib.PRECISION_MIXED])
@pytest.mark.parametrize("shared", [True, False])
@pytest.mark.parametrize("limit", ["vectors", "auto"])
def test_sliced_operators_change_no_iterate(precision, shared, limit):
    """The CTA form's sliced-ELL operators (read from global memory by LPs
    whose vectors fit shared memory but whose operators do not) sum every
    row in the CSR's order: iterates, statuses and iteration counts bit for
    bit those of the CSR layout -- for a family sharing one operator and for
    LPs with their own, in FP64 and in the mixed form."""
    if shared:
        fam = W.RefineryFamily(seed=5, periods=3, regions=2, units=5, streams=5, properties=3, pools=12,
                               scale_exponent=0.0)
        lps = [fam.instance(p) for p in fam.sample(12, 4)]
    else:
        lps = [G.random_lp(m, 2 * m, 5.0, int(0.6 * m), 300 + i) for i, m in enumerate([40, 333, 700, 1500, 65])]
    # "vectors": a limit that leaves the largest LP's iterates and row
    # pointers in shared memory and its operators in global memory; "auto":
    # each LP in the tier its size gets
    smem = max(_vectors_ptr_bytes(lp) for lp in lps) if limit == "vectors" else 0
    out = {}
    for layout in (_lib.CTA_LAYOUT_CSR, _lib.CTA_LAYOUT_AUTO):
        o = opts(tolerance=1e-6, maxIterations=20000, precision=precision, ctaSmemLimit=smem, ctaLayout=layout,
                 **CTA)
        out[layout] = pdhg.solvePdhgMulti(lps, o)
        assert _stats().multi_form == _lib.MULTI_CTA
        if smem:
            assert _stats().cta_lps_vectors > 0
            assert _stats().cta_sliced == (layout == _lib.CTA_LAYOUT_AUTO)
    for a, b in zip(out[_lib.CTA_LAYOUT_CSR], out[_lib.CTA_LAYOUT_AUTO]):
        assert a.status == b.status and a.iterations == b.iterations
        assert np.array_equal(a.x, b.x) and np.array_equal(a.rowDual, b.rowDual)
