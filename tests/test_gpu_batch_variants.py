"""Variants of the FP64 batch kernels (k cases sharing A, k-interleaved
vectors): one or two cases per thread, cached or evict-first streamed
vectors, row entries loaded per lane or once per warp and shared by shuffle,
and the thread layouts: one row's cases per block, or row tiles of 4, 8 or
16 rows per block (one warp per row, 32 cases per chunk).  Every variant does
each case's arithmetic in the same order, so all of them follow the oracle's
batch run exactly and agree with one another bit for bit; the tuner's choice
on a batch larger than L2 is one of them."""
import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200 import pdhg
from test_gpu_parity import assert_close, opts

pytestmark = pytest.mark.gpu

# (cases per thread, streamed) = (1, no), (2, no), (1, yes), (2, yes); + 8, + 16, + 24: row tiles of 4, 8, 16
VARIANTS = [1, 2, 3, 4, 9, 10, 11, 12, 17, 18, 19, 20, 25, 26, 27, 28]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("which", ["sweep", "mixed"])
def test_batch_variant_vs_oracle(oracle_mod, variant, which):
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    # odd k: with two cases per thread, the last thread of each row has one case;
    # in the row-tiled layouts most lanes of each chunk have no case
    cases = lp_cases.cost_sweep_cases(lp, 5) if which == "sweep" else lp_cases.mixed_cases(lp, 7)
    gs = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-6, maxIterations=100000, batchVariant=variant))
    os_ = oracle_mod.solve(lp, "oracle", cases=cases, tolerance=1e-6, max_iterations=100000)
    for g, o in zip(gs, os_):
        assert_close(g, o)


@pytest.mark.parametrize("variant", [5, 6, 7, 8, 13, 14, 15, 16, 21, 22, 23, 24, 29, 30, 31, 32])
@pytest.mark.parametrize("iters", [1, 64, 500])
def test_warp_row_variant_vs_oracle(oracle_mod, variant, iters):
    """k = 64: k / cases per thread is a multiple of 32, so whole warps share
    a row and its entries come by shuffle."""
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    cases = lp_cases.mixed_cases(lp, 64)
    stats = pdhg.PdhgStats()
    gs = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-30, maxIterations=iters, batchVariant=variant))
    os_ = oracle_mod.solve(lp, "oracle", cases=cases, tolerance=1e-30, max_iterations=iters)
    for g, o in zip(gs, os_):
        assert_close(g, o)


def test_batch_variants_agree_bitwise_and_tuner_runs():
    """A batch whose vectors exceed L2 (k (m + n) >= 2^22): the tuned run and
    every forced variant give identical iterates at a fixed iteration count."""
    lp = G.random_lp(20000, 40000, 4.0, 12000, 21)
    k = 128
    rng = np.random.default_rng(4)
    cases = [lp_cases.LpCase(cost=lp.col_cost * (1.0 + 0.05 * rng.standard_normal(lp.num_cols))) for _ in range(k)]
    runs = {}
    for variant in range(33):
        stats = pdhg.PdhgStats()
        rs = pdhg.solvePdhgBatch(lp, cases, opts(tolerance=1e-30, maxIterations=300, batchVariant=variant),
                                 batchStats=stats)
        runs[variant] = rs
    base = runs[1]
    for variant, rs in runs.items():
        for a, b in zip(rs, base):
            assert a.iterations == b.iterations
            assert np.array_equal(a.x, b.x) and np.array_equal(a.rowDual, b.rowDual), variant


@pytest.mark.parametrize("variant", [0, 1, 4, 5, 13, 24])
def test_case_compaction_changes_no_iterate(variant):
    """Cases of uneven difficulty: as they terminate, the live ones are packed
    into narrower interleaves (more than once).  Every case's iterations,
    status and point are bit for bit those of the same batch run without
    packing -- with the warp-row variant too, whose choice falls back when the
    packed width is no multiple of 32."""
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    cases = lp_cases.mixed_cases(lp, 64)
    out = {}
    for off in (False, True):
        with pdhg.Engine(lp, opts(tolerance=1e-6, maxIterations=100000, batchVariant=variant,
                                  batchNoCompaction=off), cases) as e:
            out[off] = (e.solve(), e.last_stats.batch_compactions)
    (packed, n_packed), (plain, n_plain) = out[False], out[True]
    assert n_plain == 0 and n_packed >= 2
    for a, b in zip(packed, plain):
        assert a.status == b.status and a.iterations == b.iterations
        assert np.array_equal(a.x, b.x) and np.array_equal(a.rowDual, b.rowDual)
        assert a.objective == b.objective and a.relativeKkt == b.relativeKkt


def test_compacted_engine_repeats_its_solve():
    """The engine's own buffers come back after a solve that packed its cases:
    a second solve from the same start is identical to the first."""
    lp = G.random_lp(150, 300, 4.0, 90, 13)
    cases = lp_cases.mixed_cases(lp, 16)
    with pdhg.Engine(lp, opts(tolerance=1e-6, maxIterations=100000), cases) as e:
        first = e.solve()
        assert e.last_stats.batch_compactions >= 1
        second = e.solve()
    for a, b in zip(first, second):
        assert a.iterations == b.iterations and np.array_equal(a.x, b.x) and np.array_equal(a.rowDual, b.rowDual)
