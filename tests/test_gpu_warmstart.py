"""The learned warm start end to end on the B200, on a 164 x 324 refinery-
planning family (16 parameters: 6 crude prices, 10 demand scales):
training solutions from batched cold PDHG, a PCA basis of [x; y], the BF16
tensor-core MLP trained on the GPU, then held-out members solved cold, from
the nearest training solution and from the network's prediction.  The test
shows what the network gains: fewer iterations than the cold start and than
the nearest-neighbour start, and every warm-started answer certified (KKT
recomputed <= 1e-6, safe dual bound within the reference's family rule)."""
import numpy as np
import pytest

from pramana_b200 import warmstart as W
from pramana_b200.mlp import TrainOptions
from pramana_b200.pdhg import PdhgOptions

pytestmark = pytest.mark.gpu

SIZE = dict(periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)


@pytest.fixture(scope="module")
def trained():
    fam = W.RefineryFamily(seed=5, **SIZE)
    opts = PdhgOptions(tolerance=1e-6, maxIterations=200000)
    P = fam.sample(4096, 100)
    tr = W.solve_family(fam, P, opts)
    ok = tr.status == 1
    lw = W.LearnedWarmStart(fam, seed=1)
    losses = lw.fit(P[ok], tr.X[ok], tr.Y[ok], TrainOptions(epochs=200, batch=512, lr=1e-3, lr_final=1e-5, seed=2))
    nn = W.NearestWarmStart(fam).fit(P[ok], tr.X[ok], tr.Y[ok])
    return fam, opts, lw, nn, losses


def test_training_converges(trained):
    _, _, lw, _, losses = trained
    assert np.all(np.isfinite(losses)) and losses[-1] < 0.1 * losses[0]
    assert lw.basis.explained > 0.999


def test_learned_start_beats_cold_and_nearest(trained):
    fam, opts, lw, nn, _ = trained
    P = fam.sample(512, 200)
    cold, cc, _ = W.solve_warm(fam, P, None, opts)
    near, cn, _ = W.solve_warm(fam, P, nn, opts)
    learn, cl, redo = W.solve_warm(fam, P, lw, opts)
    print(f"mean iterations: cold {cold.iterations.mean():.0f}, nearest {near.iterations.mean():.0f}, "
          f"learned {learn.iterations.mean():.0f}; wall cold {cold.seconds:.2f}s learned {learn.seconds:.2f}s")
    assert cl["certified"].all()
    assert redo.mean() <= 0.01
    assert learn.iterations.mean() <= 0.6 * cold.iterations.mean()
    assert learn.iterations.mean() <= near.iterations.mean()
    # same optimum as the cold solves (objectives within the family gap)
    both = cc["certified"] & cl["certified"]
    assert np.all(np.abs(learn.objective[both] - cold.objective[both])
                  <= 1e-4 * (1 + np.abs(cold.objective[both])))


def test_nonfinite_prediction_falls_back_to_cold(trained):
    fam, opts, lw, _, _ = trained
    P = fam.sample(8, 300)

    class Broken:
        def predict(self, params):
            X, Y = lw.predict(params)
            X[0, 0] = np.nan
            bad = ~np.all(np.isfinite(np.hstack([X, Y])), axis=1)
            X[bad], Y[bad] = 0.0, 0.0  # what LearnedWarmStart.predict does
            return X, Y

    cold = W.solve_family(fam, P, opts)
    got, cert, _ = W.solve_warm(fam, P, Broken(), opts)
    assert got.iterations[0] == cold.iterations[0]  # member 0 ran exactly the cold start
    assert cert["certified"].all()


def test_launch_order_by_predicted_work_changes_no_answer():
    """Members handed to the multi-LP engine in decreasing predicted work come
    back in their own order with exactly the answers of the plain order (each
    block runs its member alone)."""
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    train = fam.sample(64, 3)
    tr = W.solve_family(fam, train, PdhgOptions(tolerance=1e-6, maxIterations=200000), engine="multi")
    est = W.WorkEstimate(fam).fit(train, tr.iterations)
    P = fam.sample(48, 4)
    work = est.predict(P)
    assert work.shape == (48,) and np.all(work > 0)
    opts = PdhgOptions(tolerance=1e-6, maxIterations=200000)
    plain = W.solve_family(fam, P, opts, engine="multi")
    ordered = W.solve_family(fam, P, opts, engine="multi", work=work)
    assert np.array_equal(plain.iterations, ordered.iterations)
    assert np.array_equal(plain.X, ordered.X) and np.array_equal(plain.Y, ordered.Y)


def test_warm_cap_and_single_engine_fallback(trained):
    """Warm attempts capped at one iteration fail certification, and those
    members re-solve cold: a fallback of at most 8 members on the single-LP
    engine, each answer exactly that member's cold single-LP solve; a larger
    one on the batched engine.  Every answer certified."""
    fam, opts, lw, _, _ = trained
    P = fam.sample(12, 400)
    got, cert, redo = W.solve_warm(fam, P[:6], lw, opts, engine="multi", warm_max_iterations=1, single_fallback=8,
                                   continue_failed=False)
    assert redo.sum() >= 3 and cert["certified"].all()
    single = W.solve_family(fam, P[:6][redo], opts, engine="single")
    assert np.array_equal(got.X[redo], single.X) and np.array_equal(got.Y[redo], single.Y)
    extra = got.iterations[redo] - single.iterations  # the warm attempt's work, counted too
    assert np.all((extra >= 1) & (extra <= 2))
    got12, cert12, redo12 = W.solve_warm(fam, P, lw, opts, engine="multi", warm_max_iterations=1,
                                         single_fallback=2, continue_failed=False)
    assert redo12.sum() > 2 and cert12["certified"].all()


def test_failed_members_continue_from_their_point(trained):
    """With continue_failed, members whose one-iteration warm attempt fails
    continue from that attempt's point and primal weight on the multi-LP
    engine; every answer certified, and the iterations count both attempts."""
    fam, opts, lw, _, _ = trained
    P = fam.sample(6, 500)
    got, cert, redo = W.solve_warm(fam, P, lw, opts, engine="multi", warm_max_iterations=1, continue_failed=True)
    assert redo.sum() >= 3 and cert["certified"].all()
    X0, Y0 = lw.predict(P)
    first = W.solve_family(fam, P, PdhgOptions(tolerance=opts.tolerance, maxIterations=1), starts=(X0, Y0),
                           engine="multi")
    more = W.solve_family(fam, P[redo], opts, starts=(first.X[redo], first.Y[redo]), engine="multi",
                          weights=first.weights[redo])
    assert np.array_equal(got.X[redo], more.X) and np.array_equal(got.iterations[redo], first.iterations[redo]
                                                                    + more.iterations)
