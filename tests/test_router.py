"""Router recalibration (pramana_b200/router.py): its features, phi and
decision rule against the reference's own computeFeatures and Router::decide
(oracle/_ref), a written model file loaded by the reference's Router::load,
and the ridge fit / held-out validation on synthetic timings."""
import math

import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200 import router as R
from pramana_b200 import warmstart as W
from pramana_b200.model import Model


def _lps():
    lps = [G.config1(1), G.random_lp(300, 600, 4.0, 180, 5), lp_cases.edge_lp(5)]
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    lps.append(fam.instance(fam.sample(1, 2)[0]))
    n = 4  # free columns and no rows
    lps.append(Model(num_rows=0, num_cols=n, start=np.zeros(n + 1), index=[], value=[], col_cost=[1, -1, 2, 0],
                     col_lower=[-np.inf, 0, -np.inf, 0], col_upper=[np.inf, 1, np.inf, 2], row_lower=[],
                     row_upper=[]))
    return lps


def test_features_match_reference(oracle_mod):
    if not oracle_mod.available("ref"):
        pytest.skip("oracle/_ref not built")
    for lp in _lps():
        ours = R.features(lp)
        ref = oracle_mod.router_features(lp)
        for k, v in ours.items():
            assert v == ref[k], (k, v, ref[k])


def _synthetic_weights(seed):
    rng = np.random.default_rng(seed)
    return {e: (rng.normal(0, 0.1, 8) + np.array([-2, 0.5, 0.3, 0, 0, 0, 0, 0])).tolist() for e in R.ENGINES}


@pytest.mark.parametrize("tol", [1e-6, 1e-8])
def test_written_model_loads_and_decides_like_reference(oracle_mod, tmp_path, tol):
    if not oracle_mod.available("ref"):
        pytest.skip("oracle/_ref not built")
    for seed in range(4):
        w = _synthetic_weights(seed)
        path = tmp_path / f"router_model_{seed}.json"
        R.write_model(path, w, instances=10)
        for lp in _lps():
            ref = oracle_mod.router_decide(lp, path, gpu=True, tolerance=tol)
            assert ref["loaded"]
            eng, pred = R.decide(w, R.features(lp), True, tol)
            assert eng == ref["engine"]
            for e, p in zip(R.ENGINES, ref["predicted"]):
                assert math.isclose(pred[e], p, rel_tol=1e-12)
    # without a model file the reference uses its priors, which DEFAULT_WEIGHTS restates
    for lp in _lps():
        ref = oracle_mod.router_decide(lp, None)
        eng, pred = R.decide(R.DEFAULT_WEIGHTS, R.features(lp))
        assert eng == ref["engine"] and all(math.isclose(pred[e], p, rel_tol=1e-12)
                                            for e, p in zip(R.ENGINES, ref["predicted"]))


def test_fit_recovers_weights_and_validation():
    rng = np.random.default_rng(3)
    truth = _synthetic_weights(7)
    recs = []
    for i in range(80):
        f = {"rows": float(rng.integers(100, 100000)), "cols": float(rng.integers(100, 200000)),
             "nnz": float(rng.integers(1000, 2000000)), "avg_row_nnz": float(rng.uniform(2, 40)),
             "max_row_nnz": float(rng.uniform(5, 500)), "coefficient_range": float(10 ** rng.uniform(0, 8)),
             "equality_row_fraction": float(rng.uniform()), "free_column_fraction": float(rng.uniform(0, 0.3))}
        t = {e: math.exp(sum(w * x for w, x in zip(truth[e], R.phi(f)))) for e in R.ENGINES}
        recs.append(R.Record(name=f"lp{i}", family=f"fam{i % 3}", features=f, times=t, limit=1e9))
    w = R.fit(recs, lam=1e-6)
    for e in R.ENGINES:  # log(t + 1e-3) ~ log t for these times: near-exact recovery
        assert np.allclose(w[e], truth[e], atol=0.05), e
    v = R.validate(recs)
    assert v["instances"] == 80
    assert v["router_held_out"]["geo_mean_regret"] < 1.05
    assert v["router_held_out"]["geo_mean_regret"] <= min(v[f"always_{e}"]["geo_mean_regret"] for e in R.ENGINES)
    fold = R.folds(recs)
    for fam in ("fam0", "fam1", "fam2"):  # every fold holds out part of every family
        assert {fold[r.name] for r in recs if r.family == fam} == set(range(5))


def test_censored_times():
    r = R.Record(name="a", family="f", features={}, times={"dual": None, "ipm": 2.0}, limit=3.0)
    assert r.time("dual") == 12.0 and r.time("ipm") == 2.0


def test_committed_b200_model_loads_in_reference_router(oracle_mod):
    """The router_model_b200.json fitted from B200 timings is read by the
    reference's Router::load, and its decisions on the calibration LPs are
    the ones router.decide takes with the same weights."""
    if not oracle_mod.available("ref"):
        pytest.skip("oracle/_ref not built")
    import os

    import bench
    path = os.path.join(os.path.dirname(R.__file__), "router_model_b200.json")
    w = R.load_model(path)
    for fam, name, lp in bench.router_instances()[::3]:
        ref = oracle_mod.router_decide(lp, path, gpu=True, tolerance=1e-6)
        assert ref["loaded"]
        eng, pred = R.decide(w, R.features(lp), True, 1e-6)
        assert eng == ref["engine"], name
        for e, p in zip(R.ENGINES, ref["predicted"]):
            assert math.isclose(pred[e], p, rel_tol=1e-12)
