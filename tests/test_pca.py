"""The warm start's PCA basis (randomized range finder) against the exact SVD
of the same standardised matrix: the same captured energy and the same
leading subspace, on a matrix with a clear spectral gap and on a wide one."""
import numpy as np
import pytest

from pramana_b200.warmstart import PcaBasis


@pytest.mark.parametrize("members,width,true_rank,rank", [(300, 2000, 20, 16), (120, 40000, 10, 32)])
def test_randomized_pca_matches_exact_svd(members, width, true_rank, rank):
    rng = np.random.default_rng(members)
    Z = rng.standard_normal((members, true_rank)) @ rng.standard_normal((true_rank, width)) * 10.0
    Z += 1e-3 * rng.standard_normal(Z.shape) + rng.uniform(-5, 5, size=width)
    b = PcaBasis().fit(Z, rank)
    S = (Z - Z.mean(0)) / Z.std(0)
    _, sv, vt = np.linalg.svd(S, full_matrices=False)
    r = min(rank, true_rank)
    exact = (sv[:rank] ** 2).sum() / (sv ** 2).sum()
    assert abs(b.explained - exact) <= 1e-9
    # the leading r directions span the same subspace (principal angles ~ 0)
    cos = np.linalg.svd(b.V[:, :r].T @ vt[:r].T, compute_uv=False)
    assert cos.min() >= 1 - 1e-8
    assert b.V.shape == (width, rank)
    # encode / decode round trip: as good as the exact basis, up to the
    # noise directions beyond the true rank (a flat spectrum there)
    rec = b.decode(b.encode(Z))
    exact_rec = Z.mean(0) + ((S @ vt[:rank].T) @ vt[:rank]) * Z.std(0)
    assert np.linalg.norm(rec - Z) <= np.linalg.norm(exact_rec - Z) * 1.01 + 1e-9


def test_neighbour_primal_weight_prediction():
    """WorkEstimate.predict_weight: the geometric mean of the 4 nearest
    training members' weights, skipping members without one (0 where none
    of the 4 has one)."""
    from pramana_b200.warmstart import RefineryFamily, WorkEstimate

    fam = RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    P = fam.sample(40, 3)
    rng = np.random.default_rng(1)
    w = np.exp(rng.normal(size=40))
    w[5] = 0.0
    w[6] = np.nan
    est = WorkEstimate(fam).fit(P, np.arange(40), w)
    Q = fam.sample(10, 4)
    got = est.predict_weight(Q)
    Z = fam.normalize(P).astype(np.float64)
    for q, g in zip(fam.normalize(Q).astype(np.float64), got):
        near = np.argsort(((Z - q) ** 2).sum(1))[:4]
        ok = [w[j] for j in near if np.isfinite(w[j]) and w[j] > 0]
        assert g == pytest.approx(np.exp(np.mean(np.log(ok))), rel=1e-12)
    none = WorkEstimate(fam).fit(P, np.arange(40), np.zeros(40))
    assert np.all(none.predict_weight(Q) == 0.0)
    with pytest.raises(ValueError):
        WorkEstimate(fam).fit(P, np.arange(40)).predict_weight(Q)
