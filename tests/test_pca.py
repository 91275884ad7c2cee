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
