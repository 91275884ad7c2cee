"""CPU pins of the warm-start network's oracle (oracle/mlp_oracle.py): its
float64 backward pass against central finite differences, its BF16 rounding
against torch's float32 -> bfloat16 conversion, and the BF16-rounded network
against the float64 one.  No GPU."""
import numpy as np
import torch

from oracle import mlp_oracle as MO
from pramana_b200.mlp import he_uniform

WIDTHS = [16, 24, 24, 8]


def _batch(seed, rows=12):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((rows, WIDTHS[0])).astype(np.float32), \
        rng.standard_normal((rows, WIDTHS[-1])).astype(np.float32)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    a = np.concatenate([rng.standard_normal(10000).astype(np.float32) * 10.0 ** rng.integers(-30, 30, 10000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.4e38, 1e-40], dtype=np.float32)])
    want = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    got = MO.bf16(a)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_float64_gradient_matches_finite_differences():
    x, t = _batch(1)
    p = he_uniform(WIDTHS, 3).astype(np.float64)
    p[MO.layout(WIDTHS)[0][0][1]:MO.layout(WIDTHS)[0][0][1] + WIDTHS[1]] = 0.05  # nonzero first bias

    def loss_at(q):
        # float64 evaluation (the oracle casts params to float32 first, so do the
        # float64 network here from the same packing)
        layers, h = [], x.astype(np.float64)
        offs, _ = MO.layout(WIDTHS)
        for (wo, bo), a, b in zip(offs, WIDTHS[:-1], WIDTHS[1:]):
            layers.append((q[wo:wo + a * b].reshape(b, a), q[bo:bo + b]))
        for l, (W, b) in enumerate(layers):
            z = h @ W.T + b
            h = np.maximum(z, 0.0) if l + 1 < len(layers) else z
        return 0.5 * np.sum((h - t) ** 2) / x.shape[0]

    p32 = p.astype(np.float32).astype(np.float64)
    loss, g = MO.loss_grad(p32.astype(np.float32), WIDTHS, x, t, bf16_points=False)
    assert abs(loss - loss_at(p32)) <= 1e-12 * max(1.0, abs(loss))
    rng = np.random.default_rng(7)
    idx = rng.choice(len(p32), size=60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p32)
        e[i] = h
        fd = (loss_at(p32 + e) - loss_at(p32 - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_network_close_to_float64():
    x, t = _batch(2, rows=64)
    p = he_uniform(WIDTHS, 4)
    l64, g64 = MO.loss_grad(p, WIDTHS, x, t, bf16_points=False)
    l16, g16 = MO.loss_grad(p, WIDTHS, x, t, bf16_points=True)
    assert abs(l16 - l64) <= 2e-2 * l64
    assert np.linalg.norm(g16 - g64) <= 3e-2 * np.linalg.norm(g64)
