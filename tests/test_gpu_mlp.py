"""The warm-start network's tensor-core kernels on the B200.

* b2p_mlp_gemm_bf16 (tcgen05 MMA, FP32 accumulation in tensor memory) against
  torch's FP32 matmul of the same BF16 values, over ragged shapes,
  transposed operands and every epilogue;
* forward, loss and gradients of MlpNetwork against the CPU oracle
  (oracle/mlp_oracle.py) that rounds to BF16 at the same points, and against
  the plain float64 network;
* Adam training lowers the loss and is deterministic for a seed."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as MO
from pramana_b200 import _lib
from pramana_b200.mlp import MlpNetwork, TrainOptions, gemm_bf16, he_uniform

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _rand_bf16(shape, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.randn(shape, generator=g).to(torch.bfloat16).to(DEV)


# (2048, 2600, 200) and (2100, 2600, 96) give 176 and 187 tiles of 128 x 256,
# enough for every SM of a B200, so they run the wide-tile kernel (ragged N and K)
@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (200, 72, 40), (300, 136, 1000), (1, 8, 16), (513, 257, 200),
                                   (1024, 512, 512), (2048, 2600, 200)])
def test_gemm_matches_fp32_matmul(m, n, k):
    a = _rand_bf16((m, k), 1)
    b = _rand_bf16((k, n), 2)
    c = torch.empty((m, n), dtype=torch.float32, device=DEV)
    gemm_bf16(a, b, out_f32=c)
    torch.cuda.synchronize()
    want = a.float() @ b.float()
    scale = (a.float().abs() @ b.float().abs())
    assert torch.all((c - want).abs() <= 1e-5 * scale + 1e-30), (c - want).abs().max().item()


@pytest.mark.parametrize("m,n,k", [(260, 136, 96), (2100, 2600, 96)])
def test_gemm_transposed_operands_and_epilogue(m, n, k):
    at = _rand_bf16((k, m), 3)  # A stored k-major: A(m, k) = at[k, m]
    bt = _rand_bf16((n, k), 4)  # B stored n-major: B(k, n) = bt[n, k]
    bias = torch.randn(n, generator=torch.Generator().manual_seed(5)).float().to(DEV)
    mask = _rand_bf16((m, n), 6)
    cf = torch.empty((m, n), dtype=torch.float32, device=DEV)
    cb = torch.empty((m, n), dtype=torch.bfloat16, device=DEV)
    gemm_bf16(at, bt, alpha=0.5, bias=bias, relu=True, mask=mask, out_f32=cf, out_bf16=cb,
              a_strides=(1, m), b_strides=(1, k), m=m, n=n, k=k)
    torch.cuda.synchronize()
    want = torch.relu(0.5 * (at.float().t() @ bt.float().t()) + bias)
    want = torch.where(mask.float() > 0, want, torch.zeros_like(want))
    scale = 0.5 * (at.float().t().abs() @ bt.float().t().abs()) + bias.abs()
    assert torch.all((cf - want).abs() <= 1e-5 * scale + 1e-30)
    assert torch.equal(cb, cf.to(torch.bfloat16))
    assert (cf[mask.float() <= 0] == 0).all()


# A row-major and B stored n x k: both operands K-contiguous with 16-byte
# rows, so the kernel's TMA form runs (128-byte-swizzled tiles brought in by
# the tensor memory accelerator, zero-filled past ragged edges); the last
# shape gives enough 128 x 256 tiles for every SM (the wide-tile TMA form)
@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (200, 72, 40), (513, 257, 200), (1, 8, 16), (300, 136, 1000),
                                   (1024, 512, 512), (2048, 2600, 200)])
def test_gemm_tma_form_k_contiguous(m, n, k):
    a = _rand_bf16((m, k), 7)
    bt = _rand_bf16((n, k), 8)  # B(k, n) = bt[n, k]
    bias = torch.randn(n, generator=torch.Generator().manual_seed(9)).float().to(DEV)
    mask = _rand_bf16((m, n), 10)
    cf = torch.empty((m, n), dtype=torch.float32, device=DEV)
    cb = torch.empty((m, n), dtype=torch.bfloat16, device=DEV)
    gemm_bf16(a, bt, alpha=0.5, bias=bias, relu=True, mask=mask, out_f32=cf, out_bf16=cb, b_strides=(1, k), m=m, n=n,
              k=k)
    torch.cuda.synchronize()
    want = torch.relu(0.5 * (a.float() @ bt.float().t()) + bias)
    want = torch.where(mask.float() > 0, want, torch.zeros_like(want))
    scale = 0.5 * (a.float().abs() @ bt.float().t().abs()) + bias.abs()
    assert torch.all((cf - want).abs() <= 1e-5 * scale + 1e-30), (cf - want).abs().max().item()
    assert torch.equal(cb, cf.to(torch.bfloat16))


def test_gemm_rejects_bad_arguments():
    lib = _lib.load()
    assert lib.b2p_mlp_gemm_bf16(-1, 8, 8, None, 0, 0, None, 0, 0, 1.0, None, 0, None, 0, None, 0, None, 0,
                                 None) == 1
    assert lib.b2p_mlp_gemm_bf16(8, 8, 8, None, 0, 0, None, 0, 0, 1.0, None, 0, None, 0, None, 0, None, 0,
                                 None) == 1


WIDTHS = [16, 512, 512, 512, 128]


def _data(seed, rows):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, size=(rows, WIDTHS[0])).astype(np.float32)
    t = rng.standard_normal((rows, WIDTHS[-1])).astype(np.float32)
    return x, t


def test_forward_matches_oracle():
    net = MlpNetwork(WIDTHS, max_batch=256, seed=11)
    x, _ = _data(1, 700)  # three chunks of max_batch
    y = net.forward(x)
    _, want = MO.forward(net.get_params(), WIDTHS, x, bf16_points=True)
    err = np.abs(y - want).max()
    assert err <= 2e-3 * np.abs(want).max(), err
    _, w64 = MO.forward(net.get_params(), WIDTHS, x, bf16_points=False)
    assert np.linalg.norm(y - w64) <= 3e-2 * np.linalg.norm(w64)


@pytest.mark.parametrize("rows", [1, 100, 512])
def test_gradients_match_oracle(rows):
    net = MlpNetwork(WIDTHS, max_batch=512, seed=12)
    x, t = _data(2, rows)
    loss, g = net.loss_grad(x, t)
    p = net.get_params()
    lw, gw = MO.loss_grad(p, WIDTHS, x, t, bf16_points=True)
    assert abs(loss - lw) <= 1e-3 * lw
    offs, _ = MO.layout(WIDTHS)
    ends = [o[0] for o in offs[1:]] + [len(p)]
    for (wo, bo), end in zip(offs, ends):  # per weight and bias block
        for lo, hi in ((wo, bo), (bo, end)):
            d = np.linalg.norm(g[lo:hi] - gw[lo:hi])
            assert d <= 1e-2 * np.linalg.norm(gw[lo:hi]) + 1e-12, (lo, hi, d, np.linalg.norm(gw[lo:hi]))
    # against the float64 network: no further off than BF16 rounding itself
    # puts the oracle (about 10% of the norm at batch 1, 1-3% at 100+)
    l64, g64 = MO.loss_grad(p, WIDTHS, x, t, bf16_points=False)
    assert np.linalg.norm(g - g64) <= 1.2 * np.linalg.norm(gw - g64) + 1e-3 * np.linalg.norm(g64)


def test_training_lowers_loss_and_is_deterministic():
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, size=(4096, WIDTHS[0])).astype(np.float32)
    proj = rng.standard_normal((WIDTHS[0], WIDTHS[-1])).astype(np.float32)
    t = np.tanh(0.3 * (x @ proj)).astype(np.float32)  # a smooth target the network can fit
    opts = TrainOptions(epochs=30, batch=256, lr=1e-3, lr_final=1e-4, seed=9)
    runs = []
    for _ in range(2):
        net = MlpNetwork(WIDTHS, max_batch=1024, seed=13)
        losses = net.train(x, t, opts)
        runs.append((losses, net.get_params()))
    losses = runs[0][0]
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.2 * losses[0], losses
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    # the trained network generalises on fresh inputs
    xv = rng.uniform(-1, 1, size=(512, WIDTHS[0])).astype(np.float32)
    tv = np.tanh(0.3 * (xv @ proj))
    net = MlpNetwork(WIDTHS, max_batch=1024, seed=None)
    net.set_params(runs[0][1])
    err = 0.5 * np.sum((net.forward(xv) - tv) ** 2) / len(xv)
    assert err < 0.3 * 0.5 * np.sum(tv ** 2) / len(xv)


def test_bad_widths_rejected():
    with pytest.raises(_lib.B2pError):
        MlpNetwork([16, 20, 8])
