"""TEST INFRASTRUCTURE ONLY: CPU restatement of the warm-start network.

The reference has no learned model (its parametric layer,
src/parametric/parametric.cpp:483-530, warm-starts nothing), so this oracle
restates the network of include/b2p_mlp.h from its definition: a ReLU MLP,
layer l computing h_{l+1} = relu(h_l W_l^T + b_l) (no ReLU on the last
layer), loss (1 / B) * sum_b 0.5 * ||out_b - target_b||^2, parameters packed
per layer as W_l (out x in, row-major) then b_l.

``bf16_points=True`` rounds at exactly the points where the tensor-core path holds
BF16 values -- the weights, the network input, every hidden activation and
the back-propagated gradient fed to the GEMMs -- and does the rest in float64,
so the GPU differs from it only by FP32 accumulation order.  ``bf16_points=False`` is
the plain float64 network, pinned by central finite differences in the tests.
Only the tests may import this module.
"""
from __future__ import annotations

import numpy as np


def bf16(a) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def layout(widths):
    """[(w_offset, b_offset)] per layer and the parameter count."""
    offs, n = [], 0
    for a, b in zip(widths[:-1], widths[1:]):
        offs.append((n, n + a * b))
        n += a * b + b
    return offs, n


def unpack(params, widths):
    offs, _ = layout(widths)
    out = []
    for (wo, bo), a, b in zip(offs, widths[:-1], widths[1:]):
        out.append((params[wo:wo + a * b].reshape(b, a), params[bo:bo + b]))
    return out


def forward(params, widths, x, bf16_points: bool = True):
    """Returns (hidden inputs h_0 .. h_{L-1}, output) in float64."""
    layers = unpack(np.asarray(params, dtype=np.float32), widths)
    rnd = (lambda a: bf16(a).astype(np.float64)) if bf16_points else (lambda a: np.asarray(a, dtype=np.float64))
    h = rnd(x)
    hs = [h]
    for l, (W, b) in enumerate(layers):
        z = h @ rnd(W).T + np.asarray(b, dtype=np.float64)
        if l + 1 < len(layers):
            h = rnd(np.maximum(z, 0.0).astype(np.float32) if bf16_points else np.maximum(z, 0.0))
            hs.append(h)
        else:
            return hs, z
    raise ValueError("network has no layers")


def loss_grad(params, widths, x, target, bf16_points: bool = True):
    """(loss, packed gradient) on one batch."""
    params = np.asarray(params, dtype=np.float32)
    layers = unpack(params, widths)
    rnd = (lambda a: bf16(a).astype(np.float64)) if bf16_points else (lambda a: np.asarray(a, dtype=np.float64))
    hs, out = forward(params, widths, x, bf16_points)
    B = x.shape[0]
    if bf16_points:  # the device forms d and G in FP32
        d = (out.astype(np.float32) - np.asarray(target, dtype=np.float32)).astype(np.float32)
        gf = (d * np.float32(1.0 / B)).astype(np.float32).astype(np.float64)
        loss = 0.5 * float(np.sum(d.astype(np.float64) ** 2)) / B
    else:
        d = out - np.asarray(target, dtype=np.float64)
        gf = d / B
        loss = 0.5 * float(np.sum(d ** 2)) / B
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gb = rnd(gf.astype(np.float32)) if bf16_points else gf
        dW = gb.T @ hs[l]
        db = gf.sum(axis=0)
        grads.append((dW, db))
        if l > 0:
            g = gb @ rnd(W)
            g = np.where(hs[l] > 0, g, 0.0)
            gf = g.astype(np.float32).astype(np.float64) if bf16_points else g
    grads.reverse()
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return loss, flat

