"""Python face of the warm-start network (include/b2p_mlp.h).

``MlpNetwork`` owns a device-resident ReLU MLP whose forward, backward and
Adam steps run on the B200's tcgen05 tensor cores (BF16 operands, FP32
accumulation) through libb2p_pdhg.so.  There is no CPU path: without an
sm_100 device every call raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_lib.fptr)


def he_uniform(widths, seed: int) -> np.ndarray:
    """Packed initial parameters: W_l ~ U(-sqrt(6 / fan_in), +sqrt(6 / fan_in)), b_l = 0."""
    rng = np.random.default_rng(seed)
    parts = []
    for a, b in zip(widths[:-1], widths[1:]):
        lim = np.sqrt(6.0 / a)
        parts.append(rng.uniform(-lim, lim, size=a * b))
        parts.append(np.zeros(b))
    return np.concatenate(parts).astype(np.float32)


@dataclass
class TrainOptions:
    epochs: int = 200
    batch: int = 512
    lr: float = 1e-3
    lr_final: float = 1e-5
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    weight_decay: float = 0.0
    seed: int = 0

    def to_c(self) -> _lib.B2pMlpTrainOptions:
        return _lib.B2pMlpTrainOptions(self.epochs, self.batch, self.lr, self.lr_final, self.beta1, self.beta2,
                                       self.eps, self.weight_decay, self.seed)


class MlpNetwork:
    """widths = [in, hidden..., out] (multiples of 8)."""

    def __init__(self, widths, max_batch: int = 1024, device: int = -1, seed: int | None = 0):
        self.widths = [int(w) for w in widths]
        self.max_batch = int(max_batch)
        lib = _lib.load()
        w = np.asarray(self.widths, dtype=np.int32)
        h = C.c_void_p()
        _lib.check(lib.b2p_mlp_create(w.ctypes.data_as(_lib.iptr), len(self.widths) - 1, self.max_batch, device,
                                      C.byref(h)))
        self._h = h
        n = C.c_int64()
        _lib.check(lib.b2p_mlp_num_params(self._h, C.byref(n)))
        self.num_params = int(n.value)
        if seed is not None:
            self.set_params(he_uniform(self.widths, seed))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.check(_lib.load().b2p_mlp_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {p.size}")
        _lib.check(_lib.load().b2p_mlp_set_params(self._h, _fp(p)))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.num_params, dtype=np.float32)
        _lib.check(_lib.load().b2p_mlp_get_params(self._h, _fp(p)))
        return p

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.widths[0])
        y = np.empty((x.shape[0], self.widths[-1]), dtype=np.float32)
        _lib.check(_lib.load().b2p_mlp_forward(self._h, _fp(x), x.shape[0], _fp(y)))
        return y

    def loss_grad(self, x: np.ndarray, target: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.widths[0])
        t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1, self.widths[-1])
        g = np.empty(self.num_params, dtype=np.float32)
        loss = C.c_double()
        _lib.check(_lib.load().b2p_mlp_loss_grad(self._h, _fp(x), _fp(t), x.shape[0], C.byref(loss), _fp(g)))
        return loss.value, g

    def train(self, x: np.ndarray, target: np.ndarray, opts: TrainOptions | None = None) -> np.ndarray:
        """Adam on (x, target); returns the mean minibatch loss of every epoch."""
        opts = opts or TrainOptions()
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.widths[0])
        t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1, self.widths[-1])
        if x.shape[0] != t.shape[0]:
            raise ValueError("x and target differ in sample count")
        losses = np.zeros(max(opts.epochs, 1), dtype=np.float32)
        o = opts.to_c()
        _lib.check(_lib.load().b2p_mlp_train(self._h, _fp(x), _fp(t), x.shape[0], C.byref(o), _fp(losses)))
        return losses[:opts.epochs]


def gemm_bf16(a, b, *, alpha: float = 1.0, bias=None, relu: bool = False, mask=None, out_f32=None, out_bf16=None,
              a_strides=None, b_strides=None, m=None, n=None, k=None) -> None:
    """C = epilogue(alpha * A B) on device tensors (torch), through b2p_mlp_gemm_bf16.

    a, b: BF16 tensors; A(m, k) = a.flat[m * sam + k * sak] with (sam, sak) =
    a_strides (default: row-major m x k), likewise B(k, n) with b_strides
    (default row-major k x n).  Outputs are preallocated FP32 / BF16 tensors of
    row length n (their row stride is taken from the tensor)."""
    import torch

    m = int(m if m is not None else a.shape[0])
    k = int(k if k is not None else a.shape[1])
    n = int(n if n is not None else b.shape[1])
    sam, sak = a_strides if a_strides is not None else (a.stride(0), a.stride(1))
    sbk, sbn = b_strides if b_strides is not None else (b.stride(0), b.stride(1))
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.load().b2p_mlp_gemm_bf16(
        m, n, k, a.data_ptr(), sam, sak, b.data_ptr(), sbk, sbn, alpha,
        bias.data_ptr() if bias is not None else None, int(relu),
        mask.data_ptr() if mask is not None else None, mask.stride(0) if mask is not None else 0,
        out_f32.data_ptr() if out_f32 is not None else None, out_f32.stride(0) if out_f32 is not None else 0,
        out_bf16.data_ptr() if out_bf16 is not None else None, out_bf16.stride(0) if out_bf16 is not None else 0,
        stream))
