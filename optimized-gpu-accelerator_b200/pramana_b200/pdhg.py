"""Python mirror of PRAMANA's PDHG engine interface (src/pdhg/pdhg.h:32-80),
backed by the sm_100a engine through the C ABI of include/b2p_pdhg.h.

Names follow the reference so that code and tests read alike::

    po = PdhgOptions(); po.tolerance = 1e-7
    r = solvePdhg(model, po)            # pramana::solvePdhg
    rb = solvePdhgBatch(model, cases, po)
    gpuAvailable(); gpuInfoJson()

Every solve runs on the GPU.  There is no CPU backend behind this module:
``useGpu=False`` is rejected and a machine without a usable sm_100 device
raises ``B2pError`` (code 3).
"""
from __future__ import annotations

import ctypes as C
import json
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .model import LpCase, Model

Status = _lib.STATUS_NAMES


@dataclass
class PdhgOptions:
    """pramana::PdhgOptions (src/pdhg/pdhg.h:32-42) + deadline and device."""
    tolerance: float = 1e-6
    maxIterations: int = 1000000
    checkEvery: int = 64
    useGpu: bool = True
    ruizIterations: int = 10
    pockChambolle: bool = True
    rescaleObjectiveAndBounds: bool = True
    reflection: float = 1.0
    logInterval: int = 0
    timeLimit: float = 0.0        # seconds (pramana::Deadline); <= 0 = none
    device: int = -1
    useGraphs: bool = True
    precision: int = _lib.PRECISION_FP64
    lanesPerRowA: int = 0        # SpMV schedule overrides (0 = automatic)
    lanesPerRowAT: int = 0
    shortRowRounds: int = 0
    kernelMode: int = _lib.KERNELS_AUTO   # KERNELS_FUSED / KERNELS_RESIDENT to force a form
    spmvSchedule: int = _lib.SCHEDULE_AUTO  # multi-LP SpMV schedule (SCHEDULE_BINNED / _TILED / _TUNED)
    multiForm: int = _lib.MULTI_AUTO  # multi-LP engine form (MULTI_GRID / MULTI_CTA)
    ctaSmemLimit: int = 0  # CTA form: shared-memory bytes one LP may use (0 = device maximum)
    ctaThreads: int = 0  # CTA form: threads per block (128 / 256 / 512 / 1024; 0 = autotuned)
    ctaKernel: int = _lib.CTA_AUTO  # CTA form: CTA_GENERAL / CTA_OWNER1 / CTA_OWNER2 (0 = autotuned)
    batchVariant: int = 0  # FP64 batches: 0 = tuned; 1..4 = (cases per thread, streamed) (1,no) (2,no) (1,yes) (2,yes)
    batchNoCompaction: bool = False  # batches: keep finished cases in the interleave (no packing)
    ctaLayout: int = 0  # CTA form: 0 = sliced-ELL operators where read from global memory, 1 = CSR

    def to_c(self, cancel_flag=None) -> _lib.B2pOptions:
        if not self.useGpu:
            raise ValueError("this PDHG engine has no CPU backend (useGpu=False)")
        o = _lib.B2pOptions()
        _lib.load().b2p_default_options(C.byref(o))
        o.tolerance = float(self.tolerance)
        o.max_iterations = int(self.maxIterations)
        o.check_every = int(self.checkEvery)
        o.ruiz_iterations = int(self.ruizIterations)
        o.pock_chambolle = int(bool(self.pockChambolle))
        o.rescale_objective_and_bounds = int(bool(self.rescaleObjectiveAndBounds))
        o.reflection = float(self.reflection)
        o.log_interval = int(self.logInterval)
        o.device = int(self.device)
        o.time_limit = float(self.timeLimit)
        o.precision = int(self.precision)
        o.use_graphs = int(bool(self.useGraphs))
        o.lanes_per_row_a = int(self.lanesPerRowA)
        o.lanes_per_row_at = int(self.lanesPerRowAT)
        o.short_row_rounds = int(self.shortRowRounds)
        o.kernel_mode = int(self.kernelMode)
        o.spmv_schedule = int(self.spmvSchedule)
        o.multi_form = int(self.multiForm)
        o.cta_smem_limit = int(self.ctaSmemLimit)
        o.cta_threads = int(self.ctaThreads)
        o.cta_kernel = int(self.ctaKernel)
        o.batch_variant = int(self.batchVariant)
        o.batch_no_compaction = int(bool(self.batchNoCompaction))
        o.cta_layout = int(self.ctaLayout)
        if cancel_flag is not None:
            o.cancel_flag = C.cast(cancel_flag, C.POINTER(C.c_int32))
        return o


@dataclass
class PdhgStats:
    """pramana::PdhgStats (src/pdhg/pdhg.h:44-56)."""
    iterations: int = 0
    restarts: int = 0
    primalResidual: float = 0.0
    dualResidual: float = 0.0
    gap: float = 0.0
    primalWeight: float = 1.0
    setupSeconds: float = 0.0
    solveSeconds: float = 0.0
    kernelSeconds: float = 0.0
    transferSeconds: float = 0.0
    bytesUploaded: int = 0
    bytesDownloaded: int = 0
    kernelLaunches: int = 0
    spectralNorm: float = 0.0
    backend: str = "gpu"
    device: str = ""
    fp32Iterations: int = 0  # mixed form: iterations run in FP32 (no counterpart in the reference)

    @classmethod
    def from_c(cls, s: _lib.B2pStats, device: str = "") -> "PdhgStats":
        return cls(iterations=s.iterations, restarts=s.restarts, primalResidual=s.primal_residual,
                   dualResidual=s.dual_residual, gap=s.gap, primalWeight=s.primal_weight,
                   setupSeconds=s.setup_seconds, solveSeconds=s.solve_seconds, kernelSeconds=s.kernel_seconds,
                   transferSeconds=s.transfer_seconds, bytesUploaded=s.bytes_uploaded,
                   bytesDownloaded=s.bytes_downloaded, kernelLaunches=s.kernel_launches,
                   spectralNorm=s.spectral_norm, device=device, fp32Iterations=s.fp32_iterations)

    def toJson(self) -> dict:
        """Keys of PdhgStats::toJson (src/pdhg/pdhg.cpp:691-710)."""
        return {"backend": self.backend, "device": self.device, "iterations": self.iterations,
                "restarts": self.restarts, "relative_primal_residual": self.primalResidual,
                "relative_dual_residual": self.dualResidual, "relative_gap": self.gap,
                "primal_weight": self.primalWeight, "spectral_norm_estimate": self.spectralNorm,
                "setup_seconds": self.setupSeconds, "solve_seconds": self.solveSeconds,
                "kernel_seconds": self.kernelSeconds, "transfer_seconds": self.transferSeconds,
                "bytes_uploaded": self.bytesUploaded, "bytes_downloaded": self.bytesDownloaded,
                "kernel_launches": self.kernelLaunches}


@dataclass
class PdhgResult:
    """pramana::PdhgResult (src/pdhg/pdhg.h:58-65)."""
    status: str
    objective: float
    dualObjective: float
    x: np.ndarray
    rowDual: np.ndarray
    iterations: int
    relativeKkt: float
    stats: PdhgStats = field(default_factory=PdhgStats)
    # solvePdhgMulti: this LP's primal weight at termination in original-space
    # units (scaled weight x gamma / beta); no counterpart in the reference
    primalWeight: float = 0.0


def _lp_struct(lp: Model):
    keep = []

    def p(a, ctype):
        # a no-op for the arrays Model already holds; a copy if a field was
        # replaced by one of another dtype after construction
        a = np.ascontiguousarray(a, dtype=np.int32 if ctype is C.c_int32 else np.float64)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(ctype))

    s = _lib.B2pLp(num_rows=lp.num_rows, num_cols=lp.num_cols, start=p(lp.start, C.c_int32),
                   index=p(lp.index, C.c_int32), value=p(lp.value, C.c_double), col_cost=p(lp.col_cost, C.c_double),
                   col_lower=p(lp.col_lower, C.c_double), col_upper=p(lp.col_upper, C.c_double),
                   row_lower=p(lp.row_lower, C.c_double), row_upper=p(lp.row_upper, C.c_double),
                   obj_offset=float(lp.obj_offset))
    return s, keep


def _cases_struct(cases, n, m):
    keep = []
    arr = (_lib.B2pCase * len(cases))()

    def p(v, ln):
        if v is None:
            return None
        v = np.ascontiguousarray(v, dtype=np.float64)
        if len(v) != ln:
            raise ValueError("case vector has the wrong length")
        keep.append(v)
        return v.ctypes.data_as(_lib.dptr)

    for b, cs in enumerate(cases):
        arr[b] = _lib.B2pCase(cost=p(cs.cost, n), col_lower=p(cs.col_lower, n), col_upper=p(cs.col_upper, n),
                              row_lower=p(cs.row_lower, m), row_upper=p(cs.row_upper, m))
    return arr, keep


_DEVICE_NAME: list[str] = []


def _device_name() -> str:
    """The GPU's name for PdhgStats.device, queried once per process (the
    query reads every device property, which is not free on a solve path)."""
    if not _DEVICE_NAME:
        try:
            _DEVICE_NAME.append(gpuInfoJson().get("name", ""))
        except Exception:  # noqa: BLE001 - informational only
            return ""
    return _DEVICE_NAME[0]


def _results(lp: Model, res, x, y, k, stats) -> list[PdhgResult]:
    n, m = lp.num_cols, lp.num_rows
    return [PdhgResult(status=Status.get(res[b].status, str(res[b].status)), objective=res[b].objective,
                       dualObjective=res[b].dual_objective, x=x[b * n:(b + 1) * n].copy(),
                       rowDual=y[b * m:(b + 1) * m].copy(), iterations=res[b].iterations,
                       relativeKkt=res[b].relative_kkt, stats=stats) for b in range(k)]


def solvePdhg(lp: Model, opts: PdhgOptions | None = None, cancel_flag=None) -> PdhgResult:
    """pramana::solvePdhg (src/pdhg/pdhg.cpp:712-717); ``lp`` must be a minimisation LP."""
    opts = opts or PdhgOptions()
    lib = _lib.load()
    s, keep = _lp_struct(lp)
    o = opts.to_c(cancel_flag)
    x = np.zeros(lp.num_cols)
    y = np.zeros(lp.num_rows)
    res = (_lib.B2pResult * 1)()
    st = _lib.B2pStats()
    _lib.check(lib.b2p_solve_pdhg(C.byref(s), C.byref(o), x.ctypes.data_as(_lib.dptr), y.ctypes.data_as(_lib.dptr),
                                  res, C.byref(st)))
    del keep
    return _results(lp, res, x, y, 1, PdhgStats.from_c(st, _device_name()))[0]


def solvePdhgBatch(base: Model, cases: list[LpCase], opts: PdhgOptions | None = None,
                   batchStats: PdhgStats | None = None) -> list[PdhgResult]:
    """pramana::solvePdhgBatch (src/pdhg/pdhg.cpp:719-728): cases share A."""
    if not cases:
        return []
    opts = opts or PdhgOptions()
    lib = _lib.load()
    s, keep = _lp_struct(base)
    arr, keep2 = _cases_struct(cases, base.num_cols, base.num_rows)
    o = opts.to_c()
    k = len(cases)
    x = np.zeros(k * base.num_cols)
    y = np.zeros(k * base.num_rows)
    res = (_lib.B2pResult * k)()
    st = _lib.B2pStats()
    _lib.check(lib.b2p_solve_pdhg_batch(C.byref(s), arr, k, C.byref(o), x.ctypes.data_as(_lib.dptr),
                                        y.ctypes.data_as(_lib.dptr), res, C.byref(st)))
    del keep, keep2
    stats = PdhgStats.from_c(st, _device_name())
    if batchStats is not None:
        batchStats.__dict__.update(stats.__dict__)
    return _results(base, res, x, y, k, stats)


def solvePdhgMulti(lps: list[Model], opts: PdhgOptions | None = None, batchStats: PdhgStats | None = None,
                   starts: list | None = None, cancel_flag=None, primalWeights=None) -> list[PdhgResult]:
    """Independent LPs of different sizes solved together on the GPU, each with
    the reference's algorithm (no counterpart in the reference).  starts[b] =
    (x, y) warm-starts LP b (None entries: cold start); primalWeights[b]
    (original-space units, as the results' primalWeight; entries that are not
    finite and positive keep the default) sets LP b's initial primal weight;
    cancel_flag: a ctypes int32 array whose element 0 stops the solve when
    set."""
    if not lps:
        return []
    opts = opts or PdhgOptions()
    lib = _lib.load()
    k = len(lps)
    structs, keep = [], []
    arr = (_lib.B2pLp * k)()
    for b, lp in enumerate(lps):
        s, kp = _lp_struct(lp)
        arr[b] = s
        keep.append(kp)
    xs = [np.zeros(lp.num_cols) for lp in lps]
    ys = [np.zeros(lp.num_rows) for lp in lps]
    xp = (_lib.dptr * k)(*[a.ctypes.data_as(_lib.dptr) for a in xs])
    yp = (_lib.dptr * k)(*[a.ctypes.data_as(_lib.dptr) for a in ys])
    res = (_lib.B2pResult * k)()
    st = _lib.B2pStats()
    o = opts.to_c(cancel_flag)
    xst = yst = None
    if starts is not None:
        sx = [None if s is None or s[0] is None else np.ascontiguousarray(s[0], dtype=np.float64) for s in starts]
        sy = [None if s is None or s[1] is None else np.ascontiguousarray(s[1], dtype=np.float64) for s in starts]
        keep.append((sx, sy))
        xst = (_lib.dptr * k)(*[a.ctypes.data_as(_lib.dptr) if a is not None else None for a in sx])
        yst = (_lib.dptr * k)(*[a.ctypes.data_as(_lib.dptr) if a is not None else None for a in sy])
    w_in = None
    if primalWeights is not None:
        w_in = np.ascontiguousarray(np.asarray(primalWeights, dtype=np.float64).reshape(k))
        keep.append(w_in)
    w_out = np.zeros(k)
    _lib.check(lib.b2p_solve_pdhg_multi_warm(arr, k, C.byref(o), xst, yst,
                                              None if w_in is None else w_in.ctypes.data_as(_lib.dptr), xp, yp,
                                              w_out.ctypes.data_as(_lib.dptr), res, C.byref(st)))
    del keep, structs
    stats = PdhgStats.from_c(st, _device_name())
    if batchStats is not None:
        batchStats.__dict__.update(stats.__dict__)
    solvePdhgMulti.last_stats = st
    return [PdhgResult(status=Status.get(res[b].status, str(res[b].status)), objective=res[b].objective,
                       dualObjective=res[b].dual_objective, x=xs[b], rowDual=ys[b], iterations=res[b].iterations,
                       relativeKkt=res[b].relative_kkt, stats=stats, primalWeight=float(w_out[b]))
            for b in range(k)]


def gpuAvailable() -> bool:
    """pramana::gpuAvailable (src/pdhg/pdhg.cpp:730)."""
    return bool(_lib.load().b2p_gpu_available())


def gpuInfoJson() -> dict:
    """pramana::gpuInfoJson (src/pdhg/pdhg.cpp:732-746)."""
    lib = _lib.load()
    need = lib.b2p_gpu_info_json(None, 0)
    buf = C.create_string_buffer(need + 1)
    lib.b2p_gpu_info_json(buf, need + 1)
    return json.loads(buf.value.decode())


class Engine:
    """Two-phase solve: ``Engine(lp)`` prepares and uploads (inputs resident in
    HBM afterwards), ``solve()`` runs the PDHG loop from the initial point and
    can be repeated, ``fetch()`` returns the last solution."""

    def __init__(self, lp: Model, opts: PdhgOptions | None = None, cases: list[LpCase] | None = None):
        self.lp = lp
        self.opts = opts or PdhgOptions()
        self.k = len(cases) if cases else 1
        self._lib = _lib.load()
        s, keep = _lp_struct(lp)
        arr, keep2 = (_cases_struct(cases, lp.num_cols, lp.num_rows) if cases else (None, []))
        o = self.opts.to_c()
        h = C.c_void_p()
        t0 = time.perf_counter()
        _lib.check(self._lib.b2p_engine_create(C.byref(s), arr, len(cases) if cases else 0, C.byref(o), C.byref(h)))
        self.create_seconds = time.perf_counter() - t0
        del keep, keep2
        self._h = h
        self.last_stats: _lib.B2pStats | None = None

    def solve(self) -> list[PdhgResult]:
        res = (_lib.B2pResult * self.k)()
        st = _lib.B2pStats()
        _lib.check(self._lib.b2p_engine_solve(self._h, res, C.byref(st)))
        self.last_stats = st
        x, y = self.fetch()
        return _results(self.lp, res, x, y, self.k, PdhgStats.from_c(st))

    def set_start(self, x=None, y=None, primal_weight: float = 0.0) -> None:
        """Warm start of the following solves (original space); None, None = cold start."""
        xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        ya = None if y is None else np.ascontiguousarray(y, dtype=np.float64)
        _lib.check(self._lib.b2p_engine_set_start(self._h, None if xa is None else xa.ctypes.data_as(_lib.dptr),
                                                  None if ya is None else ya.ctypes.data_as(_lib.dptr),
                                                  float(primal_weight)))

    def fetch(self):
        x = np.zeros(self.k * self.lp.num_cols)
        y = np.zeros(self.k * self.lp.num_rows)
        _lib.check(self._lib.b2p_engine_fetch(self._h, x.ctypes.data_as(_lib.dptr), y.ctypes.data_as(_lib.dptr)))
        return x, y

    def set_profiling(self, on: bool) -> None:
        _lib.check(self._lib.b2p_engine_set_profiling(self._h, int(on)))

    def kernel_times(self, cls: int):
        n = C.c_int64()
        ms = C.c_double()
        _lib.check(self._lib.b2p_engine_kernel_times(self._h, cls, C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def kernel_bytes(self, cls: int) -> float:
        b = C.c_double()
        _lib.check(self._lib.b2p_engine_kernel_bytes(self._h, cls, C.byref(b)))
        return b.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.b2p_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def csr_spmv(ptr, idx, val, x, rows: int, cols: int, k: int = 1) -> np.ndarray:
    """Device CSR SpMV with k interleaved right-hand sides (CpuBackend::mult order)."""
    lib = _lib.load()
    ptr = np.ascontiguousarray(ptr, dtype=np.int32)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(rows * k)
    _lib.check(lib.b2p_csr_spmv(rows, cols, k, ptr.ctypes.data_as(_lib.iptr), idx.ctypes.data_as(_lib.iptr),
                                val.ctypes.data_as(_lib.dptr), x.ctypes.data_as(_lib.dptr),
                                y.ctypes.data_as(_lib.dptr)))
    return y


def kktResidual(lp: Model, x, rowDual, cases: list[LpCase] | None = None) -> np.ndarray:
    """Relative KKT error (relP, relD, gap, max) of points (x, rowDual) in the
    original space, evaluated on the GPU; one row per case."""
    lib = _lib.load()
    s, keep = _lp_struct(lp)
    k = len(cases) if cases else 1
    arr, keep2 = (_cases_struct(cases, lp.num_cols, lp.num_rows) if cases else (None, []))
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    y = np.ascontiguousarray(rowDual, dtype=np.float64).reshape(-1)
    if len(x) != k * lp.num_cols or len(y) != k * lp.num_rows:
        raise ValueError("x / rowDual have the wrong length")
    out = np.zeros(4 * k)
    _lib.check(lib.b2p_kkt_residual(C.byref(s), arr, len(cases) if cases else 0, x.ctypes.data_as(_lib.dptr),
                                    y.ctypes.data_as(_lib.dptr), out.ctypes.data_as(_lib.dptr)))
    del keep, keep2
    return out.reshape(k, 4)


def safeDualBound(lp: Model, rowDual, cases: list[LpCase] | None = None) -> list[dict]:
    """Outward-rounded Neumaier-Shcherbina lower bound (objective offset
    excluded), valid for any row dual, per case; bit-identical to the
    reference's safeDualBound."""
    lib = _lib.load()
    s, keep = _lp_struct(lp)
    k = len(cases) if cases else 1
    arr, keep2 = (_cases_struct(cases, lp.num_cols, lp.num_rows) if cases else (None, []))
    y = np.ascontiguousarray(rowDual, dtype=np.float64).reshape(-1)
    if len(y) != k * lp.num_rows:
        raise ValueError("rowDual has the wrong length")
    out = (_lib.B2pSafeBound * k)()
    _lib.check(lib.b2p_safe_dual_bound(C.byref(s), arr, len(cases) if cases else 0, y.ctypes.data_as(_lib.dptr), out))
    del keep, keep2
    return [{f: getattr(out[b], f) for f, _ in _lib.B2pSafeBound._fields_ if f != "pad0"} for b in range(k)]


def impliedBounds(lp: Model, cases: list[LpCase] | None = None):
    """Constraint-implied column bounds per case (the certifier's fallback,
    src/cert/certifier.cpp:340-356), computed on host threads; returns
    (lower, upper), each num_cases x num_cols."""
    lib = _lib.load()
    s, keep = _lp_struct(lp)
    k = len(cases) if cases else 1
    arr, keep2 = (_cases_struct(cases, lp.num_cols, lp.num_rows) if cases else (None, []))
    lo = np.zeros((k, lp.num_cols))
    up = np.zeros((k, lp.num_cols))
    _lib.check(lib.b2p_implied_bounds(C.byref(s), arr, len(cases) if cases else 0, lo.ctypes.data_as(_lib.dptr),
                                      up.ctypes.data_as(_lib.dptr)))
    del keep, keep2
    return lo, up


def certifyLp(lp: Model, x, rowDual, cases: list[LpCase] | None = None, primalFeas: float = 1e-6,
              dualFeas: float = 1e-6, relGap: float = 1e-6) -> list[dict]:
    """pramana::certify of OPTIMAL claims (x, rowDual) per case, bit-identical
    to the reference's Certificate; the safe bounds run on the GPU."""
    lib = _lib.load()
    s, keep = _lp_struct(lp)
    k = len(cases) if cases else 1
    arr, keep2 = (_cases_struct(cases, lp.num_cols, lp.num_rows) if cases else (None, []))
    xa = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    ya = np.ascontiguousarray(rowDual, dtype=np.float64).reshape(-1)
    if len(xa) != k * lp.num_cols or len(ya) != k * lp.num_rows:
        raise ValueError("x / rowDual have the wrong length")
    tol = _lib.B2pCertTolerances(primalFeas, dualFeas, relGap)
    out = (_lib.B2pCertificate * k)()
    _lib.check(lib.b2p_certify_lp(C.byref(s), arr, len(cases) if cases else 0, xa.ctypes.data_as(_lib.dptr),
                                  ya.ctypes.data_as(_lib.dptr), C.byref(tol), out))
    del keep, keep2
    return [{f: getattr(out[b], f) for f, _ in _lib.B2pCertificate._fields_} for b in range(k)]


# snake_case aliases
solve_pdhg = solvePdhg
solve_pdhg_batch = solvePdhgBatch
gpu_available = gpuAvailable
gpu_info_json = gpuInfoJson
kkt_residual = kktResidual
safe_dual_bound = safeDualBound
implied_bounds = impliedBounds
certify_lp = certifyLp
solve_pdhg_multi = solvePdhgMulti
