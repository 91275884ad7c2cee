"""TEST INFRASTRUCTURE ONLY: ctypes front end of the two CPU checkers.

* ``lib="oracle"`` -> oracle/liboracle_pdhg.so, this project's single-threaded
  C restatement of the reference PDHG (pdhg_oracle.c);
* ``lib="ref"``    -> oracle/_ref/libpramana_ref.so, the reference's own CPU
  PDHG (src/pdhg/pdhg.cpp CpuBackend) compiled from its sources.

Both export the same ``*_pdhg_solve`` signature, so every parity test can run
against either.  Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle_pdhg.so")
REF_SO = os.path.join(HERE, "_ref", "libpramana_ref.so")
# The reference tree, present only where the checkers are built (never on the
# GPU box): PRAMANA_REFERENCE names it, else the build container's copy.
REFERENCE_SRC = os.environ.get("PRAMANA_REFERENCE", "/root/reference")

STATUS_NAMES = {0: "NotSolved", 1: "Optimal", 5: "TimeLimit", 6: "IterationLimit"}


class Options(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_int64), ("check_every", C.c_int32),
                ("ruiz_iterations", C.c_int32), ("pock_chambolle", C.c_int32), ("rescale", C.c_int32),
                ("reflection", C.c_double), ("time_limit", C.c_double), ("primal_weight_start", C.c_double)]


class CaseResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("pad", C.c_int32), ("iterations", C.c_int64), ("objective", C.c_double),
                ("dual_objective", C.c_double), ("relative_kkt", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("restarts", C.c_int32), ("threads", C.c_int32),
                ("primal_weight", C.c_double), ("spectral_norm", C.c_double), ("setup_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("gap", C.c_double)]


@dataclass
class OracleResult:
    status: int
    iterations: int
    objective: float
    dual_objective: float
    relative_kkt: float
    x: np.ndarray
    y: np.ndarray


def build(reference: bool = True) -> None:
    """Compile the C restatement (and, when the reference tree is present, the reference)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if reference and os.path.isdir(REFERENCE_SRC):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={REFERENCE_SRC}"], check=True)


_libs: dict = {}


def _load(lib: str):
    if lib in _libs:
        return _libs[lib]
    path = ORACLE_SO if lib == "oracle" else REF_SO
    if not os.path.exists(path):
        build(reference=(lib == "ref"))
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    h = C.CDLL(path)
    fn = getattr(h, "oracle_pdhg_solve" if lib == "oracle" else "ref_pdhg_solve")
    fn.restype = C.c_int
    _libs[lib] = h
    if lib == "ref":
        h.ref_set_threads.argtypes = [C.c_int]
        h.ref_threads.restype = C.c_int
    return h


def available(lib: str) -> bool:
    try:
        _load(lib)
        return True
    except (FileNotFoundError, OSError, subprocess.CalledProcessError):
        return False


def set_ref_threads(n: int) -> int:
    """Size the reference ThreadPool; only effective before its first solve."""
    h = _load("ref")
    h.ref_set_threads(int(n))
    return h.ref_threads()


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def default_options(**kw) -> Options:
    o = Options(tolerance=1e-6, max_iterations=1000000, check_every=64, ruiz_iterations=10, pock_chambolle=1,
                rescale=1, reflection=1.0, time_limit=0.0, primal_weight_start=0.0)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def solve(lp, lib: str = "oracle", cases=None, backend: str = "cpu", **opts) -> list[OracleResult] | OracleResult:
    """Run solvePdhg (cases is None) or solvePdhgBatch (list of LpCase-like
    objects).  backend="gpu" (ref build only) runs the reference's own GPU
    backend; last_stats["backend"] says which backend the reference used."""
    h = _load(lib)
    fn = h.oracle_pdhg_solve if lib == "oracle" else (h.ref_pdhg_solve_gpu if backend == "gpu" else h.ref_pdhg_solve)
    m, n = lp.num_rows, lp.num_cols
    o = default_options(**opts)
    k = 0 if cases is None else len(cases)
    kk = max(k, 1)
    keep = []

    def arr(field, ln):
        if cases is None:
            return None
        p = (C.POINTER(C.c_double) * k)()
        for b, cs in enumerate(cases):
            v = getattr(cs, field)
            if v is None:
                p[b] = None
            else:
                v = np.ascontiguousarray(v, dtype=np.float64)
                assert len(v) == ln
                keep.append(v)
                p[b] = _dp(v)
        return p

    cc, cl, cu, rl, ru = arr("cost", n), arr("col_lower", n), arr("col_upper", n), arr("row_lower", m), \
        arr("row_upper", m)
    x = np.zeros(kk * n)
    y = np.zeros(kk * m)
    res = (CaseResult * kk)()
    st = Stats()
    rc = fn(C.c_int(m), C.c_int(n), _ip(lp.start), _ip(lp.index), _dp(lp.value), _dp(lp.col_cost),
            _dp(lp.col_lower), _dp(lp.col_upper), _dp(lp.row_lower), _dp(lp.row_upper), C.c_double(lp.obj_offset),
            C.c_int(k), cc, cl, cu, rl, ru, C.byref(o), _dp(x), _dp(y), res, C.byref(st))
    if rc != 0:
        raise RuntimeError(f"{lib} solve failed")
    out = [OracleResult(res[b].status, res[b].iterations, res[b].objective, res[b].dual_objective,
                        res[b].relative_kkt, x[b * n:(b + 1) * n].copy(), y[b * m:(b + 1) * m].copy())
           for b in range(kk)]
    solve.last_stats = {f: getattr(st, f) for f, _ in Stats._fields_}
    if lib == "ref":
        h.ref_last_backend.restype = C.c_char_p
        h.ref_last_kernel_seconds.restype = C.c_double
        solve.last_stats["backend"] = h.ref_last_backend().decode()
        solve.last_stats["kernel_seconds"] = h.ref_last_kernel_seconds()
    return out if cases is not None else out[0]


def load_mps(path: str, presolve: bool = True):
    """The LP that the reference's solve() hands to its LP engines for an MPS
    file: read by its own reader, in minimisation form and, with presolve,
    reduced by its Presolver (src/api/solver.cpp:251, 302-333; ref build).
    Returns (Model, rows removed, columns removed)."""
    from pramana_b200.model import Model
    h = _load("ref")
    dims = np.zeros(5, dtype=np.int32)
    off = C.c_double()
    if h.ref_load_mps(path.encode(), C.c_int(1 if presolve else 0), _ip(dims), C.byref(off)) != 0:
        h.ref_last_error.restype = C.c_char_p
        raise RuntimeError("reference MPS load failed: " + h.ref_last_error().decode())
    m, n, nnz = int(dims[0]), int(dims[1]), int(dims[2])
    start, index = np.zeros(n + 1, dtype=np.int32), np.zeros(nnz, dtype=np.int32)
    value, cost, cl, cu = np.zeros(nnz), np.zeros(n), np.zeros(n), np.zeros(n)
    rl, ru = np.zeros(m), np.zeros(m)
    h.ref_model_arrays(_ip(start), _ip(index), _dp(value), _dp(cost), _dp(cl), _dp(cu), _dp(rl), _dp(ru))
    lp = Model(num_rows=m, num_cols=n, start=start, index=index, value=value, col_cost=cost, col_lower=cl,
               col_upper=cu, row_lower=rl, row_upper=ru, obj_offset=off.value, name=os.path.basename(path))
    return lp, int(dims[3]), int(dims[4])


def loaded_column(name: str):
    """(index of column `name`, was the file a maximisation) for the model of
    the last load_mps (ref build)."""
    h = _load("ref")
    was_max = C.c_int()
    j = h.ref_loaded_column(name.encode(), C.byref(was_max))
    return int(j), bool(was_max.value)


def safe_dual_bound(lp, y, col_lower=None, col_upper=None, full: bool = False):
    """The reference's outward-rounded Neumaier-Shcherbina bound (needs the ref
    build), plus the objective offset; with full=True the whole SafeBoundResult
    (bound without offset)."""
    h = _load("ref")
    lo = np.ascontiguousarray(lp.col_lower if col_lower is None else col_lower, dtype=np.float64)
    up = np.ascontiguousarray(lp.col_upper if col_upper is None else col_upper, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    bound = C.c_double()
    inf_terms = C.c_int()
    extra = np.zeros(3)
    rc = h.ref_safe_dual_bound(C.c_int(lp.num_rows), C.c_int(lp.num_cols), _ip(lp.start), _ip(lp.index),
                               _dp(lp.value), _dp(lp.col_cost), _dp(lo), _dp(up), _dp(lp.row_lower),
                               _dp(lp.row_upper), _dp(y), C.byref(bound), C.byref(inf_terms), _dp(extra))
    if rc != 0:
        raise RuntimeError("safe bound failed")
    if full:
        return {"bound": bound.value, "infinite_terms": inf_terms.value, "max_dual_infeasibility": extra[0],
                "row_projection": extra[1], "cost_perturbation": extra[2]}
    return bound.value + lp.obj_offset


def implied_bounds(lp, col_lower=None, col_upper=None):
    """The reference certifier's constraint-implied column bounds (ref build)."""
    h = _load("ref")
    lo = np.ascontiguousarray(lp.col_lower if col_lower is None else col_lower, dtype=np.float64)
    up = np.ascontiguousarray(lp.col_upper if col_upper is None else col_upper, dtype=np.float64)
    lo_out, up_out = np.zeros(lp.num_cols), np.zeros(lp.num_cols)
    rc = h.ref_implied_bounds(C.c_int(lp.num_rows), C.c_int(lp.num_cols), _ip(lp.start), _ip(lp.index),
                              _dp(lp.value), _dp(lo), _dp(up), _dp(lp.row_lower), _dp(lp.row_upper), _dp(lo_out),
                              _dp(up_out))
    if rc != 0:
        raise RuntimeError("implied bounds failed")
    return lo_out, up_out


CERT_FIELDS = ("accepted", "primal_objective", "safe_dual_bound", "certified_gap", "max_primal_violation",
               "max_col_violation", "max_row_violation", "max_dual_violation", "cost_perturbation",
               "used_implied_bounds")


def certify(lp, x, y, tol=(1e-6, 1e-6, 1e-6)) -> dict:
    """pramana::certify of an OPTIMAL claim (x, y) of a min-form LP (ref build)."""
    h = _load("ref")
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    t = np.ascontiguousarray(tol, dtype=np.float64)
    out = np.zeros(10)
    rc = h.ref_certify_lp(C.c_int(lp.num_rows), C.c_int(lp.num_cols), _ip(lp.start), _ip(lp.index), _dp(lp.value),
                          _dp(lp.col_cost), _dp(lp.col_lower), _dp(lp.col_upper), _dp(lp.row_lower),
                          _dp(lp.row_upper), C.c_double(lp.obj_offset), _dp(x), _dp(y), _dp(t), _dp(out))
    if rc != 0:
        raise RuntimeError("certify failed")
    d = dict(zip(CERT_FIELDS, out.tolist()))
    d["accepted"] = int(d["accepted"])
    d["used_implied_bounds"] = int(d["used_implied_bounds"])
    return d


def simplex(lp, x=None, y=None) -> dict:
    """The reference's simplex (ref build): crossover from (x, y) when given,
    else a solve from scratch.  Returns status name, objective, iterations."""
    h = _load("ref")
    out = np.zeros(3)
    xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
    ya = None if y is None else np.ascontiguousarray(y, dtype=np.float64)
    rc = h.ref_simplex(C.c_int(lp.num_rows), C.c_int(lp.num_cols), _ip(lp.start), _ip(lp.index), _dp(lp.value),
                       _dp(lp.col_cost), _dp(lp.col_lower), _dp(lp.col_upper), _dp(lp.row_lower), _dp(lp.row_upper),
                       C.c_double(lp.obj_offset), _dp(xa) if xa is not None else None,
                       _dp(ya) if ya is not None else None, _dp(out))
    if rc != 0:
        raise RuntimeError("simplex failed")
    return {"status": STATUS_NAMES.get(int(out[0]), str(int(out[0]))), "objective": out[1],
            "iterations": int(out[2])}


def ruiz(lp, lib: str = "oracle", iterations: int = 10, pock_chambolle: bool = True):
    h = _load(lib)
    fn = h.oracle_ruiz_scaling if lib == "oracle" else h.ref_ruiz_scaling
    rs = np.zeros(lp.num_rows)
    cs = np.zeros(lp.num_cols)
    rc = fn(C.c_int(lp.num_rows), C.c_int(lp.num_cols), _ip(lp.start), _ip(lp.index), _dp(lp.value),
            C.c_int(iterations), C.c_int(int(pock_chambolle)), _dp(rs), _dp(cs))
    if rc != 0:
        raise RuntimeError("ruiz failed")
    return rs, cs


def power_norm(m, n, start, index, value, iters=40) -> float:
    h = _load("oracle")
    h.oracle_power_iteration.restype = C.c_double
    return h.oracle_power_iteration(C.c_int(m), C.c_int(n), _ip(start), _ip(index), _dp(value), C.c_int(iters))


def csr_mult(ptr, idx, val, x, rows, k=1):
    h = _load("oracle")
    out = np.zeros(rows * k)
    h.oracle_csr_mult(C.c_int(rows), C.c_int(k), _ip(ptr), _ip(idx), _dp(val), _dp(x), _dp(out))
    return out


# ---- the reference's router and CPU engines (ref build), for the router calibration ----

ROUTER_ENGINES = ["dual", "ipm", "pdhg-cpu", "pdhg-gpu"]


def _lp_args(lp):
    return (C.c_int(lp.num_rows), C.c_int(lp.num_cols), _ip(lp.start), _ip(lp.index), _dp(lp.value),
            _dp(lp.col_cost), _dp(lp.col_lower), _dp(lp.col_upper), _dp(lp.row_lower), _dp(lp.row_upper))


def router_features(lp) -> dict:
    """computeFeatures (src/router/router.cpp:64-95) of the reference."""
    h = _load("ref")
    out = np.zeros(10)
    if h.ref_router_features(*_lp_args(lp), _dp(out)) != 0:
        raise RuntimeError("router_features failed")
    keys = ["rows", "cols", "nnz", "avg_row_nnz", "max_row_nnz", "coefficient_range", "equality_row_fraction",
            "free_column_fraction", "is_mip", "is_qp"]
    return dict(zip(keys, out.tolist()))


def router_decide(lp, model_path=None, gpu: bool = True, tolerance: float = 1e-6) -> dict:
    """Router::decide (src/router/router.cpp:163-207) with the weights in
    `model_path` (Router::load) or the built-in priors."""
    h = _load("ref")
    eng = C.c_int(-1)
    loaded = C.c_int(0)
    pred = np.zeros(4)
    path = None if model_path is None else str(model_path).encode()
    rc = h.ref_router_decide(*_lp_args(lp), C.c_char_p(path), C.c_int(int(gpu)), C.c_double(tolerance),
                             C.byref(eng), _dp(pred), C.byref(loaded))
    if rc != 0:
        raise RuntimeError("router_decide failed")
    return {"engine": ROUTER_ENGINES[eng.value] if eng.value >= 0 else None, "predicted": pred.tolist(),
            "loaded": bool(loaded.value)}


def timed_solve(lp, engine: str, time_limit: float) -> dict:
    """A solve from scratch by the reference's dual simplex ("dual") or
    interior-point method ("ipm") under a time limit."""
    h = _load("ref")
    out = np.zeros(4)
    which = {"dual": 0, "ipm": 1}[engine]
    rc = h.ref_timed_solve(C.c_int(which), *_lp_args(lp), C.c_double(lp.obj_offset), C.c_double(time_limit),
                           _dp(out))
    if rc != 0:
        raise RuntimeError("timed_solve failed")
    return {"status": STATUS_NAMES.get(int(out[0]), str(int(out[0]))), "objective": out[1], "seconds": out[2],
            "iterations": int(out[3])}
