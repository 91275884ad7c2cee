"""Recalibration of PRAMANA's CPU <-> GPU engine router for B200 timings.

PRAMANA's router (src/router/router.cpp) predicts each engine's wall time from
eight structural features with a log-linear model, log t_e = w_e . phi(LP), and
runs the engine with the smallest predicted time (plus its rules for
first-order polish and tight tolerances).  Its weights come from
bench/fit_router.py, a ridge fit on measured runs, written to
router_model.json, which Router::load reads (router.cpp:132-149; the
PRAMANA_ROUTER_MODEL environment variable or a file beside the executable).

This module restates, from those sources:
  * the features and phi (computeFeatures, router.cpp:64-95; phi, :24-33),
  * the decision rule (Router::decide, router.cpp:163-207),
  * the fit (ridge least squares on log(t + 1e-3), unsolved runs censored at
    4x the time limit) and its validation (5 folds, members of each instance
    family spread over the folds, held-out regret against the fastest engine),
and writes the model in the file format Router::load accepts.  The timings
it is fitted on are measured on the B200 host with the engine of this
library as "pdhg-gpu" (bench.py --workload router).
"""
from __future__ import annotations

import json
import math
import random
from dataclasses import dataclass, field

import numpy as np

from .model import Model

ENGINES = ["dual", "ipm", "pdhg-cpu", "pdhg-gpu"]
FEATURE_NAMES = ["1", "log(m+n)", "log(nnz)", "log(nnz/row)", "log(max row nnz)", "log(coef range)", "eq fraction",
                 "free fraction"]
INF_BOUND = 1e20  # src/util/common.h:14

# The router's built-in priors (router.cpp:97-104): used when no model file loads.
DEFAULT_WEIGHTS = {
    "dual": [-13.0, 1.20, 0.35, 0.30, 0.00, 0.05, 0.20, 0.30],
    "ipm": [-12.0, 0.40, 1.00, 0.40, 0.10, 0.03, 0.00, 0.00],
    "pdhg-cpu": [-11.5, 0.60, 0.80, 0.00, 0.10, 0.15, 0.30, 0.00],
    "pdhg-gpu": [-6.0, 0.20, 0.35, 0.00, 0.05, 0.15, 0.30, 0.00],
}


def features(lp: Model) -> dict:
    """computeFeatures (router.cpp:64-95) of an LP given in CSC form."""
    m, n = int(lp.num_rows), int(lp.num_cols)
    index = np.asarray(lp.index, dtype=np.int64)
    value = np.abs(np.asarray(lp.value, dtype=np.float64))
    nnz = int(len(index))
    rows = np.bincount(index, minlength=m) if m else np.zeros(0, dtype=np.int64)
    nz = value[value > 0]
    mx = float(nz.max()) if nz.size else 0.0
    mn = float(nz.min()) if nz.size else math.inf
    lo, up = np.asarray(lp.col_lower, dtype=np.float64), np.asarray(lp.col_upper, dtype=np.float64)
    rl, ru = np.asarray(lp.row_lower, dtype=np.float64), np.asarray(lp.row_upper, dtype=np.float64)
    eq = int(np.count_nonzero(rl == ru))
    free = int(np.count_nonzero(~(np.abs(lo) < INF_BOUND) & ~(np.abs(up) < INF_BOUND)))
    return {"rows": float(m), "cols": float(n), "nnz": float(nnz),
            "avg_row_nnz": float(nnz) / m if m > 0 else 0.0,
            "max_row_nnz": float(rows.max()) if m > 0 else 0.0,
            "coefficient_range": mx / mn if mx > 0 else 1.0,
            "equality_row_fraction": eq / float(m) if m > 0 else 0.0,
            "free_column_fraction": free / float(n) if n > 0 else 0.0}


def phi(f: dict) -> list[float]:
    """The regression features of RouterFeatures::phi (router.cpp:24-33)."""
    def lg(v):
        return math.log(max(float(v), 1.0))
    return [1.0, lg(f["rows"] + f["cols"]), lg(f["nnz"]), lg(f["avg_row_nnz"]), lg(f["max_row_nnz"]),
            lg(f["coefficient_range"]), float(f["equality_row_fraction"]), float(f["free_column_fraction"])]


def predict(weights: dict, f: dict) -> dict:
    """Predicted seconds per engine: exp(w_e . phi)."""
    p = phi(f)
    return {e: math.exp(sum(w * x for w, x in zip(weights[e], p))) for e in ENGINES}


def decide(weights: dict, f: dict, gpu: bool = True, tolerance: float = 1e-6) -> tuple[str, dict]:
    """Router::decide's choice for an LP (router.cpp:163-207): a first-order
    engine pays a predicted crossover polish (0.15 x the dual simplex time),
    tolerances below 1e-7 multiply first-order times by 4, the IPM pays 10 %
    for its crossover; the smallest total wins (first in engine order on ties)."""
    pred = predict(weights, f)
    if not gpu:
        pred["pdhg-gpu"] = math.inf
    polish = 0.15 * pred["dual"]
    tight = 4.0 if tolerance < 1e-7 else 1.0
    total = {"dual": pred["dual"], "ipm": pred["ipm"] * 1.1, "pdhg-cpu": pred["pdhg-cpu"] * tight + polish,
             "pdhg-gpu": pred["pdhg-gpu"] * tight + polish}
    best = min(ENGINES, key=lambda e: total[e])
    return best, pred


@dataclass
class Record:
    """One LP measured by every engine: seconds per engine (None = not solved
    within `limit`), its features and its instance family."""
    name: str
    family: str
    features: dict
    times: dict
    limit: float
    statuses: dict = field(default_factory=dict)

    def time(self, engine: str) -> float:
        t = self.times.get(engine)
        return 4.0 * self.limit if t is None else float(t)  # censored at 4x the limit


def ridge(X, y, lam: float = 1e-2) -> np.ndarray:
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    return np.linalg.solve(X.T @ X + lam * np.eye(X.shape[1]), X.T @ y)


def fit(records: list[Record], lam: float = 1e-2) -> dict:
    """Per-engine ridge fit of log(t + 1e-3) on phi."""
    X = [phi(r.features) for r in records]
    return {e: ridge(X, [math.log(r.time(e) + 1e-3) for r in records], lam).tolist() for e in ENGINES}


def folds(records: list[Record], k: int = 5, seed: int = 1) -> dict:
    """Fold of each record: the members of each family are shuffled (seeded)
    and dealt round-robin, so every fold holds out part of every family."""
    rng = random.Random(seed)
    out = {}
    for fam in sorted({r.family for r in records}):
        members = sorted(r.name for r in records if r.family == fam)
        rng.shuffle(members)
        for i, name in enumerate(members):
            out[name] = i % k
    return out


def _regret(records: list[Record], choice: dict) -> dict:
    r = [(rec.time(choice[rec.name]) + 1e-3) / (min(rec.time(e) for e in ENGINES) + 1e-3) for rec in records]
    return {"geo_mean_regret": math.exp(sum(math.log(x) for x in r) / len(r)), "worst_regret": max(r),
            "picks_fastest": sum(1 for x in r if x <= 1.0001) / len(r)}


def validate(records: list[Record], k: int = 5, lam: float = 1e-2, tolerance: float = 1e-6) -> dict:
    """Held-out evaluation: for each fold, fit on the others and choose for
    the held-out LPs (smallest predicted time, as fit_router.py does, and the
    full Router::decide rule); report regret against the fastest measured
    engine, beside the fixed policies and the built-in priors."""
    fold = folds(records, k)
    by_pred, by_rule = {}, {}
    for f in range(k):
        train = [r for r in records if fold[r.name] != f]
        test = [r for r in records if fold[r.name] == f]
        if not train or not test:
            continue
        W = fit(train, lam)
        for r in test:
            p = predict(W, r.features)
            by_pred[r.name] = min(ENGINES, key=lambda e: p[e])
            by_rule[r.name] = decide(W, r.features, True, tolerance)[0]
    held = [r for r in records if r.name in by_pred]
    out = {"instances": len(held), "families": sorted({r.family for r in records}),
           "router_held_out": _regret(held, by_pred),
           "router_held_out_decide_rule": _regret(held, by_rule),
           "builtin_priors_decide_rule": _regret(held, {r.name: decide(DEFAULT_WEIGHTS, r.features, True,
                                                                       tolerance)[0] for r in held})}
    for e in ENGINES:
        out[f"always_{e}"] = _regret(held, {r.name: e for r in held})
    out["fastest_counts"] = {e: sum(1 for r in held if min(ENGINES, key=r.time) == e) for e in ENGINES}
    return out


def model_json(weights: dict, instances: int, note: str = "") -> dict:
    """The file Router::load reads: {"weights": {engine: 8 numbers}, ...}."""
    d = {"weights": {e: [float(v) for v in weights[e]] for e in ENGINES}, "features": FEATURE_NAMES,
         "instances": int(instances)}
    if note:
        d["note"] = note
    return d


def write_model(path, weights: dict, instances: int, note: str = "") -> None:
    with open(path, "w") as fh:
        json.dump(model_json(weights, instances, note), fh, indent=1)


def load_model(path) -> dict:
    with open(path) as fh:
        d = json.load(fh)
    return {e: list(map(float, d["weights"][e])) for e in ENGINES}
