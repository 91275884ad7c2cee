"""Learned warm start for a parametric LP family.

A family member differs from its base LP only in some costs and bounds, so a
whole batch shares A and is solved as one batched PDHG run (the reference's
solvePdhgBatch with per-case overrides, src/pdhg/pdhg.h:67-70 -- the same
shape as its "batched PDHG" family strategy, src/parametric/parametric.cpp:
486-520).  The pieces:

* ``RefineryFamily`` -- the multi-period refinery-planning LP with 16
  parameters: the crude prices and the demand scales of 10 product pools;
* ``PcaBasis`` -- standardised PCA of stacked primal-dual solutions [x; y];
* ``LearnedWarmStart`` -- a ReLU MLP (``MlpNetwork``, trained and evaluated
  on the tensor cores) from normalised parameters to PCA coefficients, whose
  decoded [x; y] starts PDHG;
* ``NearestWarmStart`` -- the baseline: the stored solution of the nearest
  training parameter vector;
* ``solve_family`` / ``certify_family`` -- batched solves from any start
  (one shared-A batch per chunk, or the multi-LP engine that drops members
  as they finish) and their certification: the KKT error recomputed on the
  GPU, the reference's family rule for the safe dual bound, and the
  reference certifier's full verdict.

A start only moves PDHG's initial point: the solve, its termination test and
the certification are the same as from a cold start, which stays the
fallback (``solve_family`` with ``starts=None``).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field, replace

import numpy as np

from . import generators as G
from .mlp import MlpNetwork, TrainOptions
from .model import LpCase, Model
from .pdhg import (Engine, PdhgOptions, PdhgResult, certifyLp, impliedBounds, kktResidual, safeDualBound,
                   solvePdhgMulti)

N_DEMAND = 10


class RefineryFamily:
    """Refinery-planning LPs (generators.refinery_lp) over one fixed
    structure; parameters p = (crude prices (crudes), demand scales (10))."""

    def __init__(self, seed: int = 5, crudes: int = 6, price_range=(40.0, 120.0), scale_range=(0.8, 1.2), **size):
        size.setdefault("pools", N_DEMAND)
        if size["pools"] < N_DEMAND:
            raise ValueError("the family scales the demand of 10 pools")
        self.crudes = crudes
        self.lo = np.array([price_range[0]] * crudes + [scale_range[0]] * N_DEMAND)
        self.hi = np.array([price_range[1]] * crudes + [scale_range[1]] * N_DEMAND)
        mid = 0.5 * (self.lo + self.hi)
        self.base: Model = G.refinery_lp(seed=seed, crudes=crudes, crude_prices=mid[:crudes],
                                         demand_scales=mid[crudes:], **size)
        meta = self.base.meta
        self.buy = np.asarray(meta["buy_cols"])        # T x C
        self.sale = np.asarray(meta["sale_cols"])      # R x T x P
        self.col_scale = np.asarray(meta["col_scale"])
        demand = np.asarray(meta["demand"]).copy()     # R x P, at the mid scales
        demand[:, :N_DEMAND] /= mid[crudes:]
        self.demand = demand                           # unscaled base demand
        self.num_params = crudes + N_DEMAND

    def sample(self, count: int, seed: int) -> np.ndarray:
        rng = np.random.default_rng(seed)
        return self.lo + (self.hi - self.lo) * rng.random((count, self.num_params))

    def normalize(self, params) -> np.ndarray:
        p = np.asarray(params, dtype=np.float64).reshape(-1, self.num_params)
        return ((p - 0.5 * (self.lo + self.hi)) / (0.5 * (self.hi - self.lo))).astype(np.float32)

    def case(self, p) -> LpCase:
        p = np.asarray(p, dtype=np.float64)
        cost = self.base.col_cost.copy()
        up = self.base.col_upper.copy()
        prices, scales = p[:self.crudes], p[self.crudes:]
        cost[self.buy] = prices[None, :] * self.col_scale[self.buy]
        dem = self.demand.copy()
        dem[:, :N_DEMAND] *= scales[None, :]
        R, T, P = self.sale.shape
        up[self.sale] = dem[:, None, :] / self.col_scale[self.sale]
        return LpCase(cost=cost, col_upper=up)

    def instance(self, p) -> Model:
        c = self.case(p)
        b = self.base
        return Model(num_rows=b.num_rows, num_cols=b.num_cols, start=b.start, index=b.index, value=b.value,
                     col_cost=c.cost, col_lower=b.col_lower, col_upper=c.col_upper, row_lower=b.row_lower,
                     row_upper=b.row_upper, obj_offset=b.obj_offset, name=f"{b.name}_member")


class PcaBasis:
    """Standardised PCA: z -> ((z - mean) / scale) V, V the leading right
    singular vectors of the standardised training matrix.

    The leading singular subspace is found by a randomized range finder
    (Halko, Martinsson and Tropp, SIAM Review 53 (2011), Algorithms 4.4 and
    5.1): the standardised matrix S (members x (n + m)) is multiplied by a
    Gaussian test matrix of rank + `oversample` columns, `power` subspace
    iterations (re-orthonormalised every time) sharpen the spectrum, and the
    SVD of the small projected matrix gives the basis.  Work and memory are
    O(members x (n + m) x (rank + oversample)), never the members x (n + m)
    SVD, so solution vectors of hundreds of thousands of entries are fine.
    The share of the total energy the basis keeps is recorded (`explained`)."""

    def fit(self, Z: np.ndarray, rank: int, oversample: int = 16, power: int = 3, seed: int = 0) -> "PcaBasis":
        Z = np.asarray(Z, dtype=np.float64)
        self.mean = Z.mean(axis=0)
        sd = Z.std(axis=0)
        self.scale = np.where(sd > 1e-12 * max(1.0, float(np.abs(Z).max())), sd, 1.0)
        S = (Z - self.mean) / self.scale
        members, width = S.shape
        k = min(rank + oversample, members, width)
        rng = np.random.default_rng(seed)
        Q, _ = np.linalg.qr(S @ rng.standard_normal((width, k)))
        for _ in range(power):
            W, _ = np.linalg.qr(S.T @ Q)
            Q, _ = np.linalg.qr(S @ W)
        _, sv, vt = np.linalg.svd(Q.T @ S, full_matrices=False)
        r = min(rank, vt.shape[0])
        self.V = vt[:r].T.copy()
        if r < rank:  # pad with zero directions so the coefficient count stays `rank`
            self.V = np.hstack([self.V, np.zeros((self.V.shape[0], rank - r))])
        total = float(np.einsum("ij,ij->", S, S))
        self.explained = float((sv[:r] ** 2).sum() / max(total, 1e-300))
        return self

    def encode(self, Z) -> np.ndarray:
        return ((np.asarray(Z, dtype=np.float64) - self.mean) / self.scale) @ self.V

    def decode(self, Cf) -> np.ndarray:
        return self.mean + (np.asarray(Cf, dtype=np.float64) @ self.V.T) * self.scale


class LearnedWarmStart:
    """MLP (normalised parameters -> PCA coefficients of [x; y])."""

    def __init__(self, family: RefineryFamily, hidden=(512, 512, 512), rank: int = 128, max_batch: int = 1024,
                 seed: int = 0, device: int = -1):
        self.family = family
        self.rank = rank
        self.widths = [family.num_params, *hidden, rank]
        # the input width is padded to a multiple of 8 with zero features
        self.in_width = -(-family.num_params // 8) * 8
        self.widths[0] = self.in_width
        self.net = MlpNetwork(self.widths, max_batch=max_batch, device=device, seed=seed)
        self.basis: PcaBasis | None = None
        self.coef_scale = 1.0
        self.train_seconds = 0.0

    def _features(self, params) -> np.ndarray:
        f = self.family.normalize(params)
        if self.in_width > f.shape[1]:
            f = np.hstack([f, np.zeros((f.shape[0], self.in_width - f.shape[1]), dtype=np.float32)])
        return f

    def fit(self, params, X, Y, opts: TrainOptions | None = None) -> np.ndarray:
        Z = np.hstack([np.asarray(X), np.asarray(Y)])
        self.n = np.asarray(X).shape[1]
        self.basis = PcaBasis().fit(Z, self.rank)
        Cf = self.basis.encode(Z)
        self.coef_scale = float(np.sqrt(np.mean(Cf ** 2))) or 1.0
        t0 = time.perf_counter()
        losses = self.net.train(self._features(params), (Cf / self.coef_scale).astype(np.float32), opts)
        self.train_seconds = time.perf_counter() - t0
        return losses

    def predict(self, params):
        """Starts (X, Y) in the original space; a member whose prediction is
        not finite gets x = 0, y = 0, which the engine turns into exactly
        the cold start (x projected onto the bounds)."""
        Cf = self.net.forward(self._features(params)).astype(np.float64) * self.coef_scale
        Z = self.basis.decode(Cf)
        bad = ~np.all(np.isfinite(Z), axis=1)
        Z[bad] = 0.0
        return Z[:, :self.n], Z[:, self.n:]


class NearestWarmStart:
    """Start from the stored solution of the nearest training parameters."""

    def __init__(self, family: RefineryFamily):
        self.family = family

    def fit(self, params, X, Y):
        self.P = self.family.normalize(params).astype(np.float64)
        self.X, self.Y = np.asarray(X), np.asarray(Y)
        return self

    def predict(self, params):
        Q = self.family.normalize(params).astype(np.float64)
        d = (Q ** 2).sum(1)[:, None] - 2.0 * Q @ self.P.T + (self.P ** 2).sum(1)[None, :]
        j = np.argmin(d, axis=1)
        return self.X[j], self.Y[j]


class WorkEstimate:
    """Predicted work of a member: the mean cold iteration count of its four
    nearest training members (normalised parameters).  Used to launch the
    members of a batch in decreasing predicted work, so that the hardest ones
    do not start last (longest-processing-time order).  Fitted with the
    training members' final primal weights too, it predicts a member's
    starting primal weight: their geometric mean."""

    def __init__(self, family: RefineryFamily, neighbours: int = 4):
        self.family = family
        self.k = neighbours
        self.w = None

    def fit(self, params, iterations, weights=None):
        self.P = self.family.normalize(params).astype(np.float64)
        self.it = np.asarray(iterations, dtype=np.float64)
        if weights is not None:
            w = np.asarray(weights, dtype=np.float64)
            self.w = np.where(np.isfinite(w) & (w > 0), w, np.nan)
        return self

    def _nearest(self, params) -> np.ndarray:
        Q = self.family.normalize(params).astype(np.float64)
        d = (Q ** 2).sum(1)[:, None] - 2.0 * Q @ self.P.T + (self.P ** 2).sum(1)[None, :]
        k = min(self.k, d.shape[1])
        return np.argpartition(d, k - 1, axis=1)[:, :k]

    def predict(self, params) -> np.ndarray:
        return self.it[self._nearest(params)].mean(axis=1)

    def predict_weight(self, params) -> np.ndarray:
        """Starting primal weights (original-space units, as
        solvePdhgMulti's primalWeights); 0 (the default weight) where no
        neighbour has one."""
        if self.w is None:
            raise ValueError("WorkEstimate was fitted without weights")
        lw = np.log(self.w[self._nearest(params)])
        have = np.isfinite(lw)
        mean = np.where(have, lw, 0.0).sum(axis=1) / np.maximum(have.sum(axis=1), 1)
        return np.where(have.any(axis=1), np.exp(mean), 0.0)


@dataclass
class FamilySolve:
    status: np.ndarray          # per instance (1 = Optimal)
    iterations: np.ndarray
    relative_kkt: np.ndarray
    objective: np.ndarray
    X: np.ndarray
    Y: np.ndarray
    seconds: float = 0.0        # wall time: engine setup + start + solve + fetch
    solve_seconds: float = 0.0  # the PDHG loop alone
    batches: list = field(default_factory=list)
    weights: np.ndarray = field(default_factory=lambda: np.zeros(0))  # final primal weights (engine "multi")


def solve_family(family: RefineryFamily, params, opts: PdhgOptions | None = None, starts=None,
                 batch: int = 1024, engine: str = "batch", work=None, weights=None) -> FamilySolve:
    """Batched PDHG over the family members `params`, in batches of `batch`
    members; `starts` = (X, Y) in the original space, or None (cold start).
    engine "batch": one shared-A k-case solve per chunk (the live cases are
    packed narrower as others finish); "multi": the multi-LP engine (one
    thread block per member in its CTA form); "single": the single-LP engine
    per member, one after another (every SM on one member: for a handful of
    members).  `work` (per member, optional):
    predicted work; within each chunk the multi-LP engine gets the members in
    decreasing predicted work, which is the order its blocks start in.
    `weights` (per member, optional; engine "multi"): starting primal weights.
    Results come back in the members' order; with engine "multi" the result's
    `weights` holds each member's final primal weight."""
    opts = opts or PdhgOptions()
    params = np.asarray(params, dtype=np.float64).reshape(-1, family.num_params)
    n, m = family.base.num_cols, family.base.num_rows
    out = FamilySolve(*(np.zeros(0) for _ in range(4)), X=np.zeros((0, n)), Y=np.zeros((0, m)))
    parts = []
    for b0 in range(0, len(params), batch):
        sl = slice(b0, min(b0 + batch, len(params)))
        t0 = time.perf_counter()
        if engine == "multi":
            idx = np.arange(sl.start, sl.stop)
            if work is not None:
                idx = idx[np.argsort(-np.asarray(work, dtype=np.float64)[idx], kind="stable")]
            lps = [family.instance(p) for p in params[idx]]
            st = None if starts is None else list(zip(np.asarray(starts[0])[idx], np.asarray(starts[1])[idx]))
            pw = None if weights is None else np.asarray(weights, dtype=np.float64)[idx]
            t1 = time.perf_counter()
            res = solvePdhgMulti(lps, opts, starts=st, primalWeights=pw)
            t2 = time.perf_counter()
            t1 = t2 - res[0].stats.solveSeconds if res else t1
            back = np.empty(len(idx), dtype=np.int64)
            back[idx - sl.start] = np.arange(len(idx))
            res = [res[q] for q in back]
        elif engine == "single":
            res = []
            t1 = time.perf_counter()
            for q in range(sl.start, sl.stop):
                with Engine(family.instance(params[q]), opts) as eng:
                    if starts is not None:
                        eng.set_start(np.asarray(starts[0])[q], np.asarray(starts[1])[q])
                    r = eng.solve()[0]
                res.append(PdhgResult(**{**r.__dict__, "primalWeight": 0.0}))
            t2 = time.perf_counter()
        else:
            cases = [family.case(p) for p in params[sl]]
            eng = Engine(family.base, opts, cases)
            try:
                if starts is not None:
                    eng.set_start(np.asarray(starts[0])[sl], np.asarray(starts[1])[sl])
                t1 = time.perf_counter()
                res = eng.solve()
                t2 = time.perf_counter()
            finally:
                eng.close()
        wall = time.perf_counter() - t0
        parts.append(res)
        out.seconds += wall
        out.solve_seconds += t2 - t1
        out.batches.append({"cases": len(res), "seconds": wall, "solve_seconds": t2 - t1,
                            "iterations": int(max(r.iterations for r in res))})
    res = [r for p in parts for r in p]
    out.status = np.array([1 if r.status == "Optimal" else 0 for r in res])
    out.iterations = np.array([r.iterations for r in res])
    out.relative_kkt = np.array([r.relativeKkt for r in res])
    out.objective = np.array([r.objective for r in res])
    out.X = np.array([r.x for r in res]).reshape(-1, n)
    out.Y = np.array([r.rowDual for r in res]).reshape(-1, m)
    out.weights = np.array([r.primalWeight for r in res])
    return out


def certify_family(family: RefineryFamily, params, X, Y, kkt_tol: float = 1e-6, family_gap: float = 1e-4):
    """Judges solutions of family members three ways, per member:

    * ``kkt``: the relative KKT error (relP, relD, gap, max) recomputed on the
      GPU from (x, y) in the original space (b2p_kkt_residual);
    * ``family_certified``: the reference's family rule
      (src/parametric/parametric.cpp:510-526): the safe dual bound over the
      constraint-implied column bounds is finite and within `family_gap`
      (1 + |obj|) of the objective;
    * ``certificate``: the reference certifier's full verdict on an OPTIMAL
      claim (b2p_certify_lp; 1e-6 primal, dual and gap tolerances).

    ``certified`` = max KKT <= kkt_tol and family_certified."""
    params = np.asarray(params, dtype=np.float64).reshape(-1, family.num_params)
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    base = family.base
    out = {k: [] for k in ("kkt", "objective", "bound", "family_certified", "accepted", "certified_gap",
                           "primal_violation")}
    for b0 in range(0, len(params), 1024):
        sl = slice(b0, b0 + 1024)
        cases = [family.case(p) for p in params[sl]]
        out["kkt"].append(kktResidual(base, X[sl].reshape(-1), Y[sl].reshape(-1), cases))
        lo, up = impliedBounds(base, cases)
        icases = [LpCase(cost=c.cost, col_lower=lo[q], col_upper=up[q]) for q, c in enumerate(cases)]
        sb = safeDualBound(base, Y[sl].reshape(-1), icases)
        obj = np.array([float(np.dot(c.cost, x)) for c, x in zip(cases, X[sl])]) + base.obj_offset
        bound = np.array([d["bound"] for d in sb]) + base.obj_offset
        out["objective"].append(obj)
        out["bound"].append(bound)
        out["family_certified"].append(np.isfinite(bound) & (np.abs(obj - bound) <= family_gap * (1 + np.abs(obj))))
        certs = certifyLp(base, X[sl].reshape(-1), Y[sl].reshape(-1), cases)
        out["accepted"].append(np.array([c["accepted"] for c in certs], dtype=bool))
        out["certified_gap"].append(np.array([c["certified_gap"] for c in certs]))
        out["primal_violation"].append(np.array([c["max_primal_violation"] for c in certs]))
    res = {k: (np.concatenate(v) if v else np.zeros(0)) for k, v in out.items()}
    res["certified"] = (res["kkt"][:, 3] <= kkt_tol) & res["family_certified"]
    return res


def solve_warm(family: RefineryFamily, params, predictor=None, opts: PdhgOptions | None = None, batch: int = 1024,
               engine: str = "batch", kkt_tol: float | None = None, work=None, weights=None,
               warm_max_iterations: int | None = None, single_fallback: int = 0, continue_failed: bool = True):
    """Solve from the predictor's starts (and, with engine "multi", the
    starting primal weights `weights`), judge every answer with
    certify_family, and re-solve the members that fail from a cold start
    (the fallback).  `warm_max_iterations` (optional) caps the warm attempt
    below opts.maxIterations, so that a start that leads nowhere falls back
    sooner; the fallback keeps opts.maxIterations.  A fallback of at most
    `single_fallback` members (default none) runs on the single-LP engine,
    one member at a time with every SM, instead of on `engine`.  With
    `continue_failed` (the default; engine "multi"), a member that fails
    first continues from its own final point and primal weight, and only
    what still fails then starts cold.  Returns (FamilySolve, certification,
    fallback mask)."""
    opts = opts or PdhgOptions()
    kkt_tol = opts.tolerance if kkt_tol is None else kkt_tol
    starts = predictor.predict(params) if predictor is not None else None
    warm_opts = opts
    if predictor is not None and warm_max_iterations is not None:
        warm_opts = replace(opts, maxIterations=min(opts.maxIterations, int(warm_max_iterations)))
    res = solve_family(family, params, warm_opts, starts=starts, batch=batch, engine=engine, work=work,
                       weights=weights)
    cert = certify_family(family, params, res.X, res.Y, kkt_tol=kkt_tol)
    redo = ~cert["certified"]
    if predictor is not None and continue_failed and engine == "multi" and redo.any():
        idx = np.flatnonzero(redo & np.all(np.isfinite(res.X), axis=1) & np.all(np.isfinite(res.Y), axis=1))
        if len(idx):
            w = res.weights[idx] if len(res.weights) == len(res.X) else None
            more = solve_family(family, np.asarray(params)[idx], opts, starts=(res.X[idx], res.Y[idx]), batch=batch,
                                engine=engine, work=None if work is None else np.asarray(work)[idx], weights=w)
            c3 = certify_family(family, np.asarray(params)[idx], more.X, more.Y, kkt_tol=kkt_tol)
            for f in ("status", "relative_kkt", "objective"):
                getattr(res, f)[idx] = getattr(more, f)
            res.iterations[idx] += more.iterations
            res.X[idx], res.Y[idx] = more.X, more.Y
            res.weights[idx] = more.weights
            res.seconds += more.seconds
            res.solve_seconds += more.solve_seconds
            for k in cert:
                cert[k][idx] = c3[k]
    if predictor is not None and (~cert["certified"]).any():
        idx = np.flatnonzero(~cert["certified"])
        again = solve_family(family, np.asarray(params)[idx], opts, batch=batch,
                             engine="single" if len(idx) <= single_fallback else engine,
                             work=None if work is None else np.asarray(work)[idx])
        c2 = certify_family(family, np.asarray(params)[idx], again.X, again.Y, kkt_tol=kkt_tol)
        warm_its = res.iterations[idx].copy()
        for f in ("status", "iterations", "relative_kkt", "objective"):
            getattr(res, f)[idx] = getattr(again, f)
        res.iterations[idx] += warm_its  # the work of both attempts
        res.X[idx], res.Y[idx] = again.X, again.Y
        res.weights[idx] = again.weights
        res.seconds += again.seconds
        res.solve_seconds += again.solve_seconds
        for k in cert:
            cert[k][idx] = c2[k]
    return res, cert, redo
