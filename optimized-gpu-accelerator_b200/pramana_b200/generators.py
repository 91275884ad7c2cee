"""Seeded synthetic LP generators for the PDHG workloads.

``random_lp`` builds the random sparse LPs of the two random-LP workloads:

* "C1": m=1,000 rows (600 equality, 400 <=), n=2,000 columns, 5 nonzeros per
  column at uniform random rows (10k nnz), values N(0,1), 0 <= x <= 10;
* "C2": the same construction at m=40,000, n=80,000, 6.4 nonzeros per column
  (512k nnz) with skewed rows: 1% of the rows hold 10% of the nonzeros.

Feasibility is built in (b = A x0, x0 ~ U(0,10), slack U(0,1) on the <= rows)
and so is a dual point (c = A^T y0 + s0, y0 ~ N(0,1), s0 ~ U(0,1)).  The
generator is pure numpy and deterministic for a given seed.
"""
from __future__ import annotations

import numpy as np

from .model import Model


def _draw_rows(rng, size, m, heavy_rows, light_rows, heavy_nnz_frac):
    if heavy_rows is None:
        return rng.integers(0, m, size=size, dtype=np.int64)
    is_heavy = rng.random(size) < heavy_nnz_frac
    h = heavy_rows[rng.integers(0, len(heavy_rows), size=size)]
    lt = light_rows[rng.integers(0, len(light_rows), size=size)]
    return np.where(is_heavy, h, lt)


def random_lp(m: int, n: int, nnz_per_col: float, n_eq: int, seed: int, heavy_row_frac: float = 0.0,
              heavy_nnz_frac: float = 0.0, name: str | None = None) -> Model:
    rng = np.random.default_rng(seed)
    base = int(np.floor(nnz_per_col))
    frac = nnz_per_col - base
    counts = base + (rng.random(n) < frac).astype(np.int64)
    counts = np.minimum(counts, m)
    col = np.repeat(np.arange(n, dtype=np.int64), counts)
    heavy_rows = light_rows = None
    if heavy_row_frac > 0 and heavy_nnz_frac > 0:
        nh = max(1, int(round(m * heavy_row_frac)))
        perm = rng.permutation(m)
        heavy_rows = np.sort(perm[:nh])
        light_rows = np.sort(perm[nh:])
    rows = _draw_rows(rng, len(col), m, heavy_rows, light_rows, heavy_nnz_frac)
    # Redraw entries that repeat a row inside their column until every column is duplicate-free.
    for _ in range(1000):
        key = col * m + rows
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(len(ks), dtype=bool)
        dup[1:] = ks[1:] == ks[:-1]
        if not dup.any():
            break
        idx = order[dup]
        rows[idx] = _draw_rows(rng, len(idx), m, heavy_rows, light_rows, heavy_nnz_frac)
    order = np.lexsort((rows, col))
    col, rows = col[order], rows[order]
    value = rng.standard_normal(len(col))
    start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=start[1:])

    x0 = rng.uniform(0.0, 10.0, size=n)
    b = np.zeros(m)
    np.add.at(b, rows, value * x0[col])
    eq = np.zeros(m, dtype=bool)
    eq[rng.permutation(m)[:n_eq]] = True
    slack = rng.uniform(0.0, 1.0, size=m)
    row_lower = np.where(eq, b, -np.inf)
    row_upper = np.where(eq, b, b + slack)
    y0 = rng.standard_normal(m)
    s0 = rng.uniform(0.0, 1.0, size=n)
    cost = np.zeros(n)
    np.add.at(cost, col, value * y0[rows])
    cost += s0
    return Model(num_rows=m, num_cols=n, start=start, index=rows, value=value, col_cost=cost,
                 col_lower=np.zeros(n), col_upper=np.full(n, 10.0), row_lower=row_lower,
                 row_upper=row_upper, name=name or f"random_{m}x{n}_s{seed}",
                 meta={"seed": seed, "n_eq": n_eq, "nnz_per_col": nnz_per_col,
                       "heavy_row_frac": heavy_row_frac, "heavy_nnz_frac": heavy_nnz_frac})


def config1(seed: int = 1) -> Model:
    """m=1,000 (600 =, 400 <=), n=2,000, 5 nnz/column, values N(0,1), 0<=x<=10."""
    return random_lp(1000, 2000, 5.0, 600, seed, name=f"c1_s{seed}")


def config2(seed: int = 2) -> Model:
    """m=40,000, n=80,000, 6.4 nnz/column (512k nnz); 1% of rows hold 10% of nnz."""
    return random_lp(40000, 80000, 6.4, 24000, seed, heavy_row_frac=0.01, heavy_nnz_frac=0.10,
                     name=f"c2_s{seed}")


def scaled_random_lp(m: int, seed: int, skew: bool = False) -> Model:
    """The config-1 construction at any size (n = 2m); used for parity sweeps."""
    if skew:
        return random_lp(m, 2 * m, 6.4, int(0.6 * m), seed, heavy_row_frac=0.01, heavy_nnz_frac=0.10)
    return random_lp(m, 2 * m, 5.0, int(0.6 * m), seed)


def refinery_lp(periods: int = 12, crudes: int = 6, units: int = 10, pools: int = 15, regions: int = 10,
                streams: int = 12, properties: int = 8, pools_per_stream: int = 4, seed: int = 3,
                crude_prices=None, demand_scales=None, scale_exponent: float = 3.0, name: str | None = None) -> Model:
    """Synthetic multi-period refinery-planning LP (the "C3" workload).

    Per region and period: crude feeds f[c,u] into process units, each unit
    turning its feed into `streams` intermediate streams with yields
    U(0.01, 0.6) (material-balance equalities), streams blended into product
    pools (pool balances, blending-quality <= rows with property coefficients
    U(0.5, 2.0) against specs), unit capacity rows with rhs U(1e3, 1e5),
    product sales bounded by demand U(5e2, 5e4), and stream / pool / crude
    inventories linking consecutive periods; crude purchases are shared by the
    regions.  Objective: crude cost + small operating and holding costs minus
    product revenue.  Every row and column is then rescaled by 10^U(-e, e)
    (an equivalent, badly scaled LP).  x = 0 is feasible and the LP is bounded.

    Family parameters: `crude_prices` (one per crude, default U(40, 120)) and
    `demand_scales` (multiplying the demand of the first len() pools).  meta
    holds the column indices of the crude purchases (`buy_cols`, T x C) and
    product sales (`sale_cols`, R x T x P), the demand (R x P) and the column
    scales, so that family members can be formed without rebuilding.
    Defaults give 48,072 rows, 99,144 columns and about 0.75M nonzeros.
    """
    rng = np.random.default_rng(seed)
    T, C, U, P, R, S, Q = periods, crudes, units, pools, regions, streams, properties
    yld = rng.uniform(0.01, 0.6, size=(R, C, U, S))
    cap = rng.uniform(1e3, 1e5, size=(R, U))
    supply = rng.uniform(1e3, 1e5, size=C) * R
    demand = rng.uniform(5e2, 5e4, size=(R, P))
    prop = rng.uniform(0.5, 2.0, size=(R, U, S, Q))
    spec = rng.uniform(0.8, 1.6, size=(R, P, Q))
    price = rng.uniform(150.0, 300.0, size=P)
    op_cost = rng.uniform(1.0, 5.0, size=U)
    elig = np.array([[rng.choice(P, size=pools_per_stream, replace=False) for _ in range(S)] for _ in range(U)])
    cprice = rng.uniform(40.0, 120.0, size=C)  # drawn always, so the scalings below do not depend on it
    if crude_prices is not None:
        cprice = np.asarray(crude_prices, dtype=float)
    if demand_scales is not None:
        ds = np.asarray(demand_scales, dtype=float)
        demand = demand.copy()
        demand[:, :len(ds)] *= ds

    cols = {"cost": [], "lo": [], "up": []}

    def new_cols(k, cost, up=np.inf):
        base = len(cols["cost"])
        cols["cost"].extend(np.broadcast_to(cost, (k,)).tolist())
        cols["lo"].extend([0.0] * k)
        cols["up"].extend(np.broadcast_to(up, (k,)).tolist())
        return np.arange(base, base + k)

    # column blocks
    buy = np.zeros((T, C), dtype=np.int64)
    cinv = np.zeros((T, C), dtype=np.int64)
    for t in range(T):
        buy[t] = new_cols(C, cprice, supply)
        cinv[t] = new_cols(C, 0.5)
    f = np.zeros((R, T, C, U), dtype=np.int64)
    prod = np.zeros((R, T, U, S), dtype=np.int64)
    blend = np.zeros((R, T, U, S, pools_per_stream), dtype=np.int64)
    sinv = np.zeros((R, T, U, S), dtype=np.int64)
    vol = np.zeros((R, T, P), dtype=np.int64)
    pinv = np.zeros((R, T, P), dtype=np.int64)
    sale = np.zeros((R, T, P), dtype=np.int64)
    for r in range(R):
        for t in range(T):
            f[r, t] = new_cols(C * U, np.tile(op_cost, C)).reshape(C, U)
            prod[r, t] = new_cols(U * S, 0.0).reshape(U, S)
            blend[r, t] = new_cols(U * S * pools_per_stream, 0.0).reshape(U, S, pools_per_stream)
            sinv[r, t] = new_cols(U * S, 0.2).reshape(U, S)
            vol[r, t] = new_cols(P, 0.0)
            pinv[r, t] = new_cols(P, 0.3)
            sale[r, t] = new_cols(P, -price, demand[r])
    rows_r, rows_c, rows_v, rlo, rup = [], [], [], [], []

    def add_row(cidx, vals, lo, up):
        i = len(rlo)
        rows_r.extend([i] * len(cidx))
        rows_c.extend(list(cidx))
        rows_v.extend(list(vals))
        rlo.append(lo)
        rup.append(up)

    for t in range(T):
        for c in range(C):  # crude balance: buy + inv(t-1) = feeds + inv(t)
            idx = [buy[t, c], cinv[t, c]] + list(f[:, t, c, :].ravel())
            val = [1.0, -1.0] + [-1.0] * (R * U)
            if t > 0:
                idx.append(cinv[t - 1, c])
                val.append(1.0)
            add_row(idx, val, 0.0, 0.0)
    for r in range(R):
        for t in range(T):
            for u in range(U):
                add_row(f[r, t, :, u], np.ones(C), -np.inf, cap[r, u])  # unit capacity
                for s in range(S):  # yields: prod = sum_c yld f
                    add_row([prod[r, t, u, s]] + list(f[r, t, :, u]), [1.0] + list(-yld[r, :, u, s]), 0.0, 0.0)
                    idx = [prod[r, t, u, s], sinv[r, t, u, s]] + list(blend[r, t, u, s])
                    val = [1.0, -1.0] + [-1.0] * pools_per_stream
                    if t > 0:
                        idx.append(sinv[r, t - 1, u, s])
                        val.append(1.0)
                    add_row(idx, val, 0.0, 0.0)  # stream balance with inventory
            for p in range(P):
                src = [(u, s, k) for u in range(U) for s in range(S) for k in range(pools_per_stream)
                       if elig[u, s, k] == p]
                bidx = [blend[r, t, u, s, k] for (u, s, k) in src]
                add_row(bidx + [vol[r, t, p]], [1.0] * len(bidx) + [-1.0], 0.0, 0.0)  # pool balance
                for q in range(Q):  # blending quality: sum prop b <= spec vol
                    add_row(bidx + [vol[r, t, p]], [prop[r, u, s, q] for (u, s, k) in src] + [-spec[r, p, q]],
                            -np.inf, 0.0)
                idx = [vol[r, t, p], pinv[r, t, p], sale[r, t, p]]
                val = [1.0, -1.0, -1.0]
                if t > 0:
                    idx.append(pinv[r, t - 1, p])
                    val.append(1.0)
                add_row(idx, val, 0.0, 0.0)  # pool inventory
    n, m = len(cols["cost"]), len(rlo)
    ri, ci, vv = np.array(rows_r), np.array(rows_c), np.array(rows_v)
    cost, lo, up = np.array(cols["cost"]), np.array(cols["lo"]), np.array(cols["up"])
    rl, ru = np.array(rlo), np.array(rup)
    # badly scaled equivalent LP: A' = Dr A Dc, x = Dc x'
    dr = 10.0 ** rng.uniform(-scale_exponent, scale_exponent, size=m)
    dc = 10.0 ** rng.uniform(-scale_exponent, scale_exponent, size=n)
    vv = vv * dr[ri] * dc[ci]
    cost = cost * dc
    lo = lo / dc
    up = np.where(np.isfinite(up), up / dc, np.inf)
    rl = np.where(np.isfinite(rl), rl * dr, rl)
    ru = np.where(np.isfinite(ru), ru * dr, ru)
    order = np.lexsort((ri, ci))
    ri, ci, vv = ri[order], ci[order], vv[order]
    start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(ci, minlength=n), out=start[1:])
    return Model(num_rows=m, num_cols=n, start=start, index=ri, value=vv, col_cost=cost, col_lower=lo, col_upper=up,
                 row_lower=rl, row_upper=ru, name=name or f"refinery_T{T}_R{R}_s{seed}",
                 meta={"seed": seed, "periods": T, "regions": R, "crude_prices": cprice.tolist(),
                       "buy_cols": buy, "sale_cols": sale, "demand": demand, "col_scale": dc})


def config3(seed: int = 3) -> Model:
    """The multi-period refinery-planning LP at its default size (12 periods,
    6 crudes, 10 units, 15 pools, 10 regions)."""
    return refinery_lp(seed=seed, name=f"c3_s{seed}")


def uneven_family_sizes(count: int, nnz_lo: float = 1e4, nnz_hi: float = 2e6, seed: int = 4) -> np.ndarray:
    """The nonzero counts uneven_family draws (for partitioning before building)."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(nnz_lo), np.log(nnz_hi), size=count))


def uneven_family(count: int, nnz_lo: float = 1e4, nnz_hi: float = 2e6, seed: int = 4, only=None) -> list[Model]:
    """Batched uneven workload: `count` LPs of the config-2 generator, instance i
    with seed `seed` + i and a nonzero count drawn log-uniform from
    [nnz_lo, nnz_hi] (m = nnz / 12.8 rows, n = 2m columns, 6.4 nonzeros per
    column, 1% of the rows holding 10% of the nonzeros).  `only`: build just
    these instance indices (in that order)."""
    nnz = uneven_family_sizes(count, nnz_lo, nnz_hi, seed)
    out = []
    for i in (range(count) if only is None else only):
        m = max(10, int(round(nnz[i] / 12.8)))
        out.append(random_lp(m, 2 * m, 6.4, int(0.6 * m), seed + i, heavy_row_frac=0.01, heavy_nnz_frac=0.10,
                             name=f"c4_s{seed + i}"))
    return out


# ---- the reference's per-iteration calibration instances ----------------------

_GOLDEN_GAMMA = np.uint64(0x9E3779B97F4A7C15)


def _splitmix64(seed: int, first: int, count: int) -> np.ndarray:
    """Outputs first .. first+count-1 of the SplitMix64 stream (Steele, Lea and
    Flood, 2014) started at `seed`: output i mixes seed + (i+1)*gamma with the
    published finaliser.  The reference's Rng is this generator
    (src/util/rng.h)."""
    with np.errstate(over="ignore"):
        i = np.arange(first + 1, first + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * _GOLDEN_GAMMA
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


CALIBRATION_SCALES = (1000, 4000, 16000, 64000, 256000, 1000000)


def calibration_lp(scale: int) -> Model:
    """The random transportation-like LP of the reference's PDHG per-iteration
    calibration (calibrateBandwidth, src/parametric/parametric.cpp:545-563):
    m = scale rows, n = 2 scale columns, four entries per column at rows
    below(m) with values 0.5 + uniform(), drawn in column order (row, then
    value, per entry) from one SplitMix64 stream seeded 7 that runs on across
    the scales 1e3, 4e3, 1.6e4, 6.4e4, 2.56e5, 1e6 in that order; duplicate
    entries summed (SparseMatrix::fromTriplets; a pair sums identically in
    either order, a rare triple may differ from the reference's unstable sort
    in the last bit); the costs uniform() - 0.3 are drawn after the entries;
    0 <= x <= 10; every row >= 1."""
    m, n = int(scale), 2 * int(scale)
    offset = 0
    for s in CALIBRATION_SCALES[:CALIBRATION_SCALES.index(scale)]:
        offset += 9 * 2 * s  # 8 draws per column for the entries, 1 for the cost
    draws = _splitmix64(7, offset, 8 * n)
    rows = (draws[0::2] % np.uint64(m)).astype(np.int64)
    vals = 0.5 + (draws[1::2] >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    cols = np.repeat(np.arange(n, dtype=np.int64), 4)
    order = np.lexsort((rows, cols))
    rows, cols, vals = rows[order], cols[order], vals[order]
    first = np.ones(len(rows), dtype=bool)
    first[1:] = (rows[1:] != rows[:-1]) | (cols[1:] != cols[:-1])
    group = np.cumsum(first) - 1
    merged = np.zeros(int(first.sum()))
    np.add.at(merged, group, vals)
    rows, cols = rows[first], cols[first]
    start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(cols, minlength=n), out=start[1:])
    cost = (_splitmix64(7, offset + 8 * n, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) - 0.3
    return Model(num_rows=m, num_cols=n, start=start, index=rows, value=merged, col_cost=cost,
                 col_lower=np.zeros(n), col_upper=np.full(n, 10.0), row_lower=np.ones(m),
                 row_upper=np.full(m, np.inf), name=f"calib_{scale}")
