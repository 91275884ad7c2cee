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
