"""Small deterministic LPs for parity tests (every bound type the PDHG path
distinguishes, src/pdhg/pdhg.cpp:166-197 and 506-530)."""
import os

import numpy as np

from pramana_b200.model import LpCase, Model


def edge_lp(seed: int = 5, m: int = 40, n: int = 60) -> Model:
    """Feasible, bounded LP with boxed / lower-only / upper-only / free / fixed
    columns, = / <= / >= / ranged / free rows, one empty row and one empty
    column."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    empty_col, empty_row = n - 1, m - 1
    for j in range(n - 1):
        cnt = rng.integers(1, 5)
        rr = rng.choice(m - 1, size=cnt, replace=False)
        for r in sorted(rr):
            rows.append(r)
            cols.append(j)
            vals.append(rng.normal() * 10.0 ** rng.uniform(-1, 1))
    rows, cols, vals = np.array(rows), np.array(cols), np.array(vals)
    order = np.lexsort((rows, cols))
    rows, cols, vals = rows[order], cols[order], vals[order]
    start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(cols, minlength=n), out=start[1:])
    ctype = rng.integers(0, 5, size=n)  # 0 boxed 1 lower 2 upper 3 free 4 fixed
    ctype[empty_col] = 0
    lo = np.where(np.isin(ctype, [0, 1, 4]), rng.uniform(-5, 0, n), -np.inf)
    up = np.where(np.isin(ctype, [0, 2]), rng.uniform(1, 6, n), np.inf)
    up = np.where(ctype == 4, lo, up)
    x0 = np.where(np.isfinite(lo), lo, 0.0) + rng.uniform(0, 1, n)
    x0 = np.where(ctype == 2, up - rng.uniform(0, 1, n), x0)
    x0 = np.where(ctype == 4, lo, x0)
    x0 = np.where(ctype == 0, np.minimum(x0, up), x0)
    b = np.zeros(m)
    np.add.at(b, rows, vals * x0[cols])
    rtype = rng.integers(0, 5, size=m)  # 0 eq 1 <= 2 >= 3 ranged 4 free
    rtype[empty_row] = 0
    s = rng.uniform(0.1, 1.0, m)
    rl = np.select([rtype == 0, rtype == 1, rtype == 2, rtype == 3], [b, -np.inf, b - s, b - s], -np.inf)
    ru = np.select([rtype == 0, rtype == 1, rtype == 2, rtype == 3], [b, b + s, np.inf, b + s], np.inf)
    y0 = rng.normal(size=m)
    y0 = np.select([rtype == 1, rtype == 2, rtype == 4], [-np.abs(y0), np.abs(y0), 0.0], y0)
    z = rng.uniform(0, 1, n)
    z = np.select([ctype == 1, ctype == 2, ctype == 3], [z, -z, 0.0], rng.normal(size=n))
    c = np.zeros(n)
    np.add.at(c, cols, vals * y0[rows])
    c += z
    return Model(num_rows=m, num_cols=n, start=start, index=rows, value=vals, col_cost=c, col_lower=lo,
                 col_upper=up, row_lower=rl, row_upper=ru, obj_offset=1.25, name=f"edge_s{seed}")


def cost_sweep_cases(lp: Model, k: int, col: int = 1, step: float = 0.1):
    """k cases that vary one cost entry, as the reference's batch test does
    (tests/cpp/test_solvers.cpp:132-149)."""
    out = []
    for q in range(k):
        c = lp.col_cost.copy()
        c[col] = lp.col_cost[col] - 0.4 + step * q
        out.append(LpCase(cost=c))
    return out


def mixed_cases(lp: Model, k: int, seed: int = 3):
    """k cases overriding cost, column bounds and row bounds (some left as base)."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(k):
        cs = LpCase()
        if q % 2 == 0:
            cs.cost = lp.col_cost * rng.uniform(0.8, 1.2, lp.num_cols)
        if q % 3 == 1:
            cs.col_upper = np.where(np.isfinite(lp.col_upper), lp.col_upper * 1.1, lp.col_upper)
        if q % 4 == 2:
            cs.row_upper = np.where(np.isfinite(lp.row_upper), lp.row_upper + 0.5, lp.row_upper)
            cs.row_lower = lp.row_lower.copy()
        out.append(cs)
    return out


def read_mps(path: str) -> Model:
    """Minimal fixed/free MPS reader for the reference's Netlib pins (CPU tests
    only): ROWS/COLUMNS/RHS/RANGES/BOUNDS, objective row N, default bounds
    [0, inf)."""
    import gzip
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rt") as f:
        lines = f.read().splitlines()
    section = None
    row_type, row_order, obj = {}, [], None
    col_order, col_index = [], {}
    entries = {}
    rhs, ranges, bounds = {}, {}, []
    for ln in lines:
        if not ln.strip() or ln.startswith("*"):
            continue
        if not ln[0].isspace():
            section = ln.split()[0]
            continue
        tok = ln.split()
        if section == "ROWS":
            t, name = tok[0], tok[1]
            if t == "N":
                if obj is None:
                    obj = name
                continue
            row_type[name] = t
            row_order.append(name)
        elif section == "COLUMNS":
            if "MARKER" in tok:
                continue
            cname = tok[0]
            if cname not in col_index:
                col_index[cname] = len(col_order)
                col_order.append(cname)
            for q in range(1, len(tok) - 1, 2):
                entries[(tok[q], cname)] = entries.get((tok[q], cname), 0.0) + float(tok[q + 1])
        elif section == "RHS":
            body = tok[1:] if len(tok) % 2 == 1 else tok
            for q in range(0, len(body) - 1, 2):
                rhs[body[q]] = float(body[q + 1])
        elif section == "RANGES":
            body = tok[1:] if len(tok) % 2 == 1 else tok
            for q in range(0, len(body) - 1, 2):
                ranges[body[q]] = float(body[q + 1])
        elif section == "BOUNDS":
            bt = tok[0]
            if bt in ("FR", "MI", "PL", "BV"):
                bounds.append((bt, tok[2] if len(tok) > 2 else tok[1], None))
            else:
                bounds.append((bt, tok[2], float(tok[3])))
    m, n = len(row_order), len(col_order)
    ridx = {r: i for i, r in enumerate(row_order)}
    c = np.zeros(n)
    rr, cc, vv = [], [], []
    for (r, cn), v in entries.items():
        if r == obj:
            c[col_index[cn]] += v
        elif v != 0.0:
            rr.append(ridx[r])
            cc.append(col_index[cn])
            vv.append(v)
    rr, cc, vv = np.array(rr, dtype=np.int64), np.array(cc, dtype=np.int64), np.array(vv)
    order = np.lexsort((rr, cc))
    rr, cc, vv = rr[order], cc[order], vv[order]
    start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(cc, minlength=n), out=start[1:])
    rl, ru = np.full(m, -np.inf), np.full(m, np.inf)
    for name, i in ridx.items():
        t, b = row_type[name], rhs.get(name, 0.0)
        if t == "E":
            rl[i] = ru[i] = b
            if name in ranges:
                r = ranges[name]
                if r > 0:
                    ru[i] = b + abs(r)
                else:
                    rl[i] = b - abs(r)
        elif t == "L":
            ru[i] = b
            if name in ranges:
                rl[i] = b - abs(ranges[name])
        elif t == "G":
            rl[i] = b
            if name in ranges:
                ru[i] = b + abs(ranges[name])
    lo, up = np.zeros(n), np.full(n, np.inf)
    for bt, cn, v in bounds:
        j = col_index[cn]
        if bt == "UP":
            up[j] = v
            if v < 0 and lo[j] == 0:
                lo[j] = -np.inf
        elif bt == "LO":
            lo[j] = v
        elif bt == "FX":
            lo[j] = up[j] = v
        elif bt == "FR":
            lo[j], up[j] = -np.inf, np.inf
        elif bt == "MI":
            lo[j] = -np.inf
        elif bt == "PL":
            up[j] = np.inf
    offset = -rhs.get(obj, 0.0) if obj else 0.0
    return Model(num_rows=m, num_cols=n, start=start, index=rr, value=vv, col_cost=c, col_lower=lo, col_upper=up,
                 row_lower=rl, row_upper=ru, obj_offset=offset, name=path)


GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PLANS = ("plan_6x4", "plan_10x12", "plan_20x12", "plan_20x52", "plan_30x52", "plan_40x104", "plan_60x156")


def load_plan(name: str):
    """A refinery planning LP of the reference's published PDHG runs, as
    solve() hands it to solvePdhg (presolved, minimisation form), and the
    published telemetry of those runs keyed by run ("pdhg-cpu_raw1e-4",
    "pdhg-gpu_raw1e-4", "pdhg-gpu_raw1e-6"); fixtures made by
    tests/golden/make_plan_golden.py."""
    import json
    d = np.load(os.path.join(GOLDEN_DIR, "plans", name + ".npz"))
    lp = Model(num_rows=int(d["num_rows"]), num_cols=int(d["num_cols"]), start=d["start"], index=d["index"],
               value=d["value"], col_cost=d["col_cost"], col_lower=d["col_lower"], col_upper=d["col_upper"],
               row_lower=d["row_lower"], row_upper=d["row_upper"], obj_offset=float(d["obj_offset"]), name=name)
    return lp, json.loads(str(d["published"]))


FAMILIES = ("plan_10x12_BUY_CR03_0_cost", "plan_10x12_BUY_CR03_0_upper", "plan_20x12_BUY_CR07_3_cost",
            "plan_20x52_BUY_CR05_10_upper")


def load_family(name: str):
    """The batched-PDHG leg of the reference's published repeated-solve
    experiment (compareFamilyStrategies, src/parametric/parametric.cpp:483-527):
    the model in minimisation form without presolve, its K cases (one column's
    cost or upper bound set to each theta, withParameter + toMinimization,
    :77-98), the exact optimum of every case and the published figures;
    fixtures made by tests/golden/make_family_golden.py."""
    import json
    d = np.load(os.path.join(GOLDEN_DIR, "families", name + ".npz"))
    lp = Model(num_rows=int(d["num_rows"]), num_cols=int(d["num_cols"]), start=d["start"], index=d["index"],
               value=d["value"], col_cost=d["col_cost"], col_lower=d["col_lower"], col_upper=d["col_upper"],
               row_lower=d["row_lower"], row_upper=d["row_upper"], obj_offset=float(d["obj_offset"]), name=name)
    col, kind, was_max = int(d["column"]), str(d["kind"]), bool(d["was_max"])
    cases = []
    for th in d["thetas"]:
        if kind == "cost":
            c = lp.col_cost.copy()
            c[col] = -th if was_max else th
            cases.append(LpCase(cost=c))
        else:
            u = lp.col_upper.copy()
            u[col] = th
            cases.append(LpCase(col_upper=u))
    return lp, cases, np.asarray(d["exact_objective"]), json.loads(str(d["published"]))


def family_certified(lp, cases, results, safe_bound, implied_bounds):
    """The reference's count of certified cases (parametric.cpp:508-523): the
    outward-rounded dual bound over constraint-implied column bounds, from the
    case's row duals, within 1e-4 of its objective.  `safe_bound` and
    `implied_bounds` are the engine's batched entries."""
    lo, up = implied_bounds(lp, cases)
    ok = [r.status == "Optimal" for r in results]
    cc = []
    for b, cs in enumerate(cases):
        cc.append(LpCase(cost=cs.cost, col_lower=lo[b], col_upper=up[b], row_lower=cs.row_lower,
                         row_upper=cs.row_upper))
    y = np.concatenate([r.rowDual for r in results])
    sb = safe_bound(lp, y, cc)
    n = 0
    for r, s, good in zip(results, sb, ok):
        lb = s["bound"] + lp.obj_offset
        if good and np.isfinite(s["bound"]) and abs(r.objective - lb) <= 1e-4 * (1 + abs(r.objective)):
            n += 1
    return n
