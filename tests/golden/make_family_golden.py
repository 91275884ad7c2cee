"""Regenerates the parametric-family fixtures in families/: the batched-PDHG
leg of the reference's published repeated-solve experiment.

The reference's `compareFamilyStrategies` (src/parametric/parametric.cpp:400-527)
solves K cases of one planning model, each with one column's cost or upper
bound set to theta_k = from + (to - from) k / (K - 1), by one solvePdhgBatch
call (tolerance 1e-6, at most 200,000 iterations) over the model in
minimisation form, without presolve, and counts a case as certified when the
outward-rounded dual bound over constraint-implied column bounds lies within
1e-4 of its objective.  Its published results are results/family/*.json.

For each published family this script stores the model as that code sees it
(the reference's MPS reader and minimisation form, oracle/_ref), the column,
the kind and the thetas, the published batched-PDHG figures (iterations of the
batch, cases solved and certified, largest relative objective error, seconds),
and the exact optimum of every case by the reference's dual simplex, the
reference values of that error.

Run from the repository root, with the reference tree present:

    python tests/golden/make_family_golden.py
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "optimized-gpu-accelerator_b200")]

from oracle import oracle as O  # noqa: E402
from pramana_b200.model import Model  # noqa: E402

REF = os.environ.get("PRAMANA_REFERENCE", "/root/reference")
FAMILIES = ("plan_10x12_BUY_CR03_0_cost", "plan_10x12_BUY_CR03_0_upper", "plan_20x12_BUY_CR07_3_cost",
            "plan_20x52_BUY_CR05_10_upper")


def strategy(res, name):
    s = next(s for s in res["strategies"] if s["strategy"] == name)
    it = re.search(r"(\d+) iterations", s["note"])
    return {"seconds": s["seconds"], "solved": s["solved"], "certified": s["certified"],
            "max_relative_error": s["max_relative_error"], "iterations": int(it.group(1)) if it else None,
            "note": s["note"]}


def case_model(lp, col, kind, theta, was_max):
    c, up = lp.col_cost.copy(), lp.col_upper.copy()
    if kind == "cost":
        c[col] = -theta if was_max else theta
    else:
        up[col] = theta
    return Model(num_rows=lp.num_rows, num_cols=lp.num_cols, start=lp.start, index=lp.index, value=lp.value,
                 col_cost=c, col_lower=lp.col_lower, col_upper=up, row_lower=lp.row_lower, row_upper=lp.row_upper,
                 obj_offset=lp.obj_offset)


def main():
    O.build(reference=True)
    os.makedirs(os.path.join(HERE, "families"), exist_ok=True)
    for fam in FAMILIES:
        plan, rest = fam.split("_BUY_")
        column, kind = "BUY_" + rest.rsplit("_", 1)[0], rest.rsplit("_", 1)[1]
        with open(os.path.join(REF, "results", "family", fam + ".json")) as f:
            res = json.load(f)
        lp, _, _ = O.load_mps(os.path.join(REF, "data", "gen", plan + ".mps"), presolve=False)
        col, was_max = O.loaded_column(column)
        assert col >= 0
        thetas = np.array(res["thetas"], dtype=np.float64)
        gpu = strategy(res, "batched PDHG (GPU) 1e-6 + safe bounds")
        cpu = strategy(res, "batched PDHG (CPU) 1e-6 + safe bounds")
        exact = np.full(len(thetas), np.nan)
        if gpu["solved"] > 0:
            for k, th in enumerate(thetas):
                r = O.simplex(case_model(lp, col, kind, th, was_max))
                assert r["status"] == "Optimal", r
                exact[k] = r["objective"]
        np.savez_compressed(
            os.path.join(HERE, "families", fam + ".npz"),
            num_rows=lp.num_rows, num_cols=lp.num_cols, start=lp.start, index=lp.index, value=lp.value,
            col_cost=lp.col_cost, col_lower=lp.col_lower, col_upper=lp.col_upper, row_lower=lp.row_lower,
            row_upper=lp.row_upper, obj_offset=lp.obj_offset, column=col, kind=kind, was_max=was_max,
            thetas=thetas, exact_objective=exact,
            published=json.dumps({"gpu": gpu, "cpu": cpu, "device": res.get("device", "")}))
        print(fam, lp.num_rows, lp.num_cols, len(lp.value), "col", col, kind, "K", len(thetas),
              "published GPU", gpu["iterations"], gpu["solved"], gpu["certified"], gpu["seconds"])


if __name__ == "__main__":
    main()
