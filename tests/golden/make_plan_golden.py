"""Regenerates the refinery-plan fixtures in plans/: the LPs of the
reference's published PDHG runs, with the figures it published for them.

The reference ships generated refinery planning models (data/gen/plan_*.mps)
and, for each, the JSON telemetry of its own solves (results/gpu/
plan_*.pdhg-{cpu,gpu}_raw1e-{4,6}.json): `pramana <mps> --algo pdhg-cpu|pdhg-gpu
--no-crossover --pdhg-tol T --json`, i.e. solve() -> presolve -> solvePdhg on
the reduced, minimisation-form LP.  For each plan this script stores

* the LP that solve() hands to solvePdhg, produced by the reference's own MPS
  reader, minimisation form and Presolver (oracle/_ref, `ref_load_mps`);
* the published telemetry of those runs: PDHG iterations and restarts, the
  relative KKT and its parts, primal weight, spectral norm, objective, and the
  rows presolve removed.

plan_60x156 is not shipped (its MPS is listed among the reference's missing
large blobs); it is regenerated here by the reference's own generator,
`gen/refinery.py planning --crudes 60 --periods 156 --seed 1`, run in this
container.  That generator's floating-point output differs from the shipped
files in the last digit of some coefficients (regenerating plan_40x104 changes
a few values by one ulp), so the plan_60x156 fixture is a model within
rounding of the published one, not bit-identical to it.

Run from the repository root, with the reference tree present:

    python tests/golden/make_plan_golden.py
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "optimized-gpu-accelerator_b200")]

from oracle import oracle as O  # noqa: E402

REF = os.environ.get("PRAMANA_REFERENCE", "/root/reference")
PLANS = ("plan_6x4", "plan_10x12", "plan_20x12", "plan_20x52", "plan_30x52", "plan_40x104", "plan_60x156")
RUNS = ("pdhg-cpu_raw1e-4", "pdhg-gpu_raw1e-4", "pdhg-gpu_raw1e-6")
FIELDS = ("iterations", "restarts", "relative_kkt", "relative_primal_residual", "relative_dual_residual",
          "relative_gap", "primal_weight", "spectral_norm_estimate", "objective", "solve_seconds", "setup_seconds")


def main():
    O.build(reference=True)
    for name in PLANS:
        path = os.path.join(REF, "data", "gen", name + ".mps")
        made = None
        if not os.path.exists(path):
            crudes, periods = name.split("_")[1].split("x")
            made = path = os.path.join(HERE, "plans", name + ".mps")
            os.makedirs(os.path.dirname(path), exist_ok=True)
            subprocess.run([sys.executable, os.path.join(REF, "gen", "refinery.py"), "planning", "--crudes", crudes,
                            "--periods", periods, "--seed", "1", "--out", path], check=True,
                           env=dict(os.environ, PYTHONDONTWRITEBYTECODE="1"))
        lp, rows_removed, cols_removed = O.load_mps(path)
        if made:
            os.remove(made)
        d = dict(num_rows=lp.num_rows, num_cols=lp.num_cols, start=lp.start, index=lp.index, value=lp.value,
                 col_cost=lp.col_cost, col_lower=lp.col_lower, col_upper=lp.col_upper, row_lower=lp.row_lower,
                 row_upper=lp.row_upper, obj_offset=lp.obj_offset)
        published = {}
        for run in RUNS:
            with open(os.path.join(REF, "results", "gpu", f"{name}.{run}.json")) as f:
                t = json.load(f)["telemetry"]
            assert t["presolve"]["rows_removed"] == rows_removed and t["presolve"]["cols_removed"] == cols_removed
            published[run] = {k: t["pdhg"][k] for k in FIELDS}
            published[run]["tolerance"] = float(run.rsplit("raw", 1)[1])
            published[run]["device"] = t["pdhg"].get("device", "")
        d["published"] = json.dumps(published)
        d["rows_removed"] = rows_removed
        os.makedirs(os.path.join(HERE, "plans"), exist_ok=True)
        np.savez_compressed(os.path.join(HERE, "plans", name + ".npz"), **d)
        print(name, lp.num_rows, lp.num_cols, len(lp.value),
              {r: (p["iterations"], p["restarts"]) for r, p in published.items()})


if __name__ == "__main__":
    main()
