"""Regenerates answers.json: exact answers that the mixed-precision forms are
judged against at sizes too slow for the oracle inside a test.

* config-2 (the bench LP, seed 2): the reference's own CPU PDHG
  (oracle/_ref, all host threads) to rel KKT 1e-6 and 1e-8 -- objective,
  iterations; its 1e-8 objective stands for the optimum (the reference's
  dual simplex does not finish this 40,000 x 80,000 LP within 20 minutes
  here);
* the crude-price sweep of the large refinery family (bench.py
  --workload sweep-tol): for a sample of its cases, the exact optimum by the
  reference's dual simplex.

A pure function of the generators' seeds and the reference build; run from
the repository root in the build container (with the reference build):

    python tests/golden/make_answers_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "optimized-gpu-accelerator_b200")]

from oracle import oracle as O  # noqa: E402
from pramana_b200 import generators as G  # noqa: E402

import bench  # noqa: E402


def main():
    O.build(reference=True)
    O.set_ref_threads(os.cpu_count() or 1)
    out = {"config2": {"seed": bench.SEED}, "sweep": {}}
    lp = G.config2(bench.SEED)
    for tol in (1e-6, 1e-8):
        r = O.solve(lp, "ref", tolerance=tol)
        out["config2"][f"{tol:g}"] = {"objective": r.objective, "iterations": r.iterations,
                                      "relative_kkt": r.relative_kkt, "status": r.status}
        print("config2", tol, r.status, r.iterations, r.objective, flush=True)
    out["config2"]["exact"] = {"objective": out["config2"]["1e-08"]["objective"],
                               "source": "the reference's CPU PDHG to rel KKT 1e-8"}
    fam, params = bench.sweep_family(256)
    sample = [int(i) for i in np.linspace(0, 255, 8).round()]
    out["sweep"] = {"cases": 256, "sample": sample, "exact": []}
    for i in sample:
        e = O.simplex(fam.instance(params[i]))
        assert e["status"] == "Optimal", e
        out["sweep"]["exact"].append(e["objective"])
        print("sweep case", i, e, flush=True)
    with open(os.path.join(HERE, "answers.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
