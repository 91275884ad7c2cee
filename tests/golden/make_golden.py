"""Regenerates the golden PDHG fixtures in this folder from the REFERENCE's own
CPU PDHG (oracle/_ref/libpramana_ref.so, i.e. src/pdhg/pdhg.cpp CpuBackend
compiled from the reference sources).

Each .npz holds the LP (CSC + bounds), the options, and the reference's
x, row duals, status, iterations, objective, dual objective and relative KKT.
Run from the repository root, with the reference tree present:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "optimized-gpu-accelerator_b200"), os.path.join(ROOT, "tests")]

from oracle import oracle as O  # noqa: E402
from pramana_b200 import generators as G  # noqa: E402
import lp_cases  # noqa: E402


def save(name, lp, results, opts, cases=None):
    d = dict(num_rows=lp.num_rows, num_cols=lp.num_cols, start=lp.start, index=lp.index, value=lp.value,
             col_cost=lp.col_cost, col_lower=lp.col_lower, col_upper=lp.col_upper, row_lower=lp.row_lower,
             row_upper=lp.row_upper, obj_offset=lp.obj_offset, tolerance=opts["tolerance"],
             max_iterations=opts["max_iterations"])
    rs = results if isinstance(results, list) else [results]
    d["status"] = np.array([r.status for r in rs])
    d["iterations"] = np.array([r.iterations for r in rs])
    d["objective"] = np.array([r.objective for r in rs])
    d["dual_objective"] = np.array([r.dual_objective for r in rs])
    d["relative_kkt"] = np.array([r.relative_kkt for r in rs])
    d["x"] = np.stack([r.x for r in rs])
    d["y"] = np.stack([r.y for r in rs])
    d["batch"] = cases is not None
    if cases is not None:
        d["case_cost"] = np.stack([c.cost if c.cost is not None else lp.col_cost for c in cases])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
    print(name, [(r.status, r.iterations, r.relative_kkt) for r in rs])


def main():
    O.build(reference=True)
    c1 = G.config1(1)
    for iters in (1, 64, 1000):
        o = dict(tolerance=1e-30, max_iterations=iters)
        save(f"c1_s1_it{iters}", c1, O.solve(c1, "ref", **o), o)
    o = dict(tolerance=1e-4, max_iterations=100000)
    save("c1_s1_tol1e-4", c1, O.solve(c1, "ref", **o), o)
    e = lp_cases.edge_lp(5)
    o = dict(tolerance=1e-30, max_iterations=1000)
    save("edge_s5_it1000", e, O.solve(e, "ref", **o), o)
    o = dict(tolerance=1e-6, max_iterations=200000)
    save("edge_s5_tol1e-6", e, O.solve(e, "ref", **o), o)
    small = G.random_lp(120, 240, 4.0, 70, 21)
    cases = lp_cases.cost_sweep_cases(small, 4)
    o = dict(tolerance=1e-6, max_iterations=200000)
    save("batch_small_k4_tol1e-6", small, O.solve(small, "ref", cases=cases, **o), o, cases)


if __name__ == "__main__":
    main()
