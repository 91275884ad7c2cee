"""Regenerates the Netlib fixtures in netlib/: the two LPs of the reference's
own GPU-path tests (tests/cpp/test_solvers.cpp:112-149), SC50A and AFIRO, as
its `netlib()` helper hands them to solvePdhg (the reference's MPS reader,
minimisation form, no presolve; oracle/_ref), with the reference CPU PDHG's
iteration count and objective at tolerance 1e-7 for SC50A and the dual-simplex
optimum of each of AFIRO's four cost cases (cost[1] = -0.4 + 0.1 k).

Run from the repository root, with the reference tree present:

    python tests/golden/make_netlib_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "optimized-gpu-accelerator_b200")]

from oracle import oracle as O  # noqa: E402
from pramana_b200.model import Model  # noqa: E402

REF = os.environ.get("PRAMANA_REFERENCE", "/root/reference")


def arrays(lp):
    return dict(num_rows=lp.num_rows, num_cols=lp.num_cols, start=lp.start, index=lp.index, value=lp.value,
                col_cost=lp.col_cost, col_lower=lp.col_lower, col_upper=lp.col_upper, row_lower=lp.row_lower,
                row_upper=lp.row_upper, obj_offset=lp.obj_offset)


def main():
    O.build(reference=True)
    os.makedirs(os.path.join(HERE, "netlib"), exist_ok=True)
    sc, _, _ = O.load_mps(os.path.join(REF, "data", "netlib", "sc50a.mps.gz"), presolve=False)
    r = O.solve(sc, "ref", tolerance=1e-7)
    assert r.status == 1
    np.savez_compressed(os.path.join(HERE, "netlib", "sc50a.npz"), **arrays(sc), ref_iterations=r.iterations,
                        ref_objective=r.objective)
    print("sc50a", sc.num_rows, sc.num_cols, r.iterations, r.objective)
    af, _, _ = O.load_mps(os.path.join(REF, "data", "netlib", "afiro.mps.gz"), presolve=False)
    optima = []
    for k in range(4):
        c = af.col_cost.copy()
        c[1] = -0.4 + 0.1 * k
        case = Model(num_rows=af.num_rows, num_cols=af.num_cols, start=af.start, index=af.index, value=af.value,
                     col_cost=c, col_lower=af.col_lower, col_upper=af.col_upper, row_lower=af.row_lower,
                     row_upper=af.row_upper, obj_offset=af.obj_offset)
        s = O.simplex(case)
        assert s["status"] == "Optimal"
        optima.append(s["objective"])
    np.savez_compressed(os.path.join(HERE, "netlib", "afiro.npz"), **arrays(af), case_optima=np.array(optima))
    print("afiro", af.num_rows, af.num_cols, optima)


if __name__ == "__main__":
    main()
