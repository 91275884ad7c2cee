"""PDHG -> simplex crossover handoff: the engine's (x, y) at relative KKT
1e-6, handed unchanged to the reference's own crossover (src/lp/crossover.cpp,
built into oracle/_ref), finishes at the simplex optimum -- the same objective
as the reference's dual simplex from scratch -- in no more pivots than that
cold solve needs."""
import numpy as np
import pytest

import lp_cases
from pramana_b200 import generators as G
from pramana_b200 import pdhg

pytestmark = pytest.mark.gpu


def _refinery():
    from pramana_b200 import warmstart as W
    fam = W.RefineryFamily(seed=5, periods=2, regions=1, units=4, streams=4, properties=2, scale_exponent=0.0)
    return fam.instance(fam.sample(1, 21)[0])


@pytest.mark.parametrize("which", ["c1", "edge", "random", "refinery"])
def test_crossover_from_engine_point(oracle_mod, which):
    lp = {"c1": lambda: G.config1(1), "edge": lambda: lp_cases.edge_lp(5),
          "random": lambda: G.random_lp(300, 600, 5.0, 180, 31), "refinery": _refinery}[which]()
    r = pdhg.solvePdhg(lp, pdhg.PdhgOptions(tolerance=1e-6, maxIterations=400000))
    assert r.status == "Optimal"
    cold = oracle_mod.simplex(lp)
    warm = oracle_mod.simplex(lp, r.x, r.rowDual)
    assert cold["status"] == warm["status"] == "Optimal"
    assert abs(warm["objective"] - cold["objective"]) <= 1e-9 * (1 + abs(cold["objective"]))
    assert warm["iterations"] <= cold["iterations"]
    print(f"{which}: crossover {warm['iterations']} pivots, simplex from scratch {cold['iterations']}")
