"""The reference's PDHG per-iteration calibration instances
(calibrateBandwidth, src/parametric/parametric.cpp:545-563), restated by
generators.calibration_lp: every scale has the published size, duplicates
merged exactly as the reference's generator and triplet assembly merge them
(results/gpu/calibrate.json, extracted by
tests/golden/make_calibration_golden.py)."""
import json
import os

import numpy as np
import pytest

from pramana_b200 import generators as G

PUBLISHED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "calibration_published.json")


@pytest.mark.parametrize("k", range(len(G.CALIBRATION_SCALES)))
def test_calibration_instances_have_published_sizes(k):
    with open(PUBLISHED) as f:
        pub = json.load(f)["scales"][k]
    lp = G.calibration_lp(G.CALIBRATION_SCALES[k])
    assert (lp.num_rows, lp.num_cols, lp.nnz) == (pub["rows"], pub["cols"], pub["nnz"])
    assert np.all(np.diff(lp.start) <= 4) and np.all(lp.value >= 0.5)
    assert np.all(lp.col_cost >= -0.3) and np.all(lp.col_cost < 0.7)
