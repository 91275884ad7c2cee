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
from oracle import oracle as O

PUBLISHED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "calibration_published.json")


@pytest.mark.parametrize("k", range(len(G.CALIBRATION_SCALES)))
def test_calibration_instances_have_published_sizes(k):
    with open(PUBLISHED) as f:
        pub = json.load(f)["scales"][k]
    lp = G.calibration_lp(G.CALIBRATION_SCALES[k])
    assert (lp.num_rows, lp.num_cols, lp.nnz) == (pub["rows"], pub["cols"], pub["nnz"])
    assert np.all(np.diff(lp.start) <= 4) and np.all(lp.value >= 0.5)
    assert np.all(lp.col_cost >= -0.3) and np.all(lp.col_cost < 0.7)


REF_SRC = os.path.join(O.REFERENCE_SRC, "src")


@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference sources not present")
def test_splitmix_stream_matches_reference_rng(tmp_path):
    """The restated stream equals the reference's own Rng (src/util/rng.h,
    compiled here as the checker) draw for draw, from the start and from an
    offset, for the seeds its calibration (7) and certifier test (1) use."""
    import subprocess
    src = tmp_path / "rng.cpp"
    src.write_text('#include <cstdio>\n#include <initializer_list>\n#include "util/rng.h"\n'
                   'int main(){for(unsigned long long s : {7ull, 1ull}){'
                   'pramana::Rng r(s); for(int i = 0; i < 40; ++i) std::printf("%llu\\n", '
                   '(unsigned long long)r.next());}}\n')
    exe = tmp_path / "rng"
    subprocess.run(["g++", "-std=c++17", f"-I{REF_SRC}", str(src), "-o", str(exe)], check=True)
    ref = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    ours = [int(v) for seed in (7, 1) for v in G._splitmix64(seed, 0, 40)]
    assert ours == ref
    assert [int(v) for v in G._splitmix64(7, 25, 15)] == ref[25:40]
