"""bench.py's command line (CPU only): every workload is offered, and the
reference arm's GPU backend reports itself unavailable, rather than timing the
reference's CPU backend under the GPU's name, when no GPU comes up."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_offers_every_workload():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                         check=True).stdout
    for w in ("lp", "family", "multi", "sweep", "router", "plan", "families", "calibrate"):
        assert w in out
    assert "--reference-backend" in out


def test_bench_rejects_short_warmup():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--warmup", "1"], capture_output=True,
                       text=True)
    assert r.returncode != 0 and "warmup" in r.stderr


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_reference_gpu_arm_without_gpu_is_unavailable(oracle_mod):
    if not oracle_mod.available("ref"):
        pytest.skip("reference build absent")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--reference-backend", "gpu", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, check=True, timeout=600)
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_reference_arm_times_full_solves_of_the_same_config(oracle_mod):
    """The reference arm's line carries the engine arm's config dict verbatim,
    and its timed step is a whole solve to the tolerance, not a scaled sample."""
    if not oracle_mod.available("ref"):
        pytest.skip("reference build absent")
    sys.path.insert(0, ROOT)
    import bench
    from pramana_b200 import generators as G
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, check=True, timeout=900)
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["config"] == bench.workload_config(G.config2(bench.SEED), 1)
    assert line["run"]["relative_kkt"] <= bench.TOL
    assert line["run"]["iterations"] == bench.REF_ITERS_TO_TOL - 1
    assert line["value"] == line["cpu_baseline"]["value"] == line["e2e"]["value"]
