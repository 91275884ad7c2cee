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
