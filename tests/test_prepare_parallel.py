"""The host preparation (Ruiz and Pock-Chambolle scaling, the CSR of A built
by a parallel stable counting sort, the scaled operators) gives bit-identical
results on one thread and on all host threads."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "optimized-gpu-accelerator_b200", "csrc")


def test_parallel_preparation_is_bit_identical(tmp_path):
    exe = tmp_path / "prepare_check"
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-include", "algorithm", "-include", "cmath",
           f"-I{CSRC}", os.path.join(HERE, "prepare_check.cpp"), os.path.join(CSRC, "pdhg_prepare.cpp"), "-o",
           str(exe)]
    subprocess.run(cmd, check=True)
    env = dict(os.environ, OMP_NUM_THREADS="8")
    out = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
    print(out.stdout)
    assert out.returncode == 0, out.stdout
    assert out.stdout.count("identical") == 6
