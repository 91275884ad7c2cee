"""The C++ binding shown in INTEGRATION.md compiles against the reference's
headers and this engine's C ABI (CPU only; skipped without the reference tree)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = "/root/reference/src"


@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference sources not present")
def test_integration_binding_compiles(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    shim = next(b for b in blocks if "namespace b200" in b)
    src = tmp_path / "pdhg_b200.cpp"
    src.write_text(shim)
    r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-include", "cstdint", f"-I{REF_SRC}",
                        f"-I{os.path.join(ROOT, 'include')}", str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
