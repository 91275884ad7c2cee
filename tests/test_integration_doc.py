"""Every C++ block shown in INTEGRATION.md, and the binding file it points to
(tests/dropin/pdhg_b200.cpp), compiles against the reference's headers and
this engine's C ABI (CPU only; skipped without the reference tree)."""
import os
import re
import subprocess

import pytest
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = os.path.join(O.REFERENCE_SRC, "src")


@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference sources not present")
def test_integration_binding_compiles(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = [b for b in re.findall(r"```cpp\n(.*?)```", text, flags=re.S) if "#include" in b]
    assert len(blocks) >= 1 and any("namespace b200" in b for b in blocks)
    assert "tests/dropin/pdhg_b200.cpp" in text
    sources = []
    for i, block in enumerate(blocks):
        src = tmp_path / f"block{i}.cpp"
        src.write_text(block)
        sources.append(src)
    sources.append(os.path.join(ROOT, "tests", "dropin", "pdhg_b200.cpp"))  # the binding file itself
    for src in sources:
        r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-include", "cstdint", f"-I{REF_SRC}",
                            f"-I{os.path.join(ROOT, 'include')}", str(src)], capture_output=True, text=True)
        assert r.returncode == 0, (str(src), r.stderr)
