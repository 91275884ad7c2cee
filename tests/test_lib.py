"""CPU checks of the C-ABI library: it loads, exports every symbol that
the headers under include/ declare, validates its inputs, and fails loudly (no CPU
fallback) when no sm_100 device is present.  No kernel runs here."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

from pramana_b200 import _lib, generators as G
from pramana_b200.pdhg import PdhgOptions, _lp_struct

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
HEADERS = [os.path.join(INCLUDE, h) for h in sorted(os.listdir(INCLUDE)) if h.endswith(".h")]


def declared_symbols():
    text = "\n".join(open(h).read() for h in HEADERS)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b2p_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(engine_lib):
    syms = declared_symbols()
    assert set(syms) == set(_lib.SIGNATURES)
    for s in syms:
        assert hasattr(engine_lib, s), s
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"


def test_default_options_mirror_reference(engine_lib):
    o = _lib.B2pOptions()
    engine_lib.b2p_default_options(C.byref(o))
    # src/pdhg/pdhg.h:32-42
    assert o.tolerance == 1e-6 and o.max_iterations == 1000000 and o.check_every == 64
    assert o.ruiz_iterations == 10 and o.pock_chambolle == 1 and o.rescale_objective_and_bounds == 1
    assert o.reflection == 1.0 and o.log_interval == 0 and o.use_graphs == 1


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


def test_invalid_model_is_rejected(engine_lib):
    lp = G.random_lp(20, 40, 3.0, 10, 1)
    s, keep = _lp_struct(lp)
    bad = lp.index.copy()
    bad[3] = lp.num_rows + 7
    s.index = bad.ctypes.data_as(_lib.iptr)
    o = PdhgOptions().to_c()
    res = (_lib.B2pResult * 1)()
    st = _lib.B2pStats()
    rc = engine_lib.b2p_solve_pdhg(C.byref(s), C.byref(o), None, None, res, C.byref(st))
    assert rc == 1
    assert b"out of range" in engine_lib.b2p_last_error()
    o.check_every = 0
    s.index = lp.index.ctypes.data_as(_lib.iptr)
    assert engine_lib.b2p_solve_pdhg(C.byref(s), C.byref(o), None, None, res, C.byref(st)) == 1


@pytest.mark.skipif(_gpu_present(), reason="checks the no-device path")
def test_no_device_fails_loudly(engine_lib):
    from pramana_b200 import pdhg
    assert engine_lib.b2p_gpu_available() == 0
    info = pdhg.gpuInfoJson()
    assert info["available"] is False and info["reason"]
    with pytest.raises(_lib.B2pError) as e:
        pdhg.solvePdhg(G.random_lp(20, 40, 3.0, 10, 1))
    assert e.value.code == 3
    x = np.ones(4)
    with pytest.raises(_lib.B2pError):
        pdhg.csr_spmv(np.array([0, 1, 2]), np.array([0, 1]), np.array([1.0, 2.0]), x, 2, 4)


def test_cpu_backend_is_refused():
    with pytest.raises(ValueError):
        PdhgOptions(useGpu=False).to_c()


def test_info_json_is_valid(engine_lib):
    need = engine_lib.b2p_gpu_info_json(None, 0)
    buf = C.create_string_buffer(need + 1)
    engine_lib.b2p_gpu_info_json(buf, need + 1)
    d = json.loads(buf.value.decode())
    assert {"available", "name", "reason", "compute_capability", "multiprocessors"} <= set(d)


def test_host_side_argument_checks():
    """Wrong-length case vectors, duals and points are refused on the host,
    before any device work."""
    from pramana_b200 import pdhg
    from pramana_b200.model import LpCase
    lp = G.random_lp(20, 40, 3.0, 10, 1)
    with pytest.raises(ValueError):
        pdhg.solvePdhgBatch(lp, [LpCase(cost=np.ones(lp.num_cols - 1))])
    with pytest.raises(ValueError):
        pdhg.safeDualBound(lp, np.zeros(lp.num_rows + 1))
    with pytest.raises(ValueError):
        pdhg.certifyLp(lp, np.zeros(lp.num_cols), np.zeros(lp.num_rows - 1))
    with pytest.raises(ValueError):
        pdhg.kktResidual(lp, np.zeros(lp.num_cols + 2), np.zeros(lp.num_rows))
