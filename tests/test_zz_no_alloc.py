"""The allocation-free KKT entry point, b2p_kkt_residual_noalloc.

It serves callers that cannot allocate device memory themselves (a host
framework that owns every device byte through its own pool, or a path where
allocation is forbidden): every
array is a device pointer they own, and the entry point's only scratch is a
fixed device array inside the library.  Its result must equal that of the
allocating entry point b2p_kkt_residual on the same points, call after call,
although the scratch keeps the previous call's contents.

Collected last on purpose (file name), and self-contained: it passes alone in
a fresh process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import lp_cases
from pramana_b200 import _lib
from pramana_b200 import generators as G
from pramana_b200 import pdhg
from pramana_b200.model import LpCase

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9  # the tolerance of the parity tests
MAX_POINTS = 32


def _device_inputs(torch, lp, x, y, cases):
    """Device copies of everything the no-allocation entry reads (allocated here, by the caller)."""
    k = len(cases) if cases else 1
    ptr, idx, val = lp.csr()

    def per_point(field, base):
        rows = []
        for b in range(k):
            v = getattr(cases[b], field) if cases else None
            rows.append(base if v is None else v)
        return np.concatenate(rows)

    host = {
        "a_ptr": ptr, "a_idx": idx, "a_val": val,
        "at_ptr": lp.start, "at_idx": lp.index, "at_val": lp.value,
        "cost": per_point("cost", lp.col_cost), "col_lower": per_point("col_lower", lp.col_lower),
        "col_upper": per_point("col_upper", lp.col_upper), "row_lower": per_point("row_lower", lp.row_lower),
        "row_upper": per_point("row_upper", lp.row_upper), "x": np.asarray(x), "row_dual": np.asarray(y),
    }
    dev = {k_: torch.from_numpy(np.ascontiguousarray(v)).to("cuda") for k_, v in host.items()}
    dev["out"] = torch.full((k * 4,), float("nan"), dtype=torch.float64, device="cuda")
    return dev, k


def _call(lib, lp, dev, k):
    p = lambda name: C.c_void_p(dev[name].data_ptr())  # noqa: E731
    return lib.b2p_kkt_residual_noalloc(lp.num_rows, lp.num_cols, k, p("a_ptr"), p("a_idx"), p("a_val"), p("at_ptr"),
                                        p("at_idx"), p("at_val"), p("cost"), p("col_lower"), p("col_upper"),
                                        p("row_lower"), p("row_upper"), p("x"), p("row_dual"), p("out"), None)


def _problems():
    c1 = G.config1(1)
    r1 = pdhg.solvePdhg(c1, pdhg.PdhgOptions(tolerance=1e-4))
    small = G.random_lp(150, 300, 4.0, 90, 13)
    cases = lp_cases.mixed_cases(small, 5)
    rb = pdhg.solvePdhgBatch(small, cases, pdhg.PdhgOptions(tolerance=1e-5))
    edge = lp_cases.edge_lp(7)
    rng = np.random.default_rng(0)
    xe, ye = rng.normal(size=edge.num_cols), rng.normal(size=edge.num_rows)  # an arbitrary point
    return [
        (c1, r1.x, r1.rowDual, None),
        (small, np.concatenate([r.x for r in rb]), np.concatenate([r.rowDual for r in rb]), cases),
        (edge, xe, ye, None),
    ]


def test_no_alloc_matches_allocating_entry_call_after_call():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    problems = _problems()
    expected = [pdhg.kktResidual(lp, x, y, cases).reshape(-1) for lp, x, y, cases in problems]
    devs = [_device_inputs(torch, lp, x, y, cases) for lp, x, y, cases in problems]
    torch.cuda.synchronize()
    free_before = None
    # Two rounds over three different problems: every call follows one that
    # left other contents (and another size) in the shared scratch.
    for rnd in range(2):
        for (lp, _, _, _), (dev, k), want in zip(problems, devs, expected):
            dev["out"].fill_(float("nan"))
            rc = _call(lib, lp, dev, k)
            assert rc == 0, lib.b2p_last_error()
            torch.cuda.synchronize()
            got = dev["out"].cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.allclose(got, want, rtol=REL_TOL, atol=1e-300), (got, want)
            if free_before is None:
                free_before = torch.cuda.mem_get_info()[0]
    # after the first call (which looked the scratch address up) no call changed free device memory
    assert torch.cuda.mem_get_info()[0] == free_before


def test_no_alloc_rejects_more_points_than_its_scratch_holds():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    lp = G.random_lp(40, 80, 3.0, 20, 3)
    k = MAX_POINTS + 1
    cases = [LpCase() for _ in range(k)]
    x = np.zeros(k * lp.num_cols)
    y = np.zeros(k * lp.num_rows)
    dev, kk = _device_inputs(torch, lp, x, y, cases)
    assert kk == k
    rc = _call(lib, lp, dev, k)
    assert rc == 5  # B2P_ERR_TOO_LARGE
    assert b"maximum of 32 points" in lib.b2p_last_error()
    # at the maximum it works
    dev32, _ = _device_inputs(torch, lp, x[:MAX_POINTS * lp.num_cols], y[:MAX_POINTS * lp.num_rows],
                              cases[:MAX_POINTS])
    assert _call(lib, lp, dev32, MAX_POINTS) == 0, lib.b2p_last_error()
    torch.cuda.synchronize()
    want = pdhg.kktResidual(lp, x[:MAX_POINTS * lp.num_cols], y[:MAX_POINTS * lp.num_rows],
                            cases[:MAX_POINTS]).reshape(-1)
    assert np.allclose(dev32["out"].cpu().numpy(), want, rtol=REL_TOL, atol=1e-300)


ARGS = ("a_ptr", "a_idx", "a_val", "at_ptr", "at_idx", "at_val", "cost", "col_lower", "col_upper", "row_lower",
        "row_upper", "x", "row_dual", "out")


@pytest.mark.parametrize("which", ARGS)
def test_no_alloc_rejects_a_host_pointer_in_any_position(which):
    """Every array is checked on the host before anything is launched: a host
    pointer in any one position is refused with B2P_ERR_INVALID, and the
    device output is left untouched."""
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    lp = G.random_lp(40, 80, 3.0, 20, 3)
    dev, k = _device_inputs(torch, lp, np.zeros(lp.num_cols), np.zeros(lp.num_rows), None)
    torch.cuda.synchronize()
    host = np.zeros(max(lp.num_rows, lp.num_cols, lp.start[-1]) * 4 + 8)
    ptrs = [C.c_void_p(host.ctypes.data) if name == which else C.c_void_p(dev[name].data_ptr()) for name in ARGS]
    rc = lib.b2p_kkt_residual_noalloc(lp.num_rows, lp.num_cols, k, *ptrs, None)
    assert rc == 1, lib.b2p_last_error()
    msg = lib.b2p_last_error()
    assert which.encode() in msg and b"not a device pointer" in msg
    torch.cuda.synchronize()
    assert np.all(np.isnan(dev["out"].cpu().numpy()))
