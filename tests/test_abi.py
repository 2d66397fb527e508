"""The C-ABI library loads, exports every entry point the public header
declares, and rejects bad arguments with status codes (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import pytest

import cubesphere_b200 as cs

HEADER = Path(__file__).resolve().parent.parent / "include" / "cubesphere_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\*)\s+(cs_\w+)\s*\(", text, re.M)))


def test_header_declares_what_the_binding_lists():
    assert set(declared()) == set(cs.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = cs.load_library()
    for name in declared():
        assert hasattr(lib, name), name


def test_params_check_rejects_bad_sizes():
    bad = cs.make_params(ntp=2, nr=1, nghost=3)
    assert cs.load_library().cs_params_check(ctypes.byref(bad)).decode() != ""
    with pytest.raises(cs.CsError):
        cs.Solve(bad)
    with pytest.raises(cs.CsError):
        cs.Solve(ntp=16, nr=4, nghost=4, rk_scheme=7)


def test_p2_needs_the_resident_stencil_operators():
    """CS_FLAG_P2 has no in-stage rebuild of its stencil inverses, so it is
    refused together with CS_FLAG_NO_OP_CACHE and accepted alone."""
    lib = cs.load_library()
    bad = cs.make_params(ntp=16, nr=4, flags=cs.CS_FLAG_P2 | cs.CS_FLAG_NO_OP_CACHE)
    assert "CS_FLAG_P2" in lib.cs_params_check(ctypes.byref(bad)).decode()
    with pytest.raises(cs.CsError):
        cs.Solve(bad)
    assert lib.cs_params_check(ctypes.byref(cs.make_params(ntp=16, nr=4, flags=cs.CS_FLAG_P2))).decode() == ""


def test_panel_average_needs_the_shared_copies():
    """CS_FLAG_PANEL_AVERAGE is a rule for the shared copies: refused with
    CS_FLAG_NO_PANEL_SYNC, which leaves them alone, and accepted alone."""
    lib = cs.load_library()
    bad = cs.make_params(ntp=16, nr=4, flags=cs.CS_FLAG_PANEL_AVERAGE | cs.CS_FLAG_NO_PANEL_SYNC)
    assert "CS_FLAG_PANEL_AVERAGE" in lib.cs_params_check(ctypes.byref(bad)).decode()
    with pytest.raises(cs.CsError):
        cs.Solve(bad)
    ok = cs.make_params(ntp=16, nr=4, flags=cs.CS_FLAG_PANEL_AVERAGE)
    assert lib.cs_params_check(ctypes.byref(ok)).decode() == ""


def test_calls_out_of_order_return_state_errors():
    s = cs.Solve(ntp=8, nr=2, nghost=3)
    lib = s.lib
    assert lib.cs_stage(s.h, 1, 1e-3) == 3  # CS_ERR_STATE: no mesh
    assert lib.cs_fill_ghosts(s.h) == 3
    out = ctypes.c_double()
    assert lib.cs_step(s.h, 1e-3, ctypes.byref(out)) == 3
    assert "mesh" in lib.cs_last_error(s.h).decode()


def test_geometry_getter_checks_buffer_size():
    s = cs.Solve(ntp=8, nr=2, nghost=3)
    s.mesh_build(device=False)
    import numpy as np
    buf = np.zeros(5)
    rc = s.lib.cs_geometry_get(s.h, 0, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), buf.size)
    assert rc == 1


def test_exchange_list_getters_check_their_arguments():
    """cs_fill_map_get / cs_sync_map_get: counts with null arrays, refusal
    of a wrong count, of partly null arrays and of an unknown list."""
    import numpy as np
    s = cs.Solve(ntp=8, nr=2, nghost=3)
    s.mesh_build(device=False)
    lib, n = s.lib, ctypes.c_int64(0)
    assert lib.cs_fill_map_get(s.h, None, None, None, ctypes.byref(n)) == 0 and n.value > 0
    a, b = np.zeros(n.value + 1, dtype=np.int32), np.zeros(n.value + 1, dtype=np.int32)
    m = np.zeros(n.value + 1, dtype=np.uint8)
    ip = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    u8 = m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    n1 = ctypes.c_int64(n.value + 1)
    assert lib.cs_fill_map_get(s.h, ip(a), ip(b), u8, ctypes.byref(n1)) == 1
    assert "size" in lib.cs_last_error(s.h).decode()
    assert lib.cs_fill_map_get(s.h, ip(a), None, u8, ctypes.byref(n)) == 1
    for which, expect in ((0, 4 * 8 * 2 * 6 // 2), (1, None)):
        k = ctypes.c_int64(0)
        assert lib.cs_sync_map_get(s.h, which, None, None, None, None, None, ctypes.byref(k)) == 0
        if expect is not None:  # 4 panel edges x N faces x nr layers a panel, one copy of each pair
            assert k.value == expect
        assert k.value > 0
    assert lib.cs_sync_map_get(s.h, 2, None, None, None, None, None, ctypes.byref(n)) == 1
    i8 = ctypes.POINTER(ctypes.c_int8)
    k = ctypes.c_int64(0)
    lib.cs_sync_map_get(s.h, 1, None, None, None, None, None, ctypes.byref(k))
    d, sr = np.zeros(k.value, dtype=np.int32), np.zeros(k.value, dtype=np.int32)
    assert lib.cs_sync_map_get(s.h, 1, ip(d), ip(sr), None, None, None, ctypes.byref(k)) == 1
    dst, src, dk, sk, sg = s.sync_map(1)
    assert set(np.unique(sg)) <= {-1, 1} and set(np.unique(dk)) <= {0, 1, 2}


def test_device_estimate_counts_panel_shared_row_weights():
    """The planning estimate counts the least-squares row weights the mesh
    build keeps: panel 1's serving the six panels by default (STEP 9.c's in
    FP64, both sets in the precision form), one set per panel with
    CS_FLAG_LSQ_PER_PANEL."""
    kw = dict(ntp=32, nr=16, nghost=4)
    nl = 6 * (32 + 2 * 4 - 4) ** 2 * (16 + 2 * 4 - 4)
    f64 = cs.estimate_device_bytes(**kw)
    f64_pp = cs.estimate_device_bytes(**kw, flags=cs.CS_FLAG_LSQ_PER_PANEL)
    assert f64_pp - f64 == (nl - nl // 6) * 190 * 8
    f32 = cs.estimate_device_bytes(**kw, flags=cs.CS_FLAG_FP32)
    f32_pp = cs.estimate_device_bytes(**kw, flags=cs.CS_FLAG_FP32 | cs.CS_FLAG_LSQ_PER_PANEL)
    assert f32_pp - f32 == (nl - nl // 6) * 352 * 4


def test_device_estimate_counts_the_p2_stencil_inverses():
    """With CS_FLAG_P2 the estimate adds the eight one-sided 9 x 9 (STEP 7.a)
    and 10 x 10 (STEP 9.b) inverses per zone of the least-squares range,
    panel 1's serving the six panels, one set per panel with
    CS_FLAG_LSQ_PER_PANEL, in the state's type."""
    kw = dict(ntp=32, nr=16, nghost=4)
    nl = 6 * (32 + 2 * 4 - 4) ** 2 * (16 + 2 * 4 - 4)
    for flags, n, size in ((0, nl // 6, 8), (cs.CS_FLAG_LSQ_PER_PANEL, nl, 8), (cs.CS_FLAG_FP32, nl // 6, 4)):
        base = cs.estimate_device_bytes(**kw, flags=flags)
        p2 = cs.estimate_device_bytes(**kw, flags=flags | cs.CS_FLAG_P2)
        assert p2 - base == n * (8 * 81 + 8 * 100) * size, flags
