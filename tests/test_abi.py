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
