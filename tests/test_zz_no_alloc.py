"""cs_cfl_timestep_noalloc (static device scratch, no allocation) against
cs_evaluate_timestep on the same resident state, two calls in a row.
Collected last on purpose; it also passes on its own."""
import ctypes

import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]


def test_noalloc_cfl_matches_context_timestep_twice():
    import torch

    torch.cuda.set_device(0)
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"])
    s.mesh_build()
    s.init_problem(**pr["init"])
    p = s.params
    st = s.get_state()
    U = torch.from_numpy(st["U"]).cuda()
    ent = torch.from_numpy(st["ent"]).cuda()
    vs = torch.from_numpy(s.geometry("V_SCALE")).cuda()
    mk = torch.from_numpy(s.mask()).cuda()
    torch.cuda.synchronize()
    lib = s.lib
    dt_ref = 1e30
    dt_na = 1e30
    for _ in range(2):
        out = ctypes.c_double()
        rc = lib.cs_cfl_timestep_noalloc(U.data_ptr(), ent.data_ptr(), vs.data_ptr(), mk.data_ptr(), p.ntp, p.nr,
                                         p.nghost, p.gamma, p.rhofloor, p.prsfloor, p.cfl_coef, dt_na, None,
                                         ctypes.byref(out))
        assert rc == 0
        dt_ref = s.evaluate_timestep(dt_ref)
        dt_na = out.value
        # the context's entry point also writes back its conserved->primitive
        # repair, so its second call may see last-bit changes
        assert abs(dt_na - dt_ref) <= 1e-13 * dt_ref, (dt_na, dt_ref)
    # the arrays are only read
    assert torch.equal(U.cpu(), torch.from_numpy(st["U"]))


def test_noalloc_rejects_more_layers_than_its_scratch():
    lib = cs.load_library()
    out = ctypes.c_double()
    dummy = ctypes.c_void_p(16)
    rc = lib.cs_cfl_timestep_noalloc(dummy, dummy, dummy, dummy, 8, 4096, 4, 5.0 / 3.0, 1e-12, 1e-9, 0.4, 1.0,
                                     None, ctypes.byref(out))
    assert rc == 1  # CS_ERR_ARG, nothing launched
