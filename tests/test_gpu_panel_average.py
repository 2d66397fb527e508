"""CS_FLAG_PANEL_AVERAGE on the device: the reference's rule for the copies
of shared faces and edges (every copy takes their average, the three copies
of a cube-corner radial edge their sum / 3; 334fetch_buffers_fill_in_flux_x.f
:295-395, 335fetch_buffers_fill_in_flux_y.f:761-795) against the oracle with
the same rule, over whole steps, to the parity tolerance of the default
rule.  On the CPU the oracle's averages are pinned to the exported lists in
the device kernels' grouping (tests/test_halo.py) and to the cube's rotation
symmetry (tests/test_oracle_invariants.py).

The averaging kernels (k_avg_flux, k_avg_emf) had not been run on a GPU when
these tests were written, so they are marked xfail(strict=False): "xpassed"
is the kernels' first device check passing, "xfailed" a mismatch to fix;
either way the rest of the GPU suite runs."""
import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu
from test_gpu_parity import TOL_STATE, check_state, faces, make_pair, zones

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device"),
              pytest.mark.xfail(strict=False, reason="the averaging kernels had not run on a GPU when written")]


@pytest.mark.parametrize("name,rk", [("shell16", cs.CS_IMEX_RK2), ("surface32", cs.CS_SSPRK3)])
def test_panel_average_steps_match_the_oracle(name, rk):
    s, o, st = make_pair(name, cs.CS_FLAG_PANEL_AVERAGE, rk_scheme=rk)
    dt_s = s.evaluate_timestep(1e30)
    dt_o = o.evaluate_timestep(1e30)
    for n in range(2):
        dt_s = s.step(dt_s)
        dt_o = o.step(dt_o)
        assert abs(dt_s - dt_o) <= TOL_STATE * dt_o, (n, dt_s, dt_o)
        check_state(s, s.get_state(), o.get_state())
    m, e, divb = s.diag()
    bmax = np.abs(faces(s, s.get_state()["bxf"], 0)).max()
    assert divb < 1e-12 * bmax, divb / bmax


def test_panel_average_keeps_the_cube_symmetry():
    """The hydrostatic shell without its perturbations stays the same on the
    six panels (exact rotations of one another) under the averaging rule."""
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"], flags=cs.CS_FLAG_PANEL_AVERAGE)
    s.mesh_build()
    s.init_problem(**dict(pr["init"], rho_amp=0.0, a_amp=0.0))
    dt = s.evaluate_timestep(1e30)
    for _ in range(3):
        dt = s.step(dt)
    rho = zones(s, s.get_state()["U"][0])
    assert np.abs(rho - rho[0]).max() / np.abs(rho).max() < 1e-12
