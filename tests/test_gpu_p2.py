"""LIMIT_ALL_SLOPES_P2 (CS_FLAG_P2, 420limit_all_slopes_p2.f) on the
device against the oracle: the reconstruction arrays of one
LIMIT_ALL_SLOPES call, whole steps in the three integrators, the per-panel
and panel-shared stencil inverses, the precision form, the graph replay,
and the two known answers of the third-order stencils (quadratic
primitives, the zone averages of a quadratic E).  Tolerances as in
test_gpu_parity: 1e-12 relative for the state, 1e-10 for the intermediate
reconstruction arrays."""
import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu
from test_gpu_parity import TOL_STATE, TOL_WORK, check_state, make_pair, rel, zones

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

P2 = cs.CS_FLAG_P2


def test_p2_reconstruction_matches_oracle():
    """One LIMIT_ALL_SLOPES_P2 on the seeded shell: the modes of every
    primitive (STEP 7.a's nine quadratic stencils), the entropy slopes, the
    ADP face-B values and the E point values (STEP 9.b) agree with the
    oracle, and so does the rest of the stage."""
    s, o, st = make_pair("shell16", P2)
    s.fill_ghosts()
    o.fill_ghosts()
    s.limit_all_slopes_p12()
    o.limit_all_slopes_p12()
    V, Vo = s.debug("V"), o.debug("V")
    for m in range(10):
        for c in range(8):
            e = rel(zones(s, V[m * 8 + c], 0, 1), zones(s, Vo[m * 8 + c], 0, 1))
            assert e <= TOL_WORK, ("V", m, c, e)
    for name in ("ent_modes", "flatten", "E1", "Bxq", "Byq", "Bzq"):
        e = rel(zones(s, s.debug(name), 0, 1), zones(s, o.debug(name), 0, 1))
        assert e <= TOL_WORK, (name, e)
    s.make_facial_fluxes()
    o.make_facial_fluxes()
    e = rel(zones(s, s.debug("dUdt")), zones(s, o.debug("dUdt")))
    assert e <= TOL_WORK, ("dUdt", e)
    s.make_edge_efields_p1()
    o.make_edge_efields_p1()
    for name in ("Efx", "Efy", "Efz"):
        e = rel(zones(s, s.debug(name), 0, 0), zones(s, o.debug(name), 0, 0))
        assert e <= TOL_WORK, (name, e)


@pytest.mark.parametrize("name,nsteps,flags,rk", [
    ("shell16", 2, P2, cs.CS_IMEX_RK2), ("surface32", 2, P2, cs.CS_SSPRK3),
    ("shell16", 2, P2 | cs.CS_FLAG_LSQ_PER_PANEL, cs.CS_RK2)])
def test_p2_whole_steps_match_oracle(name, nsteps, flags, rk):
    """Whole steps with P2 in place of P12: panel-shared stencil inverses by
    default, per-panel ones with CS_FLAG_LSQ_PER_PANEL."""
    s, o, st = make_pair(name, flags, rk_scheme=rk)
    dt_s = s.evaluate_timestep(1e30)
    dt_o = o.evaluate_timestep(1e30)
    for n in range(nsteps):
        dt_s = s.step(dt_s)
        dt_o = o.step(dt_o)
        assert abs(dt_s - dt_o) <= TOL_STATE * dt_o, (n, dt_s, dt_o)
        check_state(s, s.get_state(), o.get_state())


def test_p2_differs_from_p12():
    """The flag changes the scheme: after one step the states of P2 and P12
    differ by far more than round-off (the third-order stencils' truncation
    error against P12's), while both match their oracles above."""
    out = []
    for flags in (0, P2):
        pr = cs.preset("shell16")
        s = cs.Solve(**pr["params"], flags=flags)
        s.mesh_build()
        s.init_problem(**pr["init"])
        s.step(s.evaluate_timestep(1e30))
        out.append(s.get_state()["U"])
    assert rel(out[1], out[0]) > 1e-8


def test_p2_shared_inverses_match_per_panel():
    """Panel 1's stencil inverses rotated to each panel give the modes of the
    per-panel inverses to round-off."""
    Vs = []
    for flags in (P2, P2 | cs.CS_FLAG_LSQ_PER_PANEL):
        pr = cs.preset("shell16")
        s = cs.Solve(**pr["params"], flags=flags)
        s.mesh_build()
        s.init_problem(**pr["init"])
        s.fill_ghosts()
        s.limit_all_slopes_p12()
        Vs.append((s, s.debug("V"), s.debug("E1")))
    (s, V0, E0), (_, V1, E1) = Vs
    for m in range(1, 10):
        for c in range(8):
            assert rel(zones(s, V0[m * 8 + c], 0, 1), zones(s, V1[m * 8 + c], 0, 1)) <= TOL_WORK, (m, c)
    assert rel(zones(s, E0, 0, 1), zones(s, E1, 0, 1)) <= TOL_WORK


def test_p2_device_reproduces_quadratic_primitives():
    """Known answer on the device: quadratic primitives held as exact zone
    averages come back as their exact modes (test_oracle_invariants'
    quadratic case) from the resident stencil inverses."""
    from seeded_states import quadratic_state
    from test_oracle_invariants import _quadratic_errors

    pr = cs.preset("shell16")
    pr["params"].update(flatten_coef=1e30)
    s = cs.Solve(**pr["params"], flags=P2)
    s.mesh_build()
    s.put_state(quadratic_state(s))
    s.fill_ghosts()
    s.limit_all_slopes_p12()
    for c, e in _quadratic_errors(s, s.debug("V")).items():
        assert e < 1e-12, (c, e)


def test_p2_device_interpolates_e_to_zone_averages():
    """Known answer on the device: STEP 9.b returns the zone averages of the
    quadratic E of linear v and B."""
    from seeded_states import away_from_radial_padding, linear_state, linear_state_e_averages

    pr = cs.preset("shell32")
    pr["params"].update(flatten_coef=1e30)
    s = cs.Solve(**pr["params"], flags=P2)
    s.mesh_build()
    s.put_state(linear_state(s))
    s.fill_ghosts()
    s.limit_all_slopes_p12()
    E1 = s.debug("E1")
    core = lambda a: away_from_radial_padding(s, a, m=5)[..., 2:-2, 2:-2]
    for q, ex in enumerate(linear_state_e_averages(s)):
        assert np.abs(core(E1[q] - ex)).max() / np.abs(core(ex)).max() < 1e-12, q


def test_p2_precision_form_tracks_fp64():
    """P2 in the precision form: after 3 steps the state stays within FP32
    truncation of the FP64 P2 solve (max relative error per conserved
    component below 1e-5)."""
    out = []
    for flags in (P2, P2 | cs.CS_FLAG_FP32):
        pr = cs.preset("shell16")
        s = cs.Solve(**pr["params"], flags=flags)
        s.mesh_build()
        s.init_problem(**pr["init"])
        dt = s.evaluate_timestep(1e30)
        for _ in range(3):
            dt = s.step(dt)
        out.append(s.get_state())
    for q in range(8):
        e = rel(zones(s, out[1]["U"][q]), zones(s, out[0]["U"][q]))
        assert e < 1e-5, (q, e)


def test_p2_steps_graph_matches_step_loop():
    """cs_steps with P2 gives bit for bit the cs_step loop."""
    pr = cs.preset("shell16")
    out = []
    for graph in (False, True):
        s = cs.Solve(**pr["params"], flags=P2)
        s.mesh_build()
        s.init_problem(**pr["init"])
        dt = s.evaluate_timestep(1e30)
        if graph:
            dt = s.steps(3, dt)
        else:
            for _ in range(3):
                dt = s.step(dt)
        out.append((dt, s.get_state()))
    (d0, s0), (d1, s1) = out
    assert d0 == d1
    for k in s0:
        assert np.array_equal(s0[k], s1[k]), k
