"""GPU parity: the CUDA stage update against the CPU oracle on the same
geometry and the same seeded state, routine by routine and over whole steps.

Tolerance: 1e-12 relative (max |gpu - oracle| over the compared zones,
divided by max |oracle| of that field; for face B, of the largest face
component, since the radial one of the shell is about 1e-3 of the angular
ones) for the conserved state, the face B and the time step; 1e-10 for the
intermediate reconstruction arrays, whose nonlinear WENO weights amplify the
last-bit differences of FMA contraction and of the device pow/acos.  Ghost
exchange is a copy and must be exact.
"""
import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

TOL_STATE = 1e-12
TOL_WORK = 1e-10


def rel(a, b):
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def make_pair(name, flags=0, **over):
    from oracle import Oracle
    pr = cs.preset(name)
    pr["params"].update(over)
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build()
    s.init_problem(**pr["init"])
    st = s.get_state()
    o = Oracle(s)
    o.put_state(st)
    return s, o, st


def zones(s, a, lo=1, hi=0):
    """Zones lo..N+hi (angular) and lo..nr+hi (radial) of a panel-box array."""
    G, N, nr = s.G, s.N, s.nr
    return a[..., G + lo:G + nr + hi + 1, G + lo:G + N + hi + 1, G + lo:G + N + hi + 1]


def faces(s, a, d):
    """Faces of the interior zones in direction d (0 x, 1 y, 2 z)."""
    G, N, nr = s.G, s.N, s.nr
    lo = [1, 1, 1]
    lo[d] = 0
    return a[..., G + lo[2]:G + nr + 1, G + lo[1]:G + N + 1, G + lo[0]:G + N + 1]


def face_b_errors(s, got, want):
    """Per face component: max |got - want| over the interior faces, relative
    to the largest |want| of the three components."""
    den = max(np.abs(faces(s, want[k], d)).max() for d, k in enumerate(("bxf", "byf", "bzf")))
    den = den if den > 0 else 1.0
    return {k: float(np.abs(faces(s, got[k], d) - faces(s, want[k], d)).max() / den)
            for d, k in enumerate(("bxf", "byf", "bzf"))}


def check_state(s, got, want, tol=TOL_STATE):
    for q in range(8):
        e = rel(zones(s, got["U"][q]), zones(s, want["U"][q]))
        assert e <= tol, ("U", q, e)
    e = rel(zones(s, got["ent"]), zones(s, want["ent"]))
    assert e <= tol, ("ent", e)
    for k, e in face_b_errors(s, got, want).items():
        assert e <= tol, (k, e)


@pytest.fixture(scope="module")
def shell16():
    return make_pair("shell16")


def test_fill_ghosts_is_exact(shell16):
    s, o, st = shell16
    s.put_state(st)
    o.put_state(st)
    s.fill_ghosts()
    o.fill_ghosts()
    g, w = s.get_state(), o.get_state()
    for k in ("U", "ent", "bxf", "byf", "bzf"):
        assert np.array_equal(g[k], w[k]), k


def test_routines_in_sequence(shell16):
    s, o, st = shell16
    s.put_state(st)
    o.put_state(st)
    s.fill_ghosts()
    o.fill_ghosts()
    s.limit_all_slopes_p12()
    o.limit_all_slopes_p12()
    V, Vo = s.debug("V"), o.debug("V")
    for m in range(10):
        for c in range(8):
            e = rel(zones(s, V[m * 8 + c], 0, 1), zones(s, Vo[m * 8 + c], 0, 1))
            assert e <= TOL_WORK, ("V", m, c, e)
    for name in ("flatten", "E1", "Bxq", "Byq", "Bzq"):
        e = rel(zones(s, s.debug(name), 0, 1), zones(s, o.debug(name), 0, 1))
        assert e <= TOL_WORK, (name, e)
    s.make_facial_fluxes()
    o.make_facial_fluxes()
    e = rel(zones(s, s.debug("dUdt")), zones(s, o.debug("dUdt")))
    assert e <= TOL_WORK, ("dUdt", e)
    e = rel(zones(s, s.debug("entflux"), 0, 0), zones(s, o.debug("entflux"), 0, 0))
    assert e <= TOL_WORK, ("entflux", e)
    s.make_edge_efields_p1()
    o.make_edge_efields_p1()
    for name in ("Efx", "Efy", "Efz"):
        e = rel(zones(s, s.debug(name), 0, 0), zones(s, o.debug(name), 0, 0))
        assert e <= TOL_WORK, (name, e)
    s.build_non_stiff_sources()
    o.build_non_stiff_sources()
    e = rel(zones(s, s.debug("dUdt")), zones(s, o.debug("dUdt")))
    assert e <= TOL_WORK, ("dUdt+src", e)
    dt = 1e-3
    s.update_imex_rk_step_p1(dt)
    o.update_imex_rk_step_p1(dt)
    check_state(s, s.get_state(), o.get_state())
    s.cleanup_after_update()
    o.cleanup_after_update()
    check_state(s, s.get_state(), o.get_state())


@pytest.mark.parametrize("name,nsteps,flags,rk", [
    ("shell16", 2, 0, cs.CS_IMEX_RK2), ("shell16", 2, 0, cs.CS_RK2), ("surface32", 2, 0, cs.CS_SSPRK3),
    ("shell16", 1, cs.CS_FLAG_NO_ADP_CACHE | cs.CS_FLAG_NO_OP_CACHE, cs.CS_IMEX_RK2),
    ("shell16", 2, cs.CS_FLAG_NO_PANEL_SYNC, cs.CS_RK2)])
def test_whole_steps_match_oracle(name, nsteps, flags, rk):
    """flags=0 uses the resident geometry-only operators (ADP factors, least-squares
    inverses) and panel-edge ownership; the flags switch them off.  rk: RK2 (the
    reference's combine), SSP-RK3, IMEX-RK2 (ARS(2,2,2), gravity implicit)."""
    s, o, st = make_pair(name, flags, rk_scheme=rk)
    dt_s = s.evaluate_timestep(1e30)
    dt_o = o.evaluate_timestep(1e30)
    assert abs(dt_s - dt_o) <= TOL_STATE * dt_o
    for n in range(nsteps):
        dt_s = s.step(dt_s)
        dt_o = o.step(dt_o)
        assert abs(dt_s - dt_o) <= TOL_STATE * dt_o, (n, dt_s, dt_o)
        check_state(s, s.get_state(), o.get_state())


def test_steps_keep_div_b_at_roundoff_across_panel_edges(shell16):
    """With panel-edge ownership (the default) CT keeps div B at round-off in
    every zone, including those next to panel edges and cube corners."""
    s, o, st = shell16
    s.put_state(st)
    dt = s.evaluate_timestep(1e30)
    for _ in range(3):
        dt = s.step(dt)
    m, e, divb = s.diag()
    bmax = np.abs(faces(s, s.get_state()["bxf"], 0)).max()
    assert divb < 1e-12 * bmax, divb / bmax


@pytest.mark.parametrize("name,rk,flags", [("shell16", cs.CS_IMEX_RK2, 0), ("surface32", cs.CS_SSPRK3, 0),
                                           ("shell16", cs.CS_RK2, 0), ("shell16", cs.CS_IMEX_RK2, cs.CS_FLAG_FP32)])
def test_steps_graph_matches_step_loop(name, rk, flags):
    """cs_steps (one captured step replayed, time step kept on the device)
    gives bit for bit the state and time step of the cs_step loop."""
    pr = cs.preset(name)
    pr["params"]["rk_scheme"] = rk
    out = []
    for graph in (False, True):
        s = cs.Solve(**pr["params"], flags=flags)
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


@pytest.mark.parametrize("name,rk", [("shell16", cs.CS_IMEX_RK2), ("surface32", cs.CS_SSPRK3)])
def test_shared_panel_adp_matches_per_panel_factors(name, rk):
    """The default ADP factors (panel 1's, serving all six panels through
    the panel rotations) give the B modes of the per-panel factors to
    round-off, and the same steps within the parity tolerance."""
    pr = cs.preset(name)
    pr["params"]["rk_scheme"] = rk
    out = []
    for flags in (0, cs.CS_FLAG_ADP_PER_PANEL):
        s = cs.Solve(**pr["params"], flags=flags)
        s.mesh_build()
        s.init_problem(**pr["init"])
        s.fill_ghosts()
        s.limit_all_slopes_p12()
        V = s.debug("V")
        s.init_problem(**pr["init"])
        dt = s.evaluate_timestep(1e30)
        for _ in range(2):
            dt = s.step(dt)
        out.append((s, V, dt, s.get_state()))
    (s, V0, d0, st0), (_, V1, d1, st1) = out
    for m in range(10):
        for c in (5, 6, 7):
            e = rel(zones(s, V0[m * 8 + c], 0, 1), zones(s, V1[m * 8 + c], 0, 1))
            assert e <= 1e-11, ("B mode", m, c, e)
    assert abs(d0 - d1) <= TOL_STATE * d1
    check_state(s, st0, st1)


@pytest.mark.parametrize("name,rk,form", [("shell16", cs.CS_IMEX_RK2, 0), ("surface32", cs.CS_SSPRK3, 0),
                                          ("shell16", cs.CS_IMEX_RK2, cs.CS_FLAG_FP32)])
def test_shared_panel_row_weights_match_per_panel(name, rk, form):
    """The default least-squares row weights (panel 1's, summed and then
    rotated to each panel's modes) hold a sixth of the per-panel weights on
    the device (STEP 9.c's; STEP 7.b's too in the precision form), give the
    slopes of STEP 7.b and the E point values of STEP 9.c of the per-panel
    weights to round-off, and the same steps within the parity tolerance
    (FP64) or to FP32 rounding (precision form)."""
    pr = cs.preset(name)
    pr["params"]["rk_scheme"] = rk
    out = []
    for flags in (form, form | cs.CS_FLAG_LSQ_PER_PANEL):
        s = cs.Solve(**pr["params"], flags=flags)
        s.mesh_build()
        s.init_problem(**pr["init"])
        s.fill_ghosts()
        s.limit_all_slopes_p12()
        V, E1 = s.debug("V"), s.debug("E1")
        s.init_problem(**pr["init"])
        dt = s.evaluate_timestep(1e30)
        for _ in range(2):
            dt = s.step(dt)
        out.append((s, s.mesh_device_bytes(), V, E1, dt, s.get_state()))
    (s, b0, V0, E0, d0, st0), (_, b1, V1, E1, d1, st1) = out
    nl = 6 * (s.N + 2 * s.G - 4) ** 2 * (s.nr + 2 * s.G - 4)
    stride = lambda n: (n + 3) // 4 * 4  # STEP 7.b's rows start on 16-byte boundaries (its tensor map)
    if form:  # shared: both operators in FP32
        saved = ((stride(nl) - stride(nl // 6)) * 162 + (nl - nl // 6) * 190) * 4
    else:  # STEP 9.c's in FP64
        saved = (nl - nl // 6) * 190 * 8
    assert b1 - b0 == saved - 6 * 16  # the weights, less the six panel maps
    tw, ts = (1e-5, 1e-5) if form else (1e-11, TOL_STATE)
    for m in range(10):
        for c in range(8):
            e = rel(zones(s, V0[m * 8 + c], 0, 1), zones(s, V1[m * 8 + c], 0, 1))
            assert e <= tw, ("V mode", m, c, e)
    for q in range(3):
        e = rel(zones(s, E0[q], 0, 1), zones(s, E1[q], 0, 1))
        assert e <= tw, ("E point value", q, e)
    assert abs(d0 - d1) <= ts * d1
    check_state(s, st0, st1, tol=ts)


@pytest.mark.parametrize("name,flags", [("shell16", 0), ("surface32", 0), ("shell16", cs.CS_FLAG_FP32)])
def test_device_initial_state_matches_host(name, flags):
    """cs_init_problem builds the seeded state on the device; it agrees with
    the host construction (cs_init_problem_host) to 1e-13 of each field's
    largest value (face B: of the largest face component, since the radial
    one of the shell is round-off around zero; FP32 form: to FP32
    rounding), is zero where the host leaves the state zero, and its face B
    is divergence-free to round-off."""
    pr = cs.preset(name)
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build()
    host = s.init_problem_host(**pr["init"])
    s.init_problem(**pr["init"])
    dev = s.get_state()
    tol = 1e-13 if not flags else 1e-7
    bden = max(np.abs(host[k]).max() for k in ("bxf", "byf", "bzf"))
    for k in host:
        den = bden if k in ("bxf", "byf", "bzf") else np.abs(host[k]).max()
        assert np.abs(dev[k] - host[k]).max() <= tol * den, (k, np.abs(dev[k] - host[k]).max() / den)
    for k in ("U", "ent"):
        assert np.array_equal(dev[k] == 0, host[k] == 0), k
    m, e, divb = s.diag()
    bmax = np.abs(faces(s, dev["bxf"], 0)).max()
    assert divb < 1e-12 * bmax


def test_diag_matches_host_sums(shell16):
    """cs_diag (device reduction) against the same sums in numpy."""
    s, o, st = shell16
    s.put_state(st)
    dt = s.evaluate_timestep(1e30)
    s.step(dt)
    got = s.get_state()
    vol = s.geometry("V_VOL")[0]
    m, e, divb = s.diag()
    I = s.interior
    assert abs(m - (I(got["U"][0]) * I(vol)).sum()) <= 1e-13 * abs(m)
    assert abs(e - (I(got["U"][4]) * I(vol)).sum()) <= 1e-13 * abs(e)
    G, N, nr = s.G, s.N, s.nr
    ax, ay, az = s.geometry("XF_AREA")[0], s.geometry("YF_AREA")[0], s.geometry("ZF_AREA")[0]
    bx, by, bz = got["bxf"][0], got["byf"][0], got["bzf"][0]
    sl = lambda a, di, dj, dk: a[:, G + 1 + dk:G + nr + 1 + dk, G + 1 + dj:G + N + 1 + dj, G + 1 + di:G + N + 1 + di]
    flux = (sl(ax * bx, 0, 0, 0) - sl(ax * bx, -1, 0, 0) + sl(ay * by, 0, 0, 0) - sl(ay * by, 0, -1, 0) +
            sl(az * bz, 0, 0, 0) - sl(az * bz, 0, 0, -1))
    ref = (np.abs(flux) / I(vol)).max()
    bmax = np.abs(faces(s, got["bxf"], 0)).max()
    # both are round-off sized (their last bits differ with FMA contraction)
    assert divb < 1e-12 * bmax and ref < 1e-12 * bmax


def test_device_ghost_fill_reproduces_a_manufactured_linear_field():
    """The known answer of the reference's ghost-fill test (the manufactured
    linear field, 801:105-225) through the device fill."""
    from test_oracle_invariants import _empty_ghosts, _ghost_check, manufactured_linear_state

    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"], flags=cs.CS_FLAG_NO_PANEL_SYNC)
    s.mesh_build()
    exact = manufactured_linear_state(s)
    s.put_state(_empty_ghosts(s, exact))
    s.fill_ghosts()
    _ghost_check(s, s.get_state(), exact)


def test_device_reproduces_a_linear_field():
    """Known answer on the device: the linear primitive field with
    B = b (x, -2y, z) (801:105-225) through the device ghost fill and STEPS
    7.a / 7.b / 8.d gives slopes = l0 x gradient and zero higher modes to
    round-off clear of the radial padding (the oracle's test of the same
    state pins the restatement)."""
    from seeded_states import linear_state
    from test_oracle_invariants import _linear_errors

    pr = cs.preset("shell16")
    pr["params"]["flatten_coef"] = 1e30
    s = cs.Solve(**pr["params"])
    s.mesh_build()
    s.put_state(linear_state(s))
    s.fill_ghosts()
    s.limit_all_slopes_p12()
    assert np.abs(s.interior(s.debug("positivity"))).max() == 0
    for c, (slope, higher) in _linear_errors(s, s.debug("V")).items():
        assert slope < 1e-12 and higher < 1e-12, (c, slope, higher)


def test_positivity_active_state_matches_oracle():
    """The blob state drives STEP 7.c into its mode-shrinking loop and its
    give-up (440:553-830): the device records the same shrink count and
    give-up in every zone as the oracle, the same reconstruction, and the
    same state after two whole steps."""
    from seeded_states import positivity_state

    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"])
    s.mesh_build()
    st = positivity_state(s, s.init_problem_host(**pr["init"]))
    from oracle import Oracle
    o = Oracle(s)
    s.put_state(st)
    o.put_state(st)
    s.fill_ghosts()
    o.fill_ghosts()
    s.limit_all_slopes_p12()
    o.limit_all_slopes_p12()
    rg, ro = s.debug("positivity"), o.debug("positivity")
    act = s.mask()[None] == 1
    zl = lambda a: zones(s, a, 2 - s.G, s.G - 1)  # STEP 7.c's range
    assert np.array_equal(zl(np.where(act, rg, 0)), zl(np.where(act, ro, 0)))
    I = s.interior(rg)
    assert int(((I >= 2) & (I % 2 == 0)).sum()) >= 10 and int((I % 2 == 1).sum()) >= 1
    V, Vo = s.debug("V"), o.debug("V")
    for m in range(10):
        for c in range(8):
            e = rel(zones(s, V[m * 8 + c], 0, 1), zones(s, Vo[m * 8 + c], 0, 1))
            assert e <= TOL_WORK, ("V", m, c, e)
    e = rel(zones(s, s.debug("ent_modes")[0]), zones(s, o.debug("ent_modes")[0]))
    assert e <= TOL_STATE, ("entropy after give-up", e)
    s.put_state(st)
    o.put_state(st)
    dt_s, dt_o = s.evaluate_timestep(1e30), o.evaluate_timestep(1e30)
    for n in range(2):
        dt_s, dt_o = s.step(dt_s), o.step(dt_o)
        assert abs(dt_s - dt_o) <= TOL_STATE * dt_o, (n, dt_s, dt_o)
        check_state(s, s.get_state(), o.get_state())


def max_state_error(s, got, want):
    e = 0.0
    for q in range(8):
        e = max(e, rel(zones(s, got["U"][q]), zones(s, want["U"][q])))
    e = max(e, rel(zones(s, got["ent"]), zones(s, want["ent"])))
    return max(e, max(face_b_errors(s, got, want).values()))


# Relative state error bounds of the 100-step surface run at the checked
# steps: round-off differences (FMA contraction, device pow/acos) pass
# through the nonlinear WENO weights every stage and grow with the steps;
# measured on a B200 they grow from 2.6e-14 (step 1) to 3.4e-13 (step 100),
# inside the 1e-12 of the single-step checks.
C0_BOUNDS = {1: TOL_STATE, 10: TOL_STATE, 100: TOL_STATE}


def test_surface32_100_ssprk3_steps_match_oracle():
    """The CPU-runnable configuration as stated (6 x 32^2 x 1 surface, 3
    ghost layers, SSP-RK3, CFL 0.4, 100 steps) on the device against the
    oracle from the same seeded state: state and time step at steps 1, 10
    and 100 within C0_BOUNDS, and the time step of every step within
    1e-12."""
    s, o, st = make_pair("surface32")
    dt_s = s.evaluate_timestep(1e30)
    dt_o = o.evaluate_timestep(1e30)
    growth = {}
    for n in range(1, 101):
        dt_s = s.step(dt_s)
        dt_o = o.step(dt_o)
        assert abs(dt_s - dt_o) <= TOL_STATE * dt_o, (n, dt_s, dt_o)
        if n in C0_BOUNDS or n % 25 == 0:
            growth[n] = max_state_error(s, s.get_state(), o.get_state())
    print("surface32 state error by step:", {k: f"{v:.2e}" for k, v in growth.items()})
    for n, bound in C0_BOUNDS.items():
        assert growth[n] <= bound, (n, growth)


@pytest.mark.parametrize("name,flags", [("shell16", 0), ("surface32", 0), ("shell16", cs.CS_FLAG_FP32)])
def test_step10_min_max_match_oracle(name, flags):
    """STEP 10 on the device (CS_FLAG_STEP10) against the oracle after one
    whole step (the last stage's values, as the reference driver prints
    them): primitives' min / max within 1e-12 of the field scale (FP32 form:
    1e-5), the divergence entries within 1e-12 of the largest face area (they
    are round-off of a divergence-free field)."""
    s, o, st = make_pair(name, flags | cs.CS_FLAG_STEP10)
    dt_s, dt_o = s.evaluate_timestep(1e30), o.evaluate_timestep(1e30)
    s.step(dt_s)
    o.step(dt_o)
    (gmin, gmax), (wmin, wmax) = s.limit_minmax(), o.limit_minmax()
    tol = 1e-5 if flags & cs.CS_FLAG_FP32 else 1e-12
    for q in range(8):
        scale = max(abs(wmin[q]), abs(wmax[q]), 1e-300)
        assert abs(gmin[q] - wmin[q]) <= tol * scale, ("min", q, gmin[q], wmin[q])
        assert abs(gmax[q] - wmax[q]) <= tol * scale, ("max", q, gmax[q], wmax[q])
    area = float(np.abs(s.geometry("XF_AREA")).max())
    for a, b in ((gmin[8], wmin[8]), (gmax[8], wmax[8])):
        assert abs(a) < 1e-12 * area and abs(b) < 1e-12 * area
    plain = cs.Solve(**cs.preset(name)["params"], flags=flags)
    plain.mesh_build()
    with pytest.raises(cs.CsError):
        plain.limit_minmax()  # not evaluated without the flag


@pytest.mark.parametrize("flags", [0, cs.CS_FLAG_FP32])
def test_a_bounded_wait_that_gave_up_fails_the_step(flags):
    """The device flag a bounded mbarrier wait sets when it gives up (here
    set from the host: no device wait is made to fail) turns the next step
    into CS_ERR_CUDA with the reason; cleared, the solve steps again."""
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build()
    s.init_problem(**pr["init"])
    dt = s.evaluate_timestep(1e30)
    assert s.lib.cs_debug_set_wait_error(s.h, 1) == 0
    with pytest.raises(cs.CsError, match="bounded device wait"):
        s.step(dt)
    assert s.lib.cs_debug_set_wait_error(s.h, 0) == 0
    s.init_problem(**pr["init"])
    assert s.step(s.evaluate_timestep(1e30)) > 0
