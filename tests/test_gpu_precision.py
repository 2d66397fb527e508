"""The precision form (CS_FLAG_FP32) against the plain FP64 form.

The precision form stores and computes the bulk of the stage in FP32 and
keeps face B, the ADP system, the EMFs and the geometry in FP64.
It is not a parity form: its results differ from the FP64 ones by the FP32
rounding of the state, carried through the nonlinear reconstruction.  The
bounds below are stated per field as relative L1 errors,
sum |fp32 - fp64| / sum |fp64| over the interior zones (faces for B), after
the same number of steps with the same time steps:

  density, total energy, entropy      <= 1e-6
  momentum (all three components)     <= 5e-5  (the flow starts near rest,
                                                so its magnitude is small)
  face B (the three face components   <= 1e-6
  together, sum |dB| / sum |B|)

and div B stays at FP64 round-off, since CT advances the FP64 faces with
the FP64 EMFs.  Face B is measured as one vector field: the radial face
component of these states is 1e-3 of the angular ones, and an FP64 run
started from the FP32-rounded state moves it by 2e-6 of its own size, so
a per-component bound on it would measure the problem's sensitivity, not
the precision form.
"""
import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

TOL_L1 = {"rho": 1e-6, "mom": 5e-5, "E": 1e-6, "ent": 1e-6, "B": 1e-6}


def l1(a, b):
    den = np.abs(b).sum()
    return float(np.abs(a - b).sum() / (den if den > 0 else 1.0))


def faces(s, a, d):
    G, N, nr = s.G, s.N, s.nr
    lo = [1, 1, 1]
    lo[d] = 0
    return a[..., G + lo[2]:G + nr + 1, G + lo[1]:G + N + 1, G + lo[0]:G + N + 1]


def field_errors(s, got, want):
    I = s.interior
    out = {"rho": l1(I(got["U"][0]), I(want["U"][0])),
           "mom": l1(I(got["U"][1:4]), I(want["U"][1:4])),
           "E": l1(I(got["U"][4]), I(want["U"][4])),
           "ent": l1(I(got["ent"]), I(want["ent"]))}
    num = sum(np.abs(faces(s, got[k], d) - faces(s, want[k], d)).sum() for d, k in enumerate(("bxf", "byf", "bzf")))
    den = sum(np.abs(faces(s, want[k], d)).sum() for d, k in enumerate(("bxf", "byf", "bzf")))
    out["B"] = float(num / den)
    return out


def run(name, flags, nsteps, dts=None, rk=None):
    pr = cs.preset(name)
    if rk is not None:
        pr["params"]["rk_scheme"] = rk
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build()
    s.init_problem(**pr["init"])
    dt = s.evaluate_timestep(1e30)
    used = []
    for n in range(nsteps):
        d = dt if dts is None else dts[n]
        used.append(d)
        dt = s.step(d)
    return s, used


@pytest.mark.parametrize("name,nsteps,rk", [("shell16", 4, cs.CS_IMEX_RK2), ("shell32", 3, cs.CS_IMEX_RK2),
                                            ("surface32", 3, cs.CS_SSPRK3), ("shell16", 3, cs.CS_RK2)])
def test_fp32_form_tracks_fp64(name, nsteps, rk):
    s64, dts = run(name, 0, nsteps, rk=rk)
    s32, _ = run(name, cs.CS_FLAG_FP32, nsteps, dts=dts, rk=rk)
    want, got = s64.get_state(), s32.get_state()
    assert np.isfinite(got["U"]).all()
    err = field_errors(s64, got, want)
    for k, tol in TOL_L1.items():
        assert err[k] <= tol, (k, err[k], err)
    m64, e64, _ = s64.diag()
    m32, e32, divb = s32.diag()
    assert abs(m32 - m64) <= 1e-6 * abs(m64)
    bmax = np.abs(faces(s32, got["bxf"], 0)).max()
    assert divb < 1e-12 * bmax, divb / bmax


def test_fp32_form_time_step_close_to_fp64():
    s64, _ = run("shell16", 0, 0)
    s32, _ = run("shell16", cs.CS_FLAG_FP32, 0)
    d64, d32 = s64.evaluate_timestep(1e30), s32.evaluate_timestep(1e30)
    assert abs(d32 - d64) <= 1e-5 * d64


def test_fp32_state_round_trip_is_fp32_rounding():
    """cs_state_put / cs_state_get keep the FP64 boundary: U and the entropy
    come back rounded to FP32, face B unchanged."""
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"], flags=cs.CS_FLAG_FP32)
    s.mesh_build()
    st = s.init_problem_host(**pr["init"])
    s.put_state(st)
    got = s.get_state()
    assert np.array_equal(got["U"], st["U"].astype(np.float32).astype(np.float64))
    assert np.array_equal(got["ent"], st["ent"].astype(np.float32).astype(np.float64))
    for k in ("bxf", "byf", "bzf"):
        assert np.array_equal(got[k], st[k])


def test_fp32_routines_track_fp64():
    """Routine by routine from the same state: the reconstructed primitives
    and the flux divergence of the precision form stay within FP32 rounding
    amplified by the nonlinear weights (relative L1 <= 1e-4)."""
    pr = cs.preset("shell16")
    out = []
    for flags in (0, cs.CS_FLAG_FP32):
        s = cs.Solve(**pr["params"], flags=flags)
        s.mesh_build()
        s.init_problem(**pr["init"])
        s.fill_ghosts()
        s.limit_all_slopes_p12()
        V = s.debug("V")
        s.make_facial_fluxes()
        out.append((s, V, s.debug("dUdt")))
    (s, V64, D64), (_, V32, D32) = out
    for c in range(8):
        assert l1(s.interior(V32[c]), s.interior(V64[c])) <= 1e-4, ("V", c)
    assert l1(s.interior(D32[0]), s.interior(D64[0])) <= 1e-4


def test_fp32_form_long_run_stays_within_1e_5():
    """Over 200 steps (shell16, IMEX-RK2) the precision form's relative L1
    error stays below 1e-5 in every field, and its div B stays at the
    round-off level the FP64 form accumulates over the same steps (per unit
    length; the zones are about 1/16 wide)."""
    s64, dts = run("shell16", 0, 200)
    s32, _ = run("shell16", cs.CS_FLAG_FP32, 200, dts=dts)
    want, got = s64.get_state(), s32.get_state()
    err = field_errors(s64, got, want)
    for k in ("rho", "mom", "E", "ent", "B"):
        assert err[k] <= 1e-5, (k, err[k], err)
    _, _, divb64 = s64.diag()
    _, _, divb = s32.diag()
    bmax = np.abs(faces(s32, got["bxf"], 0)).max()
    assert divb < 1e-10 * bmax and divb <= 10.0 * divb64 + 1e-13 * bmax, (divb / bmax, divb64 / bmax)


def test_fp32_form_without_resident_operators_tracks_the_cached_form():
    """The precision form's fallback without resident least-squares weights
    (CS_FLAG_NO_OP_CACHE, taken on meshes too large for them: every stage
    rebuilds the rows and inverts the normal matrices, in FP64 like the
    cached weights, and rounds the inverse once) stays within FP32 rounding
    of the cached form after 3 steps: relative L1 <= 1e-6 per field, 5e-5
    for the momentum (the shell starts at rest, so it is small against its
    own rounding): TOL_L1, the bounds of test_fp32_form_tracks_fp64."""
    s0, dts = run("shell16", cs.CS_FLAG_FP32, 3)
    s1, _ = run("shell16", cs.CS_FLAG_FP32 | cs.CS_FLAG_NO_OP_CACHE, 3, dts=dts)
    err = field_errors(s0, s1.get_state(), s0.get_state())
    for k in ("rho", "mom", "E", "ent", "B"):
        assert err[k] <= TOL_L1[k], (k, err[k], err)
