"""Known answers of the pointwise physics (oracle on the CPU; the device
functions the stage kernels call, through cs_pointwise, on the GPU):

* the round trip of the reference's own test program
  _T/_660riemann_3d/660pde_3d_test_program.f:58-142: the primitive vector
  (0.33333, 1.3, 0.3, 0.7, 1.3, 0.88, 0.3001, 0.987) with gamma 5/3 and
  floors 1e-12 through PRIM_TO_CONS and back through CONS_TO_PRIM returns
  itself to machine precision, and the conserved vector is the closed form
  (rho, rho v, p/(gamma-1) + rho v^2/2 + B^2/8pi, B);
* HLL consistency: for equal left and right states the solver's flux
  F_L + Fluct_L = F_R - Fluct_R equals the ideal-MHD x-flux F(U), written
  out here independently of both implementations, the speeds are u -+ the
  fast magnetosonic speed and the entropy flux is s u.
"""
import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu
from oracle import Oracle

GAMMA = 5.0 / 3.0
PARAMS = dict(ntp=8, nr=4, gamma=GAMMA, rhofloor=1e-12, prsfloor=1e-12)
REF_V = np.array([0.33333, 1.3, 0.3, 0.7, 1.3, 0.88, 0.3001, 0.987])


def closed_form_cons(V):
    rho, v, p, B = V[..., 0], V[..., 1:4], V[..., 4], V[..., 5:8]
    U = np.zeros_like(V)
    U[..., 0] = rho
    U[..., 1:4] = rho[..., None] * v
    U[..., 4] = p / (GAMMA - 1) + 0.5 * rho * (v ** 2).sum(-1) + (B ** 2).sum(-1) / (8 * np.pi)
    U[..., 5:8] = B
    return U


def mhd_flux_x(V):
    """Ideal-MHD flux along x in Gaussian units (B0 = 0)."""
    rho, u, v, w, p, bx, by, bz = (V[..., c] for c in range(8))
    b2 = bx * bx + by * by + bz * bz
    pt = p + b2 / (8 * np.pi)
    E = p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v + w * w) + b2 / (8 * np.pi)
    vb = u * bx + v * by + w * bz
    return np.stack([rho * u, rho * u * u + pt - bx * bx / (4 * np.pi), rho * u * v - bx * by / (4 * np.pi),
                     rho * u * w - bx * bz / (4 * np.pi), (E + pt) * u - bx * vb / (4 * np.pi), 0.0 * u,
                     u * by - v * bx, u * bz - w * bx], axis=-1)


def fast_speed_x(V):
    rho, p, bx, by, bz = V[..., 0], V[..., 4], V[..., 5], V[..., 6], V[..., 7]
    a2 = GAMMA * p / rho
    b2 = (bx * bx + by * by + bz * bz) / (4 * np.pi * rho)
    bx2 = bx * bx / (4 * np.pi * rho)
    return np.sqrt(0.5 * ((a2 + b2) + np.sqrt((a2 + b2) ** 2 - 4 * a2 * bx2)))


def seeded_prims(n=500, seed=17):
    rng = np.random.default_rng(seed)
    V = np.zeros((n, 8))
    V[:, 0] = rng.uniform(0.1, 10.0, n)
    V[:, 1:4] = rng.normal(size=(n, 3))
    V[:, 4] = rng.uniform(0.05, 10.0, n)
    V[:, 5:8] = rng.normal(size=(n, 3))
    return V


def roundtrip_cases(V):
    ent = V[:, 4] / V[:, 0] ** (GAMMA - 1)
    return np.concatenate([V, ent[:, None]], axis=1)


def hll_cases(V):
    ent = V[:, 4] / V[:, 0] ** (GAMMA - 1)
    return np.concatenate([V, V, ent[:, None], ent[:, None]], axis=1), ent


def check_roundtrip(to_cons, to_prim, tol):
    V = np.concatenate([REF_V[None], seeded_prims()], axis=0)
    cases = roundtrip_cases(V)
    U = to_cons(cases)
    np.testing.assert_allclose(U, closed_form_cons(V), rtol=tol, atol=tol)
    back = to_prim(np.concatenate([U, cases[:, 8:9]], axis=1))
    assert np.all(back[:, 9] == 0)  # no floor applied
    err = np.abs(back[:, :8] - V).sum(axis=1)
    assert err[0] <= 8 * tol, err[0]  # the reference program's SUM(ABS(Vpt - Fpt))
    np.testing.assert_allclose(back[:, :8], V, rtol=tol, atol=tol * np.abs(V).max())


def check_hll(hll, tol):
    V = seeded_prims(seed=23)
    V[:50, 1] += 20.0  # supersonic to the right: the upwind branch S_L >= 0
    V[50:100, 1] -= 20.0  # supersonic to the left: S_R <= 0
    cases, ent = hll_cases(V)
    out = hll(cases)
    FlL, FlR, FL, FR = out[:, 0:8], out[:, 8:16], out[:, 16:24], out[:, 24:32]
    F = mhd_flux_x(V)
    scale = np.abs(F).max(axis=1, keepdims=True) + np.abs(closed_form_cons(V)).max(axis=1, keepdims=True) * (
        np.abs(V[:, 1:2]) + fast_speed_x(V)[:, None])
    assert np.all(np.abs(FL + FlL - F) <= tol * scale)
    assert np.all(np.abs(FR - FlR - F) <= tol * scale)
    cf = fast_speed_x(V)
    np.testing.assert_allclose(out[:, 32], V[:, 1] - cf, rtol=tol, atol=tol * cf.max())
    np.testing.assert_allclose(out[:, 33], V[:, 1] + cf, rtol=tol, atol=tol * cf.max())
    np.testing.assert_allclose(out[:, 34], ent * V[:, 1], rtol=tol, atol=tol * np.abs(ent * V[:, 1]).max())
    # the supersonic branches take the upwind flux with zero fluctuations exactly
    assert np.all(FlL[:100] == 0.0) and np.all(FlR[:100] == 0.0)


def _oracle():
    return Oracle(params=cs.make_params(**PARAMS), mesh=False)


def test_oracle_prim_cons_roundtrip_of_the_reference_program():
    o = _oracle()
    check_roundtrip(lambda c: o.pointwise(0, c), lambda c: o.pointwise(1, c), 1e-14)


def test_oracle_hll_is_consistent():
    o = _oracle()
    check_hll(lambda c: o.pointwise(2, c), 1e-13)


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
@pytest.mark.parametrize("flags,tol", [(0, 1e-14), (cs.CS_FLAG_FP32, 2e-6)])
def test_device_prim_cons_roundtrip_of_the_reference_program(flags, tol):
    check_roundtrip(lambda c: cs.pointwise(0, c, flags=flags, **PARAMS),
                    lambda c: cs.pointwise(1, c, flags=flags, **PARAMS), tol)


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
@pytest.mark.parametrize("flags,tol", [(0, 1e-13), (cs.CS_FLAG_FP32, 2e-5)])
def test_device_hll_is_consistent_and_matches_oracle(flags, tol):
    check_hll(lambda c: cs.pointwise(2, c, flags=flags, **PARAMS), tol)
    if not flags:
        V = seeded_prims(seed=29)
        rng = np.random.default_rng(31)
        W = V.copy()
        W[:, :8] += 0.3 * rng.normal(size=W.shape) * np.abs(W)
        W[:, 0] = np.abs(W[:, 0]) + 0.1
        W[:, 4] = np.abs(W[:, 4]) + 0.05
        eL = V[:, 4] / V[:, 0] ** (GAMMA - 1)
        eR = W[:, 4] / W[:, 0] ** (GAMMA - 1)
        cases = np.concatenate([V, W, eL[:, None], eR[:, None]], axis=1)
        got = cs.pointwise(2, cases, **PARAMS)
        want = _oracle().pointwise(2, cases)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
