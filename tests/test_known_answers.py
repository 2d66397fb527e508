"""Known answers of the reference's own test programs for the edge-EMF
Riemann solvers (_T/_620riemann_2d):

* 631_2d_rs_ez_test_twod_rs_ez_4state.f:16-30 -- four identical states
  (S = +-1, sin_t = 1, Bneta_U = Bneta_D = 1, By = 0.27, v = (0.5, -0.3)):
  the solver returns the common Ez = -(vx By - vy Bx) = -0.435;
* 630_2d_rs_ez_test_twod_rs_ez_3state.f:32-110 -- three identical states
  V = (1, 0.5, 0.7, -0.4, 0.8, 1.0, 0.3, 1.6) with the face normals at
  120 degrees: ESSz = Ez = -(0.5*0.3 - 0.7*1.0) = 0.55.

Uniform states give the common Ez for any speeds and angle (no jumps to
dissipate); the oracle restatement is checked on the reference's cases and
on seeded uniform cases, and the device solvers (through cs_twod_rs_ez)
against both the known answers and the oracle on seeded non-uniform cases.
"""
import math

import numpy as np
import pytest

import oracle
from conftest import has_gpu


def case4(sin_t, Bn, By, vx, vy, S=(1.0, -1.0, 1.0, -1.0)):
    cos_t = math.sqrt(1.0 - sin_t ** 2)
    Bx = (Bn + cos_t * By) / sin_t
    Ez = -(vx * By - vy * Bx)
    return (*S, cos_t, sin_t, Ez, Ez, Ez, Ez, Bn, Bn, By, By), Ez


def case3(V):
    sq3_2 = math.sqrt(3.0) / 2.0
    vx, vy, Bx, By = V[1], V[2], V[5], V[6]
    Bn1 = -(By + By) * 0.5
    Bn2 = (sq3_2 * Bx + 0.5 * By + sq3_2 * Bx + 0.5 * By) * 0.5
    Bn3 = (-sq3_2 * Bx + 0.5 * By - sq3_2 * Bx + 0.5 * By) * 0.5
    Ez = -(vx * By - vy * Bx)
    return (1.0, -1.0, 1.0, -1.0, 1.0, -1.0, Ez, Ez, Ez, Bn1, Bn2, Bn3), Ez


def test_four_state_reference_case():
    args, Ez = case4(1.0, 1.0, 0.27, 0.5, -0.3)
    assert Ez == pytest.approx(-0.435, abs=1e-15)
    assert oracle.twod_rs_ez_4state(*args) == pytest.approx(-0.435, abs=1e-14)


def test_three_state_reference_case():
    args, Ez = case3([1.0, 0.5, 0.7, -0.4, 0.8, 1.0, 0.3, 1.6])
    assert Ez == pytest.approx(0.55, abs=1e-15)
    assert oracle.twod_rs_ez_3state(*args) == pytest.approx(0.55, abs=1e-14)


def test_uniform_states_return_their_ez():
    rng = np.random.default_rng(5)
    for _ in range(200):
        S = (rng.uniform(0.1, 2), -rng.uniform(0.1, 2), rng.uniform(0.1, 2), -rng.uniform(0.1, 2))
        args, Ez = case4(rng.uniform(0.3, 1.0), rng.normal(), rng.normal(), rng.normal(), rng.normal(), S)
        assert oracle.twod_rs_ez_4state(*args) == pytest.approx(Ez, abs=1e-12 * (1 + abs(Ez)))
        V = rng.normal(size=8)
        args3, Ez3 = case3(V)
        S3 = [rng.uniform(0.1, 2) * sg for sg in (1, -1, 1, -1, 1, -1)]
        args3 = (*S3, *args3[6:])
        assert oracle.twod_rs_ez_3state(*args3) == pytest.approx(Ez3, abs=1e-12 * (1 + abs(Ez3)))


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_device_solvers_match_known_answers_and_oracle():
    import cubesphere_b200 as cs

    rng = np.random.default_rng(6)
    a4, a3, want4, want3 = [], [], [], []
    args, Ez = case4(1.0, 1.0, 0.27, 0.5, -0.3)
    a4.append(args[:7] + args[10:])
    want4.append(Ez)
    args, Ez = case3([1.0, 0.5, 0.7, -0.4, 0.8, 1.0, 0.3, 1.6])
    a3.append(args[:7] + args[9:])
    want3.append(Ez)
    for _ in range(500):
        S = (rng.uniform(0.1, 2), -rng.uniform(0.1, 2), rng.uniform(0.1, 2), -rng.uniform(0.1, 2))
        ct = rng.uniform(-0.7, 0.7)
        st = math.sqrt(1 - ct * ct)
        Ez, BnU, BnD, ByR, ByL = rng.normal(size=5)
        full = (*S, ct, st, Ez, Ez, Ez, Ez, BnU, BnD, ByR, ByL)
        a4.append((*S, ct, st, Ez, BnU, BnD, ByR, ByL))
        want4.append(oracle.twod_rs_ez_4state(*full))
        S3 = [rng.uniform(0.1, 2) * sg for sg in (1, -1, 1, -1, 1, -1)]
        Ez, b1, b2, b3 = rng.normal(size=4)
        a3.append((*S3, Ez, b1, b2, b3))
        want3.append(oracle.twod_rs_ez_3state(*S3, Ez, Ez, Ez, b1, b2, b3))
    got4 = cs.twod_rs_ez(4, np.array(a4))
    got3 = cs.twod_rs_ez(3, np.array(a3))
    assert got4[0] == pytest.approx(-0.435, abs=1e-14)
    assert got3[0] == pytest.approx(0.55, abs=1e-14)
    np.testing.assert_allclose(got4, want4, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(got3, want3, rtol=1e-12, atol=1e-13)
