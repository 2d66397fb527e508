"""Batched form (cs_batch_*): independent solves of different sizes, RK
schemes and precisions advanced together by one graph launch per step give
bit for bit the results each gives alone; the launch-shape autotuner changes
no result and restores the members' states."""
import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

MEMBERS = [  # (preset, overrides, init overrides, flags)
    ("shell16", {}, {"seed": 101}, 0),
    ("surface32", {}, {"seed": 102}, 0),
    ("shell16", {"ntp": 24, "nr": 4}, {"seed": 103}, cs.CS_FLAG_FP32),
    ("shell16", {"rk_scheme": cs.CS_RK2}, {"seed": 104}, 0),
    ("shell16", {}, {"seed": 105}, 0),
]


def make(m):
    name, over, iover, flags = m
    pr = cs.preset(name)
    pr["params"].update(over)
    pr["init"].update(iover)
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build()
    s.init_problem(**pr["init"])
    return s


def alone(nsteps):
    out = []
    for m in MEMBERS:
        s = make(m)
        dt = s.evaluate_timestep(1e30)
        dt = s.steps(nsteps, dt)
        out.append((dt, s.get_state()))
        s.close()
    return out


def test_batch_matches_each_solve_alone():
    want = alone(3)
    sols = [make(m) for m in MEMBERS]
    b = cs.Batch(sols)
    dts = [s.evaluate_timestep(1e30) for s in sols]
    dts = b.steps(2, dts)
    dts = b.steps(1, dts)
    for q, s in enumerate(sols):
        dt0, st0 = want[q]
        assert dts[q] == dt0, q
        st = s.get_state()
        for k in st0:
            assert np.array_equal(st[k], st0[k]), (q, k)
    b.close()


def test_batch_is_reproducible_under_concurrency():
    """Members running side by side on the device must not change each
    other's results: four batched runs of the five members all equal the
    solves run alone, bit for bit (a STEP 7.b kernel that split each
    32-zone tile over four warps once made 15-25% of the member runs differ
    in a few tiles)."""
    want = alone(3)
    for rep in range(4):
        sols = [make(m) for m in MEMBERS]
        b = cs.Batch(sols)
        dts = b.steps(3, [s.evaluate_timestep(1e30) for s in sols])
        for q, s in enumerate(sols):
            dt0, st0 = want[q]
            assert dts[q] == dt0, (rep, q)
            st = s.get_state()
            for k in st0:
                assert np.array_equal(st[k], st0[k]), (rep, q, k)
        b.close()
        for s in sols:
            s.close()


def test_batch_of_p2_solves_matches_each_solve_alone():
    """The same members with LIMIT_ALL_SLOPES_P2 (CS_FLAG_P2: the kernels with
    the largest per-thread stacks of the library) batched side by side, twice,
    equal each solve run alone, bit for bit."""
    members = [(n, o, i, f | cs.CS_FLAG_P2) for (n, o, i, f) in MEMBERS]
    want = []
    for m in members:
        s = make(m)
        dt = s.steps(3, s.evaluate_timestep(1e30))
        want.append((dt, s.get_state()))
        s.close()
    for rep in range(2):
        sols = [make(m) for m in members]
        b = cs.Batch(sols)
        dts = b.steps(3, [s.evaluate_timestep(1e30) for s in sols])
        for q, s in enumerate(sols):
            dt0, st0 = want[q]
            assert dts[q] == dt0, (rep, q)
            st = s.get_state()
            for k in st0:
                assert np.array_equal(st[k], st0[k]), (rep, q, k)
        b.close()
        for s in sols:
            s.close()


def test_autotune_changes_no_result():
    want = alone(2)
    sols = [make(m) for m in MEMBERS]
    before = [s.get_state() for s in sols]
    b = cs.Batch(sols)
    ms = b.autotune(1)
    assert ms > 0
    for q, s in enumerate(sols):
        assert b.grid_fraction(q) in (1.0, 0.5, 0.25, 0.125)
        st = s.get_state()
        for k in st:
            assert np.array_equal(st[k], before[q][k]), (q, k)
    dts = b.steps(2, [s.evaluate_timestep(1e30) for s in sols])
    for q, s in enumerate(sols):
        dt0, st0 = want[q]
        assert dts[q] == dt0, q
        st = s.get_state()
        for k in st0:
            assert np.array_equal(st[k], st0[k]), (q, k)
    b.close()


def test_batch_refuses_a_member_without_state():
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"])
    s.mesh_build()
    with pytest.raises(cs.CsError):
        cs.Batch([s])
