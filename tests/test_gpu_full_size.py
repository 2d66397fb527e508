"""The shell workload at its stated size (6 x 128^2 x 64 zones, 4 ghost
layers, radii 1..2 with stretch 1.02, IMEX-RK2 with implicit point-mass
gravity): one whole step on the device against the oracle, from the
oracle's own seeded initial state (the oracle builds its mesh with the
host mesh builder compiled into it and runs on all host threads; about
40 GB of host memory).  Tolerance as in test_gpu_parity: 1e-12 relative."""
import os

import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]


def test_shell128_one_step_matches_oracle():
    from oracle import Oracle
    from test_gpu_parity import TOL_STATE, check_state

    pr = cs.preset("shell128")
    o = Oracle(params=cs.make_params(**pr["params"]))
    o.init_problem(cs.make_init(**pr["init"]))
    st = o.get_state()
    s = cs.Solve(**pr["params"])
    s.mesh_build()
    s.put_state(st)
    dt_s = s.evaluate_timestep(1e30)
    dt_o = o.evaluate_timestep(1e30)
    assert abs(dt_s - dt_o) <= TOL_STATE * dt_o
    dt_s = s.step(dt_s)
    dt_o = o.step(dt_o)
    assert abs(dt_s - dt_o) <= TOL_STATE * dt_o, (dt_s, dt_o)
    check_state(s, s.get_state(), o.get_state())
    s.close()
    o.close()
