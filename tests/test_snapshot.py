"""Snapshot files (checkpoint / resume): format round trip, corruption and
parameter checks on the host, and a bit-identical resume on the GPU."""
import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu


def _host_state():
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"])
    s.mesh_build(device=False)
    return s, s.init_problem_host(**pr["init"])


def test_round_trip_on_the_host(tmp_path):
    s, st = _host_state()
    path = tmp_path / "a.snap"
    assert cs.snapshot_write_host(path, s.params, st, 1.25, 3.5e-3, 17) == 0
    back = s.empty_state()
    rc, t, dt, n = cs.snapshot_read_host(path, s.params, back)
    assert (rc, t, dt, n) == (0, 1.25, 3.5e-3, 17)
    for k in st:
        assert np.array_equal(st[k], back[k]), k
    head = path.read_bytes()[:8]
    assert head == b"CSB2SNP1"


def test_corrupted_payload_and_other_parameters_are_refused(tmp_path):
    s, st = _host_state()
    path = tmp_path / "b.snap"
    assert cs.snapshot_write_host(path, s.params, st, 0.0, 1e-3, 0) == 0
    raw = bytearray(path.read_bytes())
    raw[-100] ^= 0x01
    bad = tmp_path / "bad.snap"
    bad.write_bytes(bytes(raw))
    assert cs.snapshot_read_host(bad, s.params, s.empty_state())[0] == 5  # CS_ERR_NUMERIC: hash mismatch
    other = cs.make_params(**dict(cs.preset("shell16")["params"], gamma=1.4))
    assert cs.snapshot_read_host(path, other, s.empty_state())[0] == 3  # CS_ERR_STATE: other physics


@pytest.mark.parametrize("change", [dict(rk_scheme=cs.CS_RK2), dict(rhofloor=1e-10), dict(prsfloor=1e-8),
                                    dict(cfl_coef=0.3), dict(gm=2.0), dict(smallnum=1e-14),
                                    dict(flatten_coef=0.5), dict(prs_flatten_coef=2.0), dict(bc_upper=0)])
def test_scheme_and_physics_of_a_snapshot_are_checked(tmp_path, change):
    """A snapshot resumes only under the integrator, floors, CFL number,
    gravity, limiter constants and boundary codes it was written with."""
    s, st = _host_state()
    path = tmp_path / "d.snap"
    assert cs.snapshot_write_host(path, s.params, st, 0.0, 1e-3, 0) == 0
    assert cs.snapshot_read_host(path, s.params, s.empty_state())[0] == 0
    other = cs.make_params(**dict(cs.preset("shell16")["params"], **change))
    assert cs.snapshot_read_host(path, other, s.empty_state())[0] == 3


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_resume_continues_bit_for_bit(tmp_path):
    pr = cs.preset("shell16")
    a = cs.Solve(**pr["params"])
    a.mesh_build()
    a.init_problem(**pr["init"])
    dt = a.evaluate_timestep(1e30)
    for _ in range(2):
        dt = a.step(dt)
    path = tmp_path / "c.snap"
    a.snapshot_save(path, 0.5, dt, 2)
    b = cs.Solve(**pr["params"])
    b.mesh_build()
    t, dtb, n = b.snapshot_load(path)
    assert (t, dtb, n) == (0.5, dt, 2)
    for _ in range(2):
        dt = a.step(dt)
        dtb = b.step(dtb)
    assert dt == dtb
    sa, sb = a.get_state(), b.get_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
