"""Serving loop (cs_serve_*): concurrent admission by device memory, the
result of a solve is the same alone and in a mix, latency statistics."""
import numpy as np
import pytest

import cubesphere_b200 as cs
from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]


def _req(ntp, nr, seed, kind=1):
    pr = cs.preset("shell16")
    params = dict(pr["params"])
    params.update(ntp=ntp, nr=nr, nghost=4 if nr > 1 else 3)
    init = dict(pr["init"])
    init.update(seed=seed, kind=kind)
    if kind == 0:
        params.update(gm=0.0, rmin=1.0, rmax=1.05, radial_mesh="uniform", rk_scheme=cs.CS_SSPRK3)
        init.update(v_amp=0.5, p0=1.0, rho_amp=0.1, a_amp=0.1)
    return params, init


def test_result_is_the_same_alone_and_in_a_mix():
    import torch

    torch.cuda.set_device(0)
    pa, ia = _req(16, 8, 11)
    srv = cs.Server(max_active=1, keep_state=True)
    a = srv.submit(3, pa, ia)
    ra = srv.wait(a)
    assert ra.status == 0
    alone = srv.state(a, cs.make_params(**pa))
    srv.close()

    srv = cs.Server(max_active=4, keep_state=True)
    others = [srv.submit(4, *_req(24, 4, 5)), srv.submit(2, *_req(16, 1, 6, kind=0))]
    a2 = srv.submit(3, pa, ia)
    others.append(srv.submit(3, *_req(32, 8, 7)))
    r2 = srv.wait(a2)
    assert r2.status == 0
    mixed = srv.state(a2, cs.make_params(**pa))
    for o in others:
        assert srv.wait(o).status == 0
    st = srv.stats()
    srv.close()
    for k in alone:
        assert np.array_equal(alone[k], mixed[k]), k
    assert ra.mass == r2.mass and ra.max_divb == r2.max_divb
    assert st["completed"] == 4 and 0 < st["p50_s"] <= st["p99_s"]
    assert st["zone_updates_per_s"] > 0


def test_request_larger_than_the_budget_is_refused():
    srv = cs.Server(max_active=2, mem_fraction=1e-6)
    rid = srv.submit(1, *_req(16, 8, 1))
    assert srv.wait(rid).status == 4  # CS_ERR_NOMEM
    srv.close()


def test_requests_on_one_mesh_share_it_and_match_a_private_build():
    """The first request on a mesh builds it; later requests with the same
    mesh parameters (different seeds) run on the cached resident mesh and
    give the same state as a solve that builds its own mesh."""
    pa, ia = _req(16, 8, 21)
    srv = cs.Server(max_active=2, keep_state=True)
    first = srv.submit(2, pa, ia)
    assert srv.wait(first).status == 0
    ids = [srv.submit(2, pa, dict(ia, seed=22 + q)) for q in range(3)]
    res = [srv.wait(i) for i in ids]
    assert srv.wait(first).mesh_reused == 0
    assert all(r.status == 0 and r.mesh_reused == 1 for r in res)
    served = srv.state(ids[-1], cs.make_params(**pa))
    srv.close()
    s = cs.Solve(**pa)
    s.mesh_build()
    s.init_problem(**dict(ia, seed=24))
    dt = s.evaluate_timestep(1e30)
    for _ in range(2):
        dt = s.step(dt)
    own = s.get_state()
    for k in own:
        assert np.array_equal(own[k], served[k]), k


def test_mesh_share_gives_the_same_steps():
    pa, ia = _req(16, 4, 31)
    a = cs.Solve(**pa)
    a.mesh_build()
    b = cs.Solve(**pa)
    b.mesh_share(a)
    for s in (a, b):
        s.init_problem(**ia)
    da, db = a.evaluate_timestep(1e30), b.evaluate_timestep(1e30)
    for _ in range(2):
        da, db = a.step(da), b.step(db)
    assert da == db
    sa, sb = a.get_state(), b.get_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
    a.close()  # the mesh lives on with b
    db = b.step(db)
    assert np.isfinite(b.get_state()["U"]).all()


def test_mesh_share_refuses_another_mesh():
    pa, _ = _req(16, 4, 1)
    pb, _ = _req(16, 8, 1)
    a = cs.Solve(**pa)
    a.mesh_build()
    b = cs.Solve(**pb)
    with pytest.raises(cs.CsError):
        b.mesh_share(a)
