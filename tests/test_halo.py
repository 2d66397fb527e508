"""The stage's two cross-panel exchanges as explicit lists and their split
across ranks that each own whole panels (cubesphere_b200.halo), on the CPU:
the ghost fill (cs_fill_map_get) and the panel-edge ownership of face
fluxes and edge EMFs (cs_sync_map_get), each applied on the host, reproduce
the oracle's; ranks that hold only their own panels (gloo, 2 and 3 ranks)
fill their ghost values and owned copies from their peers exactly as the
single-process application does."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

import cubesphere_b200 as cs
from cubesphere_b200.halo import (FIELDS, apply_edge_average, apply_edge_sync, apply_face_average, apply_face_sync,
                                  apply_fill_map, edge_classes)
from oracle import Oracle

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.parametrize("name", ["shell16", "surface32"])
def test_fill_map_reproduces_the_oracle_ghost_fill(name):
    """Every destination of the map in the radial interior layers (the radial
    padding overwrites the others) receives the oracle's value bit for bit,
    and no destination appears twice."""
    pr = cs.preset(name)
    s = cs.Solve(**pr["params"])
    s.mesh_build(device=False)
    st = s.init_problem_host(**pr["init"])
    src, dst, meta = s.fill_map()
    key = (meta & 7).astype(np.int64) * (1 << 40) + dst
    assert len(np.unique(key)) == len(key)
    mine = {k: v.copy() for k, v in st.items()}
    apply_fill_map(mine, src, dst, meta)
    o = Oracle(s)
    o.put_state(st)
    o.fill_ghosts()
    ref = o.get_state()
    box = s.NI * s.NJ * s.NK
    for f, k in enumerate(FIELDS):
        d = dst[(meta & 7) == f]
        kk = (d % box) // (s.NI * s.NJ) - s.G
        d = d[(kk >= 1) & (kk <= s.nr)]
        assert len(d) > 0
        assert np.array_equal(mine[k].reshape(-1)[d], ref[k].reshape(-1)[d]), k


def _oracle_fluxes_and_emfs(pr, flags):
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build(device=False)
    st = s.init_problem_host(**pr["init"])
    o = Oracle(s)
    o.put_state(st)
    o.fill_ghosts()
    o.limit_all_slopes_p12()
    o.make_facial_fluxes()
    o.make_edge_efields_p1()
    return s, o.debug("entflux"), [o.debug(k) for k in ("Efx", "Efy", "Efz")]


@pytest.mark.parametrize("name", ["shell16", "surface32"])
def test_sync_maps_reproduce_the_oracle_ownership(name):
    """The ownership lists applied on the host to the oracle's per-panel
    values (CS_FLAG_NO_PANEL_SYNC) give its synchronised entropy fluxes and
    edge EMFs bit for bit; no (offset, kind) pair is both a source and a
    destination, so the lists need no ordering."""
    pr = cs.preset(name)
    s, ef_on, e_on = _oracle_fluxes_and_emfs(pr, 0)
    _, ef_off, e_off = _oracle_fluxes_and_emfs(pr, cs.CS_FLAG_NO_PANEL_SYNC)
    for which in (0, 1):
        dst, src, dk, sk, sg = s.sync_map(which)
        assert len(dst) > 0
        d = set((dk.astype(np.int64) << 40 | dst).tolist())
        owners = (sk.astype(np.int64) << 40 | src).tolist()
        assert len(d) == len(dst)
        assert not d & set(owners)
        # one entry a face, one run of one or two entries an edge (its
        # owner's copy shared by the run only): the averaging kernels' threads
        # touch disjoint copies
        cls = edge_classes(src, sk)
        assert len(set(owners)) == len(cls) - 1
        assert set(np.diff(cls).tolist()) <= ({1} if which == 0 else {1, 2})
    dst, src, dk, sk, sg = s.sync_map(0)
    assert set(dk.tolist()) <= {0, 1} and (sg == -1).all()
    EF = [a.reshape(-1).copy() for a in ef_off]
    fcon = [np.zeros((16, EF[0].size)) for _ in range(3)]
    apply_face_sync(fcon, EF, dst, src, dk, sk)
    for q in range(3):
        assert np.array_equal(EF[q], ef_on[q].reshape(-1)), q
    dst, src, dk, sk, sg = s.sync_map(1)
    assert set(sg.tolist()) == {-1, 1}
    Ef = [a.reshape(-1).copy() for a in e_off]
    apply_edge_sync(Ef, dst, src, dk, sk, sg)
    for q in range(3):
        assert np.array_equal(Ef[q], e_on[q].reshape(-1)), q


def _oracle_stage_arrays(pr, flags):
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build(device=False)
    o = Oracle(s)
    o.put_state(s.init_problem_host(**pr["init"]))
    o.fill_ghosts()
    o.limit_all_slopes_p12()
    o.make_facial_fluxes()
    o.make_edge_efields_p1()
    fcon = [np.concatenate([o.stage_array("cL", d), o.stage_array("cR", d)]) for d in range(2)]
    return s, fcon, [o.stage_array("EF", d).copy() for d in range(3)], [o.stage_array("Ef", c).copy() for c in range(3)]


@pytest.mark.parametrize("name", ["shell16", "surface32"])
def test_average_rule_through_the_lists_reproduces_the_oracle(name):
    """CS_FLAG_PANEL_AVERAGE (the reference's rule): the averages formed
    through the exported ownership lists, in the order and grouping the
    device kernels use (each face entry on its own, each edge's entries as
    one run from its owner copy), turn the oracle's per-panel contributions,
    entropy fluxes and EMFs into its averaged ones bit for bit."""
    pr = cs.preset(name)
    s, fcon, EF, Ef = _oracle_stage_arrays(pr, cs.CS_FLAG_NO_PANEL_SYNC)
    _, fcon_avg, EF_avg, Ef_avg = _oracle_stage_arrays(pr, cs.CS_FLAG_PANEL_AVERAGE)
    dst, src, dk, sk, _ = s.sync_map(0)
    apply_face_average(fcon, EF, dst, src, dk, sk)
    for d in range(2):
        assert np.array_equal(fcon[d], fcon_avg[d]), d
    for d in range(3):
        assert np.array_equal(EF[d], EF_avg[d]), d
    dst, src, dk, sk, sg = s.sync_map(1)
    apply_edge_average(Ef, dst, src, dk, sk, sg)
    for c in range(3):
        assert np.array_equal(Ef[c], Ef_avg[c]), c
    assert not np.array_equal(Ef_avg[2], _oracle_stage_arrays(pr, 0)[3][2])  # the rules differ


def _rank(rank, world, port, panel_rank, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist

    import cubesphere_b200 as cs
    from cubesphere_b200.halo import (EdgeSync, FaceSync, GhostExchange, apply_edge_sync, apply_face_sync,
                                      apply_fill_map)

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pr = cs.preset("shell16")
        s = cs.Solve(**pr["params"])
        s.mesh_build(device=False)
        st = s.init_problem_host(**pr["init"])
        src, dst, meta = s.fill_map()
        want = {k: v.copy() for k, v in st.items()}
        apply_fill_map(want, src, dst, meta)
        owned = [p for p in range(6) if panel_rank[p] == rank]
        other = [p for p in range(6) if panel_rank[p] != rank]
        held = {k: torch.from_numpy(v.copy()) for k, v in st.items()}
        for v in held.values():
            v[:, other] = float("nan")  # this rank holds only its own panels
        box = s.NI * s.NJ * s.NK
        plan = GhostExchange(src, dst, meta, box, panel_rank, rank)
        plan.exchange(held, dist)
        ok = all(np.array_equal(held[k].numpy()[:, owned], want[k][:, owned]) for k in want)
        sent, received = plan.values_bytes(), 8 * sum(len(v) for v in plan.recv.values())

        # ownership copies of seeded face contributions and edge EMFs
        rng = np.random.default_rng(7)
        fcon = [rng.standard_normal((16, 6 * box)) for _ in range(3)]
        EF = [rng.standard_normal(6 * box) for _ in range(3)]
        Ef = [rng.standard_normal(6 * box) for _ in range(3)]
        dst_f, src_f, dk_f, sk_f, _ = s.sync_map(0)
        dst_e, src_e, dk_e, sk_e, sg_e = s.sync_map(1)
        w_fcon, w_EF, w_Ef = [a.copy() for a in fcon], [a.copy() for a in EF], [a.copy() for a in Ef]
        apply_face_sync(w_fcon, w_EF, dst_f, src_f, dk_f, sk_f)
        apply_edge_sync(w_Ef, dst_e, src_e, dk_e, sk_e, sg_e)

        def hold(a):
            t = torch.from_numpy(a.copy())
            v = t.view(-1, 6, box)
            v[:, other] = float("nan")
            return t

        h_fcon, h_EF, h_Ef = [hold(a) for a in fcon], [hold(a) for a in EF], [hold(a) for a in Ef]
        fs = FaceSync(dst_f, src_f, dk_f, sk_f, box, panel_rank, rank)
        fs.exchange(h_fcon, h_EF, dist)
        es = EdgeSync(dst_e, src_e, dk_e, sk_e, sg_e, box, panel_rank, rank)
        es.exchange(h_Ef, dist)
        mine = lambda a: a.reshape(-1, 6, box)[:, owned]
        for got, ref in zip(h_fcon + h_EF + h_Ef, w_fcon + w_EF + w_Ef):
            ok = ok and np.array_equal(mine(got.numpy()), mine(ref))
        sent += fs.values_bytes(17) + es.values_bytes()
        received += 8 * (17 * sum(len(v) for v in fs.recv.values()) + sum(len(v) for v in es.recv.values()))
        q.put((rank, ok, sent, received))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("panel_rank", [[0, 0, 0, 1, 1, 1], [0, 0, 1, 1, 2, 2]])
def test_panel_split_exchanges_match_the_single_process_application(panel_rank):
    world = max(panel_rank) + 1
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29900 + os.getpid() % 1000 + world
    procs = [ctx.Process(target=_rank, args=(r, world, port, panel_rank, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, sent, received in out:
        assert ok, rank
        assert sent > 0 and received > 0, rank
    # every value one rank sends, another receives
    assert sum(o[2] for o in out) == sum(o[3] for o in out)


def _sharded_rank(rank, world, port, name, flags, panel_rank, nsteps, q):
    """Whole steps of the oracle on a rank that holds only its own panels:
    each stage runs over them alone, with the ghost fill, the face-flux and
    the EMF ownership exchanged between its phases and the time step's
    minimum all-reduced.  Puts the time steps and its panels' state."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="2")
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist

    import cubesphere_b200 as cs
    from cubesphere_b200.halo import EdgeSync, FaceSync, GhostExchange
    from oracle import Oracle

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pr = cs.preset(name)
        s = cs.Solve(**pr["params"], flags=flags)
        s.mesh_build(device=False)
        st = s.init_problem_host(**pr["init"])
        box = s.NI * s.NJ * s.NK
        owned = [p for p in range(6) if panel_rank[p] == rank]
        other = [p for p in range(6) if panel_rank[p] != rank]
        mask = sum(1 << p for p in owned)
        fill = GhostExchange(*s.fill_map(), box, panel_rank, rank)
        dst, src, dk, sk, _ = s.sync_map(0)
        face = FaceSync(dst, src, dk, sk, box, panel_rank, rank, ncomp=80)
        edge = EdgeSync(*s.sync_map(1), box, panel_rank, rank)
        o = Oracle(s)
        held = {k: v.copy() for k, v in st.items()}
        for v in held.values():
            v[:, other] = np.nan
        o.put_state(held)

        def all_min(x):
            t = torch.tensor([x], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
            return float(t[0])

        dts = [all_min(o.evaluate_timestep_panels(1e30, mask))]
        nst = 3 if s.params.rk_scheme == cs.CS_SSPRK3 else 2
        for _ in range(nsteps):
            for irk in range(1, nst + 1):
                cur = o.get_state()
                fill.exchange({k: torch.from_numpy(v) for k, v in cur.items()}, dist)
                o.put_state(cur)
                o.stage_phase(0, panels=mask)
                o.stage_phase(1, panels=mask)
                cL = [o.stage_array("cL", d) for d in range(2)]
                cR = [o.stage_array("cR", d) for d in range(2)]
                fcon = [torch.from_numpy(np.concatenate([cL[d], cR[d]])) for d in range(2)]
                face.exchange(fcon, [torch.from_numpy(o.stage_array("EF", d)) for d in range(2)], dist)
                for d in range(2):
                    cL[d][:] = fcon[d][:40].numpy()
                    cR[d][:] = fcon[d][40:].numpy()
                o.stage_phase(2, panels=mask)
                edge.exchange([torch.from_numpy(o.stage_array("Ef", c)) for c in range(3)], dist)
                o.stage_phase(3, irk, dts[-1], panels=mask)
            dts.append(all_min(o.evaluate_timestep_panels(dts[-1], mask)))
        got = o.get_state()
        q.put((rank, owned, dts, {k: v[:, owned] for k, v in got.items()}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,flags,panel_rank", [("shell16", 0, [0, 0, 0, 1, 1, 1]),
                                                   ("surface32", 0, [0, 0, 1, 1, 2, 2]),
                                                   ("shell16", cs.CS_FLAG_P2, [0, 1, 0, 1, 0, 1])])
def test_panel_sharded_steps_match_the_single_process_solve(name, flags, panel_rank):
    """The two exchange lists (plus the time step's all-reduce) are all a
    panel-sharded stage needs: ranks that hold only their own panels and run
    every stage phase over them alone end two whole steps (IMEX-RK2 with
    gravity on shell16, also with LIMIT_ALL_SLOPES_P2 and interleaved
    panels; SSP-RK3 on surface32) with the single-process oracle's state on
    their panels and its time steps, bit for bit."""
    world = max(panel_rank) + 1
    nsteps = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000 + 7 * world
    procs = [ctx.Process(target=_sharded_rank, args=(r, world, port, name, flags, panel_rank, nsteps, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=600) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pr = cs.preset(name)
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build(device=False)
    o = Oracle(s)
    o.put_state(s.init_problem_host(**pr["init"]))
    dts = [o.evaluate_timestep(1e30)]
    for _ in range(nsteps):
        dts.append(o.step(dts[-1]))
    want = o.get_state()
    for rank, owned, got_dts, got in out:
        assert got_dts == dts, rank
        for k in want:
            assert np.array_equal(got[k], want[k][:, owned]), (rank, k)
