"""The ghost exchange as an explicit list (cs_fill_map_get) and its split
across ranks that each own whole panels (cubesphere_b200.halo), on the CPU:
the list applied on the host reproduces the oracle's ghost fill, and ranks
that hold only their own panels (gloo, 2 and 3 ranks) fill their ghost
values from their peers exactly as the single-process fill does."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

import cubesphere_b200 as cs
from cubesphere_b200.halo import FIELDS, apply_fill_map
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


def _rank(rank, world, port, panel_rank, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist

    import cubesphere_b200 as cs
    from cubesphere_b200.halo import PanelSplit, apply_fill_map

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
        plan = PanelSplit(src, dst, meta, s.NI * s.NJ * s.NK, panel_rank, rank)
        plan.exchange(held, dist)
        ok = all(np.array_equal(held[k].numpy()[:, owned], want[k][:, owned]) for k in want)
        q.put((rank, ok, plan.values_bytes(), sum(len(v) for v in plan.recv.values())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("panel_rank", [[0, 0, 0, 1, 1, 1], [0, 0, 1, 1, 2, 2]])
def test_panel_split_exchange_matches_the_single_process_fill(panel_rank):
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
    assert sum(o[2] for o in out) == 8 * sum(o[3] for o in out)
