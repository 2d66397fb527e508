"""Invariants of the CPU oracle (no GPU): CT keeps div B at round-off across
panel edges when every shared face and edge has one owner, and the ghost
fill is a pure copy of neighbour values."""
import numpy as np
import pytest

import cubesphere_b200 as cs
from oracle import Oracle


def _setup(flags, **over):
    pr = cs.preset("shell16")
    pr["params"].update(over)
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build(device=False)
    st = s.init_problem_host(**pr["init"])
    o = Oracle(s)
    o.put_state(st)
    return s, o, st


def _divb(s, st):
    G, N, nr = s.G, s.N, s.nr
    vol = s.geometry("V_VOL")[0]
    A = [s.geometry(n)[0] for n in ("XF_AREA", "YF_AREA", "ZF_AREA")]
    bx, by, bz = st["bxf"][0], st["byf"][0], st["bzf"][0]

    def sl(a, di, dj, dk):
        return a[:, G + 1 + dk:G + nr + 1 + dk, G + 1 + dj:G + N + 1 + dj, G + 1 + di:G + N + 1 + di]

    div = (sl(A[0] * bx, 0, 0, 0) - sl(A[0] * bx, -1, 0, 0) + sl(A[1] * by, 0, 0, 0) - sl(A[1] * by, 0, -1, 0) +
           sl(A[2] * bz, 0, 0, 0) - sl(A[2] * bz, 0, 0, -1))
    return float(np.abs(div / sl(vol, 0, 0, 0)).max() / np.abs(sl(bx, 0, 0, 0)).max())


def test_initial_field_is_divergence_free():
    s, o, st = _setup(0)
    assert _divb(s, st) < 1e-12


@pytest.mark.parametrize("rk", [cs.CS_RK2, cs.CS_IMEX_RK2])
def test_panel_edge_ownership_keeps_div_b_at_roundoff(rk):
    s, o, st = _setup(0, rk_scheme=rk)
    dt = o.evaluate_timestep(1e30)
    for _ in range(2):
        dt = o.step(dt)
    assert _divb(s, o.get_state()) < 1e-12


def test_per_panel_edges_let_div_b_grow():
    """Without ownership each panel evolves its copy of a shared face with
    its own EMFs; the copies drift apart near the cube corners."""
    s, o, st = _setup(cs.CS_FLAG_NO_PANEL_SYNC, rk_scheme=cs.CS_RK2)
    dt = o.evaluate_timestep(1e30)
    dt = o.step(dt)
    assert _divb(s, o.get_state()) > 1e-6


def test_ghost_fill_copies_neighbour_interior_values():
    s, o, st = _setup(0)
    o.fill_ghosts()
    g = o.get_state()
    G, N = s.G, s.N
    # right ghost strip of panel 0 holds the right neighbour's interior (k in the interior)
    rt = 2  # panel 1's right neighbour is panel 3 (1-based) -> index 2
    U = g["U"][0]
    for k in range(G + 1, G + s.nr + 1):
        for j in range(1, N + 1):
            for i in range(N + 1, N + G + 1):
                src = U[rt, k, G + (2 * N + 1 - i), G + j]
                assert U[0, k, G + j, G + i] == src
