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


@pytest.mark.parametrize("rk,flags", [(cs.CS_RK2, 0), (cs.CS_IMEX_RK2, 0), (cs.CS_IMEX_RK2, cs.CS_FLAG_P2),
                                     (cs.CS_IMEX_RK2, cs.CS_FLAG_PANEL_AVERAGE)])
def test_panel_edge_ownership_keeps_div_b_at_roundoff(rk, flags):
    """CT with one value on every shared face and edge (ownership, or the
    reference's averages) keeps div B at round-off whichever reconstruction
    (P12 or P2) feeds the EMFs."""
    s, o, st = _setup(flags, rk_scheme=rk)
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


def manufactured_linear_state(s):
    """The reference's manufactured field (iproblem 0, 801: exact linear U
    and B = (x, -2y, z)) on the solve's geometry: every conserved component
    a_q + b_q . centroid on the active zones, face B the quadrature average
    of B . n over each face; zero elsewhere."""
    G = s.G
    cen = s.geometry("V_CEN")
    active = s.mask() == 1  # [panel, k, j, i]
    coef = np.array([[1.0, 0.3, -0.2, 0.1], [0.2, 0.5, 0.1, -0.3], [-0.1, 0.2, 0.4, 0.1], [0.3, -0.1, 0.2, 0.6],
                     [5.0, 0.1, 0.2, 0.3], [0.1, 1.0, 0.0, 0.0], [0.0, 0.0, -2.0, 0.0], [0.0, 0.0, 0.0, 1.0]])
    st = s.empty_state()
    for q in range(8):
        val = coef[q, 0] + coef[q, 1] * cen[0] + coef[q, 2] * cen[1] + coef[q, 3] * cen[2]
        st["U"][q] = np.where(active, val, 0.0)
    st["ent"][0] = np.where(active, 1.0 + 0.1 * cen[0], 0.0)
    for d, (k, QP, QW, NF) in enumerate((("bxf", "XF_QP", "XF_QW", "XF_N"), ("byf", "YF_QP", "YF_QW", "YF_N"),
                                         ("bzf", "ZF_QP", "ZF_QW", "ZF_N"))):
        qp, qw, nf = s.geometry(QP), s.geometry(QW), s.geometry(NF)
        acc = 0.0
        for q in range(5):
            x, y, z = qp[q], qp[5 + q], qp[10 + q]
            n = (nf[q], nf[5 + q], nf[10 + q]) if d == 2 else (nf[0], nf[1], nf[2])
            acc = acc + qw[q] * (x * n[0] - 2.0 * y * n[1] + z * n[2])
        st[k][0] = acc
    return st


# interior index ranges of each field in (i, j): zones 1..N, x-faces 0..N in i, y-faces 0..N in j
_LO = {"U": (1, 1), "ent": (1, 1), "bxf": (0, 1), "byf": (1, 0), "bzf": (1, 1)}


def _outside(s, key):
    """[j, i] mask of the box points outside the field's interior range."""
    G, N = s.G, s.N
    box = np.arange(-G, N + G + 1)
    li, lj = _LO[key]
    return (box[None, :] < li) | (box[None, :] > N) | (box[:, None] < lj) | (box[:, None] > N)


def _ghost_check(s, filled, exact):
    """Ghost zones and faces (angular strips, radial interior) whose
    neighbouring zones are all active hold the manufactured values."""
    G, N, nr = s.G, s.N, s.nr
    ks = slice(G + 1, G + nr + 1)
    act = s.mask()[:, ks] == 1  # [panel, k, j, i]
    sel = _outside(s, "U")[None, None] & act
    U, Ue = filled["U"][:, :, ks], exact["U"][:, :, ks]
    assert np.count_nonzero(sel) > 0
    assert np.abs(np.where(sel[None], U - Ue, 0.0)).max() <= 1e-12 * np.abs(Ue).max()
    for d, k in enumerate(("bxf", "byf")):
        both = act & np.roll(act, -1, axis=3 - d)  # active zones on both sides of the face
        edge = np.zeros_like(both)  # the last face of the box has no zone beyond it
        if d == 0:
            edge[..., -1] = True
        else:
            edge[..., -1, :] = True
        fsel = _outside(s, k)[None, None] & both & ~edge
        B, Be = filled[k][0][:, ks], exact[k][0][:, ks]
        assert np.count_nonzero(fsel) > 0
        assert np.abs(np.where(fsel, B - Be, 0.0)).max() <= 1e-12 * np.abs(Be).max(), k


def _empty_ghosts(s, st):
    """A copy of st with every box point outside each field's interior zeroed."""
    out = {}
    for k, v in st.items():
        out[k] = np.where(_outside(s, k), 0.0, v)
    return out


def test_ghost_fill_reproduces_a_manufactured_linear_field():
    """Known answer of the reference's ghost-fill test (309, with the
    manufactured field of 801:105-225): after the fill, the ghost zones and
    faces hold the linear field evaluated on their own geometry."""
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"], flags=cs.CS_FLAG_NO_PANEL_SYNC)
    s.mesh_build(device=False)
    exact = manufactured_linear_state(s)
    start = _empty_ghosts(s, exact)  # only the fill can put the ghost values there
    o = Oracle(s)
    o.put_state(start)
    o.fill_ghosts()
    _ghost_check(s, o.get_state(), exact)


def _linear_errors(s, V):
    """Max relative error of modes 2-4 against l0 x gradient and max |mode 5-10|
    of every primitive, away from the radial padding."""
    from seeded_states import away_from_radial_padding as inner, linear_gradients

    l0 = s.geometry("V_SCALE")[0]
    out = {}
    for c, gr in linear_gradients().items():
        slope = max(np.abs(inner(s, V[m * 8 + c] - gr[m] * l0)).max() for m in range(1, 4))
        scale = max(abs(gr[m]) for m in range(1, 4)) * np.abs(inner(s, l0)).max()
        higher = max(np.abs(inner(s, V[m * 8 + c])).max() for m in range(4, 10))
        out[c] = (slope / scale, higher / scale)
    return out


def test_linear_field_is_reproduced_by_steps_7ab_and_the_adp_solve():
    """Known answer: a linear primitive field with the divergence-free
    B = b (x, -2y, z) of 801:105-225 is reproduced exactly by the WENO-AO
    stencils (7.a), the MRWENO least squares (7.b) and the ADP constrained
    least squares (8.d, B modes): slopes = l0 x gradient, higher modes 0,
    to round-off, in every zone clear of the radial padding (the ghost fill
    across panel edges included)."""
    from seeded_states import linear_state

    pr = cs.preset("shell16")
    pr["params"]["flatten_coef"] = 1e30
    s = cs.Solve(**pr["params"])
    s.mesh_build(device=False)
    o = Oracle(s)
    o.put_state(linear_state(s))
    o.fill_ghosts()
    o.limit_all_slopes_p12()
    assert np.abs(s.interior(o.debug("positivity"))).max() == 0
    for c, (slope, higher) in _linear_errors(s, o.debug("V")).items():
        assert slope < 1e-12 and higher < 1e-12, (c, slope, higher)


def _quadratic_errors(s, V, m=3):
    """Max error of modes 2-10 of primitives 0-4 against quadratic_modes,
    relative to the largest exact mode, in zones m layers clear of the
    radial padding."""
    from seeded_states import away_from_radial_padding, quadratic_modes

    ex = quadratic_modes(s)
    out = {}
    for c in range(5):
        err = max(np.abs(away_from_radial_padding(s, V[(t + 1) * 8 + c] - ex[c][t], m)).max() for t in range(9))
        out[c] = err / max(np.abs(away_from_radial_padding(s, ex[c][t], m)).max() for t in range(9))
    return out


def test_p2_reproduces_quadratic_primitives():
    """Known answer of LIMIT_ALL_SLOPES_P2 ("at third order, all stencils
    are third order", 420:2469): each zone holding the exact zone average of
    quadratic primitives, STEP 7.a's eight one-sided 9-zone stencils and the
    central least squares all return the quadratic's modes, so the WENO
    combination does too: slopes l grad q, square modes l^2 H_aa / 2, cross
    modes l^2 H_ab, to round-off, across panel edges, in zones three layers
    clear of the radial padding (P2's radial reach is two).  P12's linear
    stencils do not (its MRWENO blend keeps a truncation-size part of them)."""
    from seeded_states import quadratic_state

    errs = {}
    for flags in (cs.CS_FLAG_P2, 0):
        pr = cs.preset("shell16")
        pr["params"].update(flatten_coef=1e30, flags=flags)
        s = cs.Solve(**pr["params"])
        s.mesh_build(device=False)
        o = Oracle(s)
        o.put_state(quadratic_state(s))
        o.fill_ghosts()
        o.limit_all_slopes_p12()
        assert np.abs(s.interior(o.debug("positivity"))).max() == 0
        assert np.abs(s.interior(o.debug("flatten"))).max() == 0
        errs[flags] = _quadratic_errors(s, o.debug("V"))
    for c, e in errs[cs.CS_FLAG_P2].items():
        assert e < 1e-12, (c, e)
    assert min(errs[0].values()) > 1e-6, errs[0]


def test_p2_interpolates_a_quadratic_electric_field_to_its_zone_averages():
    """Known answer of P2's STEP 9.b (420:8553-12285): with the linear v and
    linear divergence-free B of linear_state, the zone-centred E = -v x B
    (STEP 9.a) is quadratic; the eight one-sided 10-zone interpolation
    stencils and the central 19-zone least squares all recover it, so the
    unflattened mode 1 is its zone average (centroid value plus the
    second-moment terms) to round-off, in zones two clear of the panel edges
    and five of the radial padding (the ghost zones' face-B constraints make
    the ADP inexact one and two layers out, which P2's wider stencils reach
    from the first interior rows)."""
    from seeded_states import away_from_radial_padding, linear_state, linear_state_e_averages

    pr = cs.preset("shell32")
    pr["params"].update(flatten_coef=1e30, flags=cs.CS_FLAG_P2)
    s = cs.Solve(**pr["params"])
    s.mesh_build(device=False)
    o = Oracle(s)
    o.put_state(linear_state(s))
    o.fill_ghosts()
    o.limit_all_slopes_p12()
    E1 = o.debug("E1")
    core = lambda a: away_from_radial_padding(s, a, m=5)[..., 2:-2, 2:-2]
    for q, ex in enumerate(linear_state_e_averages(s)):
        err = np.abs(core(E1[q] - ex)).max() / np.abs(core(ex)).max()
        assert err < 1e-12, (q, err)


@pytest.mark.parametrize("flags", [0, cs.CS_FLAG_P2])
def test_uniform_static_gas_stays_uniform_to_the_mesh_closure(flags):
    """A uniform gas at rest (no field, no gravity) changes in one step only
    through the discrete closure of each zone's faces (sum of area x
    quadrature-weighted normals, 2.5e-8 of the face area on shell16: the
    reference's quadrature-based areas and normals close to truncation
    error, not round-off): the pressure force on the open surface gives
    momentum of at most dt p max|closure| / V = 3.6e-8 here.  Radial layers
    the upper boundary's volume-scaled outflow copy does not reach stay
    uniform to 1e-7; the field stays zero exactly."""
    from seeded_states import uniform_state

    pr = cs.preset("shell16")
    pr["params"].update(gm=0.0, flags=flags)
    s = cs.Solve(**pr["params"])
    s.mesh_build(device=False)
    st = uniform_state(s)
    o = Oracle(s)
    o.put_state(st)
    dt = o.evaluate_timestep(1e30)
    o.step(dt)
    w = o.get_state()
    G, N, nr = s.G, s.N, s.nr
    lower = lambda a: a[..., G + 1:G + nr - 2, G + 1:G + N + 1, G + 1:G + N + 1]  # layers 1 .. nr-3
    for q in range(8):
        assert np.abs(lower(w["U"][q] - st["U"][q])).max() <= 1e-7, q
    for k in ("bxf", "byf", "bzf"):
        assert np.array_equal(w[k], st[k]), k


def test_positivity_shrinks_and_gives_up_on_the_blob_state():
    """Branch coverage of STEP 7.c (440:553-830): on the blob state some
    zones shrink their higher modes and some give up; the unperturbed state
    triggers neither."""
    from seeded_states import positivity_state

    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"])
    s.mesh_build(device=False)
    st = s.init_problem_host(**pr["init"])
    counts = []
    for state in (st, positivity_state(s, st)):
        o = Oracle(s)
        o.put_state(state)
        o.fill_ghosts()
        o.limit_all_slopes_p12()
        rec = s.interior(o.debug("positivity"))
        counts.append((int(((rec >= 2) & (rec % 2 == 0)).sum()), int((rec % 2 == 1).sum())))
        o.close()
    assert counts[0] == (0, 0)
    shrunk, gave_up = counts[1]
    assert shrunk >= 10 and gave_up >= 1, counts


def step10_numpy(s, V, st):
    """STEP 10 (421:9354-9976) restated with numpy from the zone primitives V
    (mode 0 of the reconstruction) and the face field of the state."""
    G, N, nr = s.G, s.N, s.nr
    act = s.interior(s.mask() == 1)
    v = [s.interior(V[q]) for q in range(8)]
    vmin = [float(x[act].min()) for x in v]
    vmax = [float(x[act].max()) for x in v]
    A = [s.geometry(n)[0] for n in ("XF_AREA", "YF_AREA", "ZF_AREA")]
    B = [st[k][0] for k in ("bxf", "byf", "bzf")]

    def sl(a, di, dj, dk):
        return a[:, G + 1 + dk:G + nr + 1 + dk, G + 1 + dj:G + N + 1 + dj, G + 1 + di:G + N + 1 + di]

    up = [sl(B[0], 0, 0, 0), sl(B[1], 0, 0, 0), sl(B[2], 0, 0, 0)]
    lo = [sl(B[0], -1, 0, 0), sl(B[1], 0, -1, 0), sl(B[2], 0, 0, -1)]
    a21 = (sl(A[0], 0, 0, 0) * up[0] + sl(A[1], 0, 0, 0) * up[1] + sl(A[2], 0, 0, 0) * up[2] -
           sl(A[0], -1, 0, 0) * lo[0] - sl(A[1], 0, -1, 0) * lo[1] - sl(A[2], 0, 0, -1) * lo[2])
    gam = s.params.gamma
    with np.errstate(invalid="ignore", divide="ignore"):
        ms = np.sqrt((gam * v[4] + (v[5] ** 2 + v[6] ** 2 + v[7] ** 2) / (4 * np.pi)) / v[0])
        den = np.maximum(np.maximum(np.sqrt(sum(b * b for b in up)), np.sqrt(sum(b * b for b in lo))),
                         ms * np.sqrt(4 * 3.14 * v[0]))
        dv = a21 / den
    return np.array(vmin + [float(dv[act].min())]), np.array(vmax + [float(dv[act].max())]), float(
        np.abs(sl(A[0], 0, 0, 0)).max())


def test_step10_min_max_of_the_oracle():
    """The oracle's STEP 10 against the same quantities in numpy, on the
    reconstruction of the seeded shell (B after the ADP solve)."""
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"])
    s.mesh_build(device=False)
    st = s.init_problem_host(**pr["init"])
    o = Oracle(s)
    o.put_state(st)
    o.fill_ghosts()
    o.limit_all_slopes_p12()
    vmin, vmax = o.limit_minmax()
    wmin, wmax, area = step10_numpy(s, o.debug("V"), o.get_state())
    scale = np.maximum(np.abs(wmin), np.abs(wmax))
    np.testing.assert_allclose(vmin[:8], wmin[:8], rtol=0, atol=1e-14 * scale[:8].max())
    np.testing.assert_allclose(vmax[:8], wmax[:8], rtol=0, atol=1e-14 * scale[:8].max())
    assert vmin[0] > 0 and vmin[4] > 0  # density and pressure
    # the divergence entries are round-off of a divergence-free field
    assert abs(vmin[8]) < 1e-12 * area and abs(vmax[8]) < 1e-12 * area
    assert abs(vmin[8] - wmin[8]) < 1e-13 * area and abs(vmax[8] - wmax[8]) < 1e-13 * area


@pytest.mark.parametrize("flags", [cs.CS_FLAG_PANEL_AVERAGE, cs.CS_FLAG_NO_PANEL_SYNC, 0])
def test_shared_copies_and_the_cube_symmetry(flags):
    """A spherically symmetric state (the hydrostatic shell without its
    perturbations) on panels that are exact rotations of one another stays
    the same on all six panels, to round-off, when the shared copies take
    their average (the reference's rule) or keep their own values; giving
    them the lowest-numbered panel's value breaks the symmetry near the cube
    corners by the copies' difference (truncation size)."""
    pr = cs.preset("shell16")
    s = cs.Solve(**pr["params"], flags=flags)
    s.mesh_build(device=False)
    init = dict(pr["init"], rho_amp=0.0, a_amp=0.0)
    o = Oracle(s)
    o.put_state(s.init_problem_host(**init))
    dt = o.evaluate_timestep(1e30)
    for _ in range(3):
        dt = o.step(dt)
    G, N, nr = s.G, s.N, s.nr
    rho = o.get_state()["U"][0][:, G + 1:G + nr + 1, G + 1:G + N + 1, G + 1:G + N + 1]
    asym = np.abs(rho - rho[0]).max() / np.abs(rho).max()
    if flags:
        assert asym < 1e-13
    else:
        assert asym > 1e-7
