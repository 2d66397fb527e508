"""Special initial states for known-answer and branch-coverage tests, built
on the geometry of a Solve (or a standalone oracle's shape) with numpy.

* ``linear_state``: every primitive linear in the zone centroid and the
  divergence-free field B = b (x, -2y, z) of the reference's manufactured
  problem (iproblem 0, 801:105-225); face B the B-field quadrature average
  of B . n over each face.  STEPS 7.a / 7.b reproduce such a field exactly
  (the one-sided 3x3 stencils and the quadratic least squares all return
  the gradient of a linear function, and the higher modes vanish), and the
  ADP solve (STEP 8.d) returns the linear B modes, in every zone whose
  stencils do not reach the radial padding.
* ``uniform_state``: uniform rho, p, v = 0 and a uniform field.
* ``positivity_state``: the seeded shell state with six Gaussian blobs of
  deep pressure dips and density bumps, which makes STEP 7.c shrink the
  higher modes of some zones and give up in others.
"""
import numpy as np

GAMMA = 5.0 / 3.0
LIN = np.array([[2.0, 0.1, -0.05, 0.08], [0.1, 0.02, 0.01, -0.03], [-0.1, 0.01, 0.02, 0.01],
                [0.05, -0.01, 0.01, 0.02], [3.0, 0.2, 0.1, -0.1]])
LIN_B = 0.3


def cons_from_prims(rho, v, p, B, gamma=GAMMA):
    U = np.zeros((8,) + np.shape(rho))
    U[0] = rho
    U[1:4] = rho * v
    U[4] = p / (gamma - 1) + 0.5 * rho * (v ** 2).sum(0) + (B ** 2).sum(0) / (8 * np.pi)
    U[5:8] = B
    return U


def prims_from_cons(U, gamma=GAMMA):
    rho = U[0]
    safe = np.where(rho > 0, rho, 1.0)
    v = U[1:4] / safe
    B = U[5:8]
    p = (gamma - 1) * (U[4] - 0.5 * rho * (v ** 2).sum(0) - (B ** 2).sum(0) / (8 * np.pi))
    return rho, v, p, B


def face_field(s, bfun):
    """Face-normal B: the B-field quadrature average of bfun(x, y, z) . n."""
    out = {}
    for d, (k, QP, BW, NF) in enumerate((("bxf", "XF_QP", "XB_QW", "XF_N"), ("byf", "YF_QP", "YB_QW", "YF_N"),
                                         ("bzf", "ZF_QP", "ZB_QW", "ZF_N"))):
        qp, qw, nf = s.geometry(QP), s.geometry(BW), s.geometry(NF)
        acc = 0.0
        for q in range(5):
            bx, by, bz = bfun(qp[q], qp[5 + q], qp[10 + q])
            n = (nf[q], nf[5 + q], nf[10 + q]) if d == 2 else (nf[0], nf[1], nf[2])
            acc = acc + qw[q] * (bx * n[0] + by * n[1] + bz * n[2])
        out[k] = acc[None]
    return out


def _finish(s, U, p, rho, bfun, act):
    st = s.empty_state()
    st["U"] = np.where(act[None], U, 0.0)
    st["ent"][0] = np.where(act, p / np.where(rho > 0, rho, 1.0) ** (GAMMA - 1), 0.0)
    st.update(face_field(s, bfun))
    return st


def linear_state(s):
    x, y, z = s.geometry("V_CEN")
    act = s.mask() == 1
    rho, vx, vy, vz, p = [r[0] + r[1] * x + r[2] * y + r[3] * z for r in LIN]
    B = np.stack([LIN_B * x, -2 * LIN_B * y, LIN_B * z])
    U = cons_from_prims(rho, np.stack([vx, vy, vz]), p, B)
    return _finish(s, U, p, rho, lambda a, b, c: (LIN_B * a, -2 * LIN_B * b, LIN_B * c), act)


def linear_gradients():
    """Per primitive component: (value, d/dx, d/dy, d/dz) of linear_state."""
    g = {c: LIN[c] for c in range(5)}
    g[5] = (0.0, LIN_B, 0.0, 0.0)
    g[6] = (0.0, 0.0, -2 * LIN_B, 0.0)
    g[7] = (0.0, 0.0, 0.0, LIN_B)
    return g


QUAD_A = {0: 2.0, 1: 0.1, 2: -0.2, 3: 0.05, 4: 3.0}
QUAD_G = {0: (0.1, -0.05, 0.08), 1: (0.02, 0.01, -0.03), 2: (0.01, 0.02, 0.01), 3: (-0.01, 0.01, 0.02),
          4: (0.2, 0.1, -0.1)}
QUAD_H = {0: ((0.04, 0.01, -0.02), (0.01, 0.03, 0.005), (-0.02, 0.005, 0.05)),
          1: ((0.01, 0.002, 0.0), (0.002, -0.01, 0.003), (0.0, 0.003, 0.02)),
          2: ((-0.02, 0.0, 0.004), (0.0, 0.01, 0.002), (0.004, 0.002, 0.01)),
          3: ((0.01, -0.003, 0.0), (-0.003, 0.02, 0.001), (0.0, 0.001, -0.01)),
          4: ((0.06, 0.02, 0.01), (0.02, -0.03, 0.01), (0.01, 0.01, 0.05))}


def quadratic_state(s):
    """rho, v, p quadratic in the global coordinates (QUAD_A + QUAD_G . X +
    X . QUAD_H . X / 2), each zone holding the exact zone average of its
    primitive (the centroid value plus the second moments from the zone's
    Taylor-basis coefficients: avg = q(c) + l^2 (H_xx C5 + H_yy C6 + H_zz C7)
    / 2 + l^2 (H_xy C8 + H_yz C9 + H_xz C10)), and the linear
    divergence-free field of linear_state.  Third-order stencils reproduce
    its modes exactly: slopes l grad q(c), square modes l^2 H_aa / 2, cross
    modes l^2 H_ab."""
    x, y, z = s.geometry("V_CEN")
    l = s.geometry("V_SCALE")[0]
    C = s.geometry("COEF")
    act = s.mask() == 1
    prim = {}
    for c in range(5):
        g, H = np.array(QUAD_G[c]), np.array(QUAD_H[c])
        X = (x, y, z)
        val = QUAD_A[c] + sum(g[a] * X[a] for a in range(3)) + 0.5 * sum(
            H[a, b] * X[a] * X[b] for a in range(3) for b in range(3))
        mom = 0.5 * (H[0, 0] * C[4] + H[1, 1] * C[5] + H[2, 2] * C[6]) + H[0, 1] * C[7] + H[1, 2] * C[8] + H[0, 2] * C[9]
        prim[c] = val + l * l * mom
    B = np.stack([LIN_B * x, -2 * LIN_B * y, LIN_B * z])
    U = cons_from_prims(prim[0], np.stack([prim[1], prim[2], prim[3]]), prim[4], B)
    return _finish(s, U, prim[4], prim[0], lambda a, b, c: (LIN_B * a, -2 * LIN_B * b, LIN_B * c), act)


def quadratic_modes(s):
    """Per primitive 0..4: the exact modes 2..10 of quadratic_state, shape
    (9,) + box."""
    x, y, z = s.geometry("V_CEN")
    l = s.geometry("V_SCALE")[0]
    out = {}
    for c in range(5):
        g, H = np.array(QUAD_G[c]), np.array(QUAD_H[c])
        X = (x, y, z)
        grad = [g[a] + sum(H[a, b] * X[b] for b in range(3)) for a in range(3)]
        out[c] = np.stack([l * grad[0], l * grad[1], l * grad[2],
                           0.5 * l * l * H[0, 0] + 0 * x, 0.5 * l * l * H[1, 1] + 0 * x, 0.5 * l * l * H[2, 2] + 0 * x,
                           l * l * H[0, 1] + 0 * x, l * l * H[1, 2] + 0 * x, l * l * H[0, 2] + 0 * x])
    return out


def linear_state_e_averages(s):
    """Zone averages of E = -v x B for linear_state, per component (shape
    box): v and B are linear, so E is quadratic with Hessian -(gv_a gB_b^T +
    gB_b gv_a^T - gv_b gB_a^T - gB_a gv_b^T), and its zone average is the
    centroid value plus the second-moment terms (quadratic_state)."""
    x, y, z = s.geometry("V_CEN")
    l = s.geometry("V_SCALE")[0]
    C = s.geometry("COEF")
    X = np.stack([x, y, z])
    gv = [np.array(LIN[c][1:]) for c in (1, 2, 3)]
    v0 = [LIN[c][0] for c in (1, 2, 3)]
    gB = [np.array([LIN_B, 0.0, 0.0]), np.array([0.0, -2 * LIN_B, 0.0]), np.array([0.0, 0.0, LIN_B])]
    val = lambda f0, g: f0 + np.tensordot(g, X, 1)
    out = []
    for a, b in ((1, 2), (2, 0), (0, 1)):
        e = -(val(v0[a], gv[a]) * val(0.0, gB[b]) - val(v0[b], gv[b]) * val(0.0, gB[a]))
        H = -(np.outer(gv[a], gB[b]) + np.outer(gB[b], gv[a]) - np.outer(gv[b], gB[a]) - np.outer(gB[a], gv[b]))
        mom = 0.5 * (H[0, 0] * C[4] + H[1, 1] * C[5] + H[2, 2] * C[6]) + H[0, 1] * C[7] + H[1, 2] * C[8] + H[0, 2] * C[9]
        out.append(e + l * l * mom)
    return out


def uniform_state(s, B=(0.0, 0.0, 0.0), rho=1.0, p=1.0):
    act = s.mask() == 1
    shape = act.shape
    Bv = np.array(B, dtype=float)
    U = cons_from_prims(np.full(shape, rho), np.zeros((3,) + shape), np.full(shape, p),
                        np.broadcast_to(Bv[:, None, None, None, None], (3,) + shape))
    return _finish(s, U, np.full(shape, p), np.full(shape, rho), lambda a, b, c: (Bv[0] + 0 * a, Bv[1] + 0 * a,
                                                                                   Bv[2] + 0 * a), act)


def positivity_state(s, st, seed=3, width=0.05, dip=0.99, bump=5.0):
    """st (a seeded shell state) with six Gaussian blobs centred at seeded
    radii 1.2..1.8: pressure times (1 - dip * blob), density times
    (1 + bump * blob); face B and velocity unchanged."""
    rng = np.random.default_rng(seed)
    rho, v, p, B = prims_from_cons(st["U"])
    cen = s.geometry("V_CEN")
    act = rho > 0
    for _ in range(6):
        c = rng.normal(size=3)
        c = c / np.linalg.norm(c) * rng.uniform(1.2, 1.8)
        blob = np.exp(-((cen - c[:, None, None, None, None]) ** 2).sum(0) / width)
        p = p * (1 - dip * blob)
        rho = rho * (1 + bump * blob)
    out = dict(st)
    out["U"] = np.where(act[None], cons_from_prims(rho, v, p, B), 0.0)
    out["ent"] = np.where(act, p / np.where(act, rho, 1.0) ** (GAMMA - 1), 0.0)[None]
    return out


def away_from_radial_padding(s, a, m=2):
    """Interior zones whose reconstruction stencils stay clear of the radial
    padding (radial layers m+1 .. nr-m)."""
    G, N, nr = s.G, s.N, s.nr
    return a[..., G + 1 + m:G + nr + 1 - m, G + 1:G + N + 1, G + 1:G + N + 1]
