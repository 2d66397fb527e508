"""ORACLE -- test infrastructure only.

ctypes wrapper of ``oracle/liboracle.so``, the CPU restatement of the
CubeSphere per-stage update (``oracle/oracle.cpp``).  Only the tests,
``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py`` use it,
and only as the checker / the timed CPU reference; the library never calls
it.  Parity status: see the header of ``oracle/oracle_core.h``.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "liboracle.so"
_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} missing: run `python -m cubesphere_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    P, D, dp = ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int32)
    sig = {
        "oracle_create": ([P], P),
        "oracle_destroy": ([P], None),
        "oracle_set_geometry": ([P, ctypes.c_int, dp], None),
        "oracle_set_mask_stencil": ([P, ip, ip], None),
        "oracle_set_state": ([P, dp, dp, dp, dp, dp], None),
        "oracle_get_state": ([P, dp, dp, dp, dp, dp], None),
        "oracle_debug_get": ([P, ctypes.c_int, dp], ctypes.c_int),
        "oracle_update": ([P, D], None),
        "oracle_evaluate_timestep": ([P, D], D),
        "oracle_stage": ([P, ctypes.c_int, D], None),
        "oracle_step": ([P, D], D),
        "oracle_twod_rs_ez_4state": ([dp], D),
        "oracle_twod_rs_ez_3state": ([dp], D),
        "oracle_build_mesh": ([P, ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
        "oracle_init_problem": ([P, P, ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
        "oracle_get_geometry": ([P, ctypes.c_int, dp], None),
        "oracle_get_mask_stencil": ([P, ip, ip], None),
        "oracle_pointwise": ([P, ctypes.c_int, ctypes.c_int, dp, dp], ctypes.c_int),
        "oracle_limit_minmax": ([P, dp, dp], ctypes.c_int),
        "oracle_stage_phase": ([P, ctypes.c_int, ctypes.c_int, D, ctypes.c_uint], ctypes.c_int),
        "oracle_evaluate_timestep_panels": ([P, D, ctypes.c_uint], D),
        "oracle_set_panel_rule": ([P, ctypes.c_int], None),
        "oracle_stage_array": ([P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)], dp),
    }
    for n in ("oracle_fill_ghosts", "oracle_limit_all_slopes_p12", "oracle_make_facial_fluxes",
              "oracle_make_edge_efields", "oracle_build_non_stiff_sources", "oracle_cleanup"):
        sig[n] = ([P], None)
    for n, (a, r) in sig.items():
        f = getattr(lib, n)
        f.argtypes = a
        f.restype = r
    _lib = lib
    return lib


def _d(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


STATE_KEYS = ("U", "ent", "bxf", "byf", "bzf")
DEBUG_WHICH = {"V": 0, "ent_modes": 1, "flatten": 2, "dUdt": 3, "Efx": 4, "Efy": 5, "Efz": 6, "Bxq": 7,
               "Byq": 8, "Bzq": 9, "E1": 10, "speeds": 11, "entflux": 12, "positivity": 13}
DEBUG_NCOMP = {"V": 80, "ent_modes": 4, "flatten": 1, "dUdt": 8, "Efx": 1, "Efy": 1, "Efz": 1, "Bxq": 5,
               "Byq": 5, "Bzq": 5, "E1": 3, "speeds": 6, "entflux": 3, "positivity": 1}


class _Shape:
    """Panel-box shapes of a parameter set (the library's layout)."""

    def __init__(self, params):
        self.params = params
        self.N, self.nr, self.G = params.ntp, params.nr, params.nghost
        self.NI = self.NJ = self.N + 2 * self.G + 1
        self.NK = self.nr + 2 * self.G + 1

    def shape(self, ncomp: int) -> tuple:
        return (ncomp, 6, self.NK, self.NJ, self.NI)

    def zeros(self, ncomp: int) -> np.ndarray:
        return np.zeros(self.shape(ncomp), dtype=np.float64)

    def empty_state(self) -> dict:
        return {"U": self.zeros(8), "ent": self.zeros(1), "bxf": self.zeros(1), "byf": self.zeros(1),
                "bzf": self.zeros(1)}

    def interior(self, a: np.ndarray) -> np.ndarray:
        G, N, nr = self.G, self.N, self.nr
        return a[..., G + 1:G + nr + 1, G + 1:G + N + 1, G + 1:G + N + 1]


class Oracle:
    """CPU solve.  Given a library Solve, it runs on that solve's geometry,
    mask and stencil; given ``params`` (a ``cubesphere_b200.CsParams``)
    instead, it builds its own mesh with the host mesh builder compiled into
    ``liboracle.so`` and needs no other library (``init_problem`` then
    writes the seeded initial state)."""

    def __init__(self, solve=None, params=None, mesh: bool = True):
        self.lib = load()
        if solve is None and params is None:
            raise ValueError("Oracle needs a Solve or a parameter set")
        self.s = solve if solve is not None else _Shape(params)
        self.h = self.lib.oracle_create(ctypes.byref(self.s.params))
        if solve is None:
            if not mesh:  # pointwise physics only
                return
            why = ctypes.create_string_buffer(256)
            if self.lib.oracle_build_mesh(self.h, why, 256):
                raise RuntimeError("oracle mesh build failed: " + why.value.decode())
            return
        from cubesphere_b200 import GEOM_FIELDS
        for f, name in enumerate(GEOM_FIELDS):
            g = np.ascontiguousarray(solve.geometry(name))
            self.lib.oracle_set_geometry(self.h, f, _d(g))
        m = np.ascontiguousarray(solve.mask())
        st = np.ascontiguousarray(solve.stencil())
        self.lib.oracle_set_mask_stencil(self.h, _i(m), _i(st))

    def pointwise(self, kind: int, cases: np.ndarray) -> np.ndarray:
        """The pointwise physics on rows of ``cases`` (the layouts of the
        library's ``cs_pointwise``): kind 0 PRIM_TO_CONS, 1 CONS_TO_PRIM,
        2 the HLL solve."""
        nin, nout = {0: (9, 8), 1: (9, 18), 2: (18, 35)}[kind]
        a = np.ascontiguousarray(cases, dtype=np.float64).reshape(-1, nin)
        out = np.zeros((a.shape[0], nout))
        assert self.lib.oracle_pointwise(self.h, kind, a.shape[0], _d(a), _d(out)) == 0
        return out

    def limit_minmax(self):
        """STEP 10 of the last LIMIT_ALL_SLOPES_P12: (v_min[9], v_max[9])."""
        vmin, vmax = np.zeros(9), np.zeros(9)
        assert self.lib.oracle_limit_minmax(self.h, _d(vmin), _d(vmax)) == 0
        return vmin, vmax

    def init_problem(self, desc) -> None:
        """The seeded initial state of a ``cubesphere_b200.CsInitDesc``."""
        why = ctypes.create_string_buffer(256)
        if self.lib.oracle_init_problem(self.h, ctypes.byref(desc), why, 256):
            raise RuntimeError("oracle initial state failed: " + why.value.decode())

    def geometry(self, f: int) -> np.ndarray:
        from cubesphere_b200 import GEOM_NCOMP
        out = self.s.zeros(GEOM_NCOMP[f])
        self.lib.oracle_get_geometry(self.h, f, _d(out))
        return out

    def mask_stencil(self):
        m = np.zeros((6, self.s.NK, self.s.NJ, self.s.NI), dtype=np.int32)
        st = np.zeros((6, 12, 2, self.s.NJ, self.s.NI), dtype=np.int32)
        self.lib.oracle_get_mask_stencil(self.h, _i(m), _i(st))
        return m, st

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def put_state(self, st: dict):
        self.lib.oracle_set_state(self.h, *[_d(np.ascontiguousarray(st[k])) for k in STATE_KEYS])

    def get_state(self) -> dict:
        st = self.s.empty_state()
        self.lib.oracle_get_state(self.h, *[_d(st[k]) for k in STATE_KEYS])
        return st

    def debug(self, name: str) -> np.ndarray:
        out = self.s.zeros(DEBUG_NCOMP[name])
        rc = self.lib.oracle_debug_get(self.h, DEBUG_WHICH[name], _d(out))
        assert rc == 0
        return out

    def fill_ghosts(self):
        self.lib.oracle_fill_ghosts(self.h)

    def limit_all_slopes_p12(self):
        self.lib.oracle_limit_all_slopes_p12(self.h)

    def make_facial_fluxes(self):
        self.lib.oracle_make_facial_fluxes(self.h)

    def make_edge_efields_p1(self):
        self.lib.oracle_make_edge_efields(self.h)

    def build_non_stiff_sources(self):
        self.lib.oracle_build_non_stiff_sources(self.h)

    def update_imex_rk_step_p1(self, dt: float):
        self.lib.oracle_update(self.h, dt)

    def cleanup_after_update(self):
        self.lib.oracle_cleanup(self.h)

    def evaluate_timestep(self, dtcur: float) -> float:
        return self.lib.oracle_evaluate_timestep(self.h, dtcur)

    def stage(self, irk: int, dtcur: float):
        self.lib.oracle_stage(self.h, irk, dtcur)

    def step(self, dtcur: float) -> float:
        return self.lib.oracle_step(self.h, dtcur)

    # A stage in phases over a set of panels (bit p of `panels` = panel p),
    # for runs in which ranks hold some of the panels and exchange between
    # the phases: 0 radial padding, 1 reconstruction + face fluxes, 2 flux
    # scatter + edge EMFs, 3 the rest of the stage.
    def stage_phase(self, phase: int, irk: int = 1, dtcur: float = 0.0, panels: int = 63):
        assert self.lib.oracle_stage_phase(self.h, phase, irk, dtcur, panels) == 0

    def set_panel_rule(self, rule: int):
        """Value of the copies of a shared face or edge: 0 the lowest-numbered
        panel's (the library's default), 1 their average (the reference's
        defect correction; what CS_FLAG_PANEL_AVERAGE selects)."""
        self.lib.oracle_set_panel_rule(self.h, rule)

    def evaluate_timestep_panels(self, dtcur: float, panels: int) -> float:
        return self.lib.oracle_evaluate_timestep_panels(self.h, dtcur, panels)

    def stage_array(self, which: str, d: int) -> np.ndarray:
        """In-place view of a stage array: "cL" / "cR" (direction d's one-sided
        face contributions, (5 * 8, 6 * box)), "EF" (entropy flux) or "Ef"
        (EMF component d), (6 * box)."""
        n = ctypes.c_size_t(0)
        ptr = self.lib.oracle_stage_array(self.h, ("cL", "cR", "EF", "Ef").index(which), d, ctypes.byref(n))
        assert ptr
        a = np.ctypeslib.as_array(ptr, shape=(n.value,))
        return a.reshape(40, -1) if which in ("cL", "cR") else a


def twod_rs_ez_4state(S_R, S_L, S_U, S_D, cos_t, sin_t, Ez_RU, Ez_LU, Ez_LD, Ez_RD, Bneta_U, Bneta_D, By_R, By_L):
    """Two_D_RS_Ez_4State_HLL (630_2d_rs_ez_two_d_rs_ez_4state_hll.f:10): ESSz."""
    a = np.array([S_R, S_L, S_U, S_D, cos_t, sin_t, Ez_RU, Ez_LU, Ez_LD, Ez_RD, Bneta_U, Bneta_D, By_R, By_L],
                 dtype=np.float64)
    return load().oracle_twod_rs_ez_4state(_d(a))


def twod_rs_ez_3state(S_R1, S_L1, S_R2, S_L2, S_R3, S_L3, Ez_1, Ez_2, Ez_3, Bneta_1, Bneta_2, Bneta_3):
    """Two_D_RS_Ez_3State_HLL (631_2d_rs_ez_two_d_rs_ez_3state_hll.f:9): ESSz."""
    a = np.array([S_R1, S_L1, S_R2, S_L2, S_R3, S_L3, Ez_1, Ez_2, Ez_3, Bneta_1, Bneta_2, Bneta_3], dtype=np.float64)
    return load().oracle_twod_rs_ez_3state(_d(a))
