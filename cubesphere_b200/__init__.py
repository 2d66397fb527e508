"""B200 per-stage volume update of the CubeSphere cubed-sphere MHD code.

Python mirror of the reference's riemann_integrate call sequence on top of
the C ABI in ``include/cubesphere_b200.h`` (``libcubesphere_b200.so``, built
in-tree by ``python -m cubesphere_b200.build``).  The compute path is the
CUDA library; there is no CPU fallback: every entry point that computes
raises when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from .configs import PRESETS, preset  # noqa: F401

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libcubesphere_b200.so"

GEOM_FIELDS = [
    "VERT", "XF_QP", "XF_QW", "XF_N", "XF_AREA", "XF_CEN",
    "YF_QP", "YF_QW", "YF_N", "YF_AREA", "YF_CEN",
    "ZF_QP", "ZF_QW", "ZF_N", "ZF_AREA", "ZF_CEN",
    "XB_QW", "YB_QW", "ZB_QW", "V_SCALE", "V_VOL", "V_CEN", "COEF",
]
GEOM = {n: i for i, n in enumerate(GEOM_FIELDS)}
GEOM_NCOMP = [3, 15, 5, 3, 1, 3, 15, 5, 3, 1, 3, 15, 5, 15, 1, 3, 5, 5, 5, 1, 1, 3, 10]

# cs_debug_get arrays: name -> (which, components)
DEBUG = {
    "V": (0, 80), "ent_modes": (1, 4), "flatten": (2, 1), "dUdt": (3, 8),
    "Efx": (4, 1), "Efy": (5, 1), "Efz": (6, 1),
    "Bxq": (7, 5), "Byq": (8, 5), "Bzq": (9, 5), "E1": (10, 3),
    "speeds": (11, 6), "entflux": (12, 3), "positivity": (13, 1),
}

RADIAL = {"uniform": 0, "log": 1, "stretched": 2}
CS_RK2, CS_SSPRK3, CS_IMEX_RK2 = 2, 3, 4

EXPORTS = [
    "cs_geom_ncomp", "cs_create", "cs_destroy", "cs_last_error", "cs_box_dims", "cs_params_check",
    "cs_mesh_build", "cs_mesh_share", "cs_mesh_device_bytes", "cs_mesh_build_host", "cs_geometry_get", "cs_mask_get", "cs_stencil_get",
    "cs_fill_map_get", "cs_sync_map_get",
    "cs_geometry_single_zone", "cs_init_problem", "cs_init_problem_host", "cs_state_put", "cs_state_get",
    "cs_stage", "cs_step", "cs_steps", "cs_evaluate_timestep", "cs_synchronize", "cs_fill_ghosts",
    "cs_limit_all_slopes_p12", "cs_make_facial_fluxes", "cs_make_edge_efields_p1",
    "cs_build_non_stiff_sources", "cs_update_imex_rk_step_p1", "cs_cleanup_after_update",
    "cs_debug_get", "cs_diag", "cs_get_stream", "cs_launch_count", "cs_profile_begin", "cs_profile_end",
    "cs_cfl_timestep_noalloc", "cs_estimate_device_bytes", "cs_serve_create", "cs_serve_submit",
    "cs_serve_wait", "cs_serve_state", "cs_serve_stats", "cs_serve_destroy",
    "cs_batch_create", "cs_batch_steps", "cs_batch_autotune", "cs_batch_grid_fraction", "cs_batch_last_error",
    "cs_batch_destroy", "cs_twod_rs_ez", "cs_pointwise", "cs_fp64_fma_rate", "cs_limit_minmax",
    "cs_state_put_amr", "cs_state_get_amr", "cs_debug_set_wait_error",
    "cs_snapshot_save", "cs_snapshot_load", "cs_snapshot_write_host", "cs_snapshot_read_host",
]


class CsParams(ctypes.Structure):
    _fields_ = [
        ("ntp", ctypes.c_int32), ("nr", ctypes.c_int32), ("nghost", ctypes.c_int32),
        ("radial_mesh", ctypes.c_int32),
        ("rmin", ctypes.c_double), ("rmax", ctypes.c_double), ("radial_ratio", ctypes.c_double),
        ("gamma", ctypes.c_double), ("rhofloor", ctypes.c_double), ("prsfloor", ctypes.c_double),
        ("smallnum", ctypes.c_double), ("cfl_coef", ctypes.c_double), ("flatten_coef", ctypes.c_double),
        ("prs_flatten_coef", ctypes.c_double), ("gm", ctypes.c_double),
        ("bc_lower", ctypes.c_int32), ("bc_upper", ctypes.c_int32), ("rk_scheme", ctypes.c_int32),
        ("flags", ctypes.c_int32),
    ]


class CsInitDesc(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64), ("kind", ctypes.c_int32), ("lmax", ctypes.c_int32),
        ("rho_amp", ctypes.c_double), ("a_amp", ctypes.c_double), ("v_amp", ctypes.c_double),
        ("p0", ctypes.c_double),
    ]


DEFAULT_PARAMS = dict(
    nghost=4, radial_mesh="uniform", rmin=1.0, rmax=2.0, radial_ratio=1.0, gamma=5.0 / 3.0,
    rhofloor=1.0e-12, prsfloor=1.0e-9, smallnum=1.0e-12, cfl_coef=0.2, flatten_coef=0.4,
    prs_flatten_coef=1.5, gm=0.0, bc_lower=2, bc_upper=2, rk_scheme=CS_RK2, flags=0,
)
CS_FLAG_NO_ADP_CACHE = 1
CS_FLAG_NO_OP_CACHE = 2
CS_FLAG_NO_PANEL_SYNC = 4
CS_FLAG_FP32 = 8
CS_FLAG_ADP_PER_PANEL = 16
CS_FLAG_LSQ_PER_PANEL = 32
CS_FLAG_STEP10 = 64
CS_FLAG_P2 = 128
CS_FLAG_PANEL_AVERAGE = 256


def make_params(**kw) -> CsParams:
    d = dict(DEFAULT_PARAMS)
    d.update(kw)
    p = CsParams()
    for name, _ in CsParams._fields_:
        v = d[name]
        if name == "radial_mesh" and isinstance(v, str):
            v = RADIAL[v]
        setattr(p, name, v)
    return p


def make_init(**kw) -> CsInitDesc:
    d = dict(seed=1, kind=1, lmax=4, rho_amp=0.05, a_amp=0.05, v_amp=0.0, p0=1.0e-2)
    d.update(kw)
    r = CsInitDesc()
    for name, _ in CsInitDesc._fields_:
        setattr(r, name, d[name])
    return r


class CsRequest(ctypes.Structure):
    _fields_ = [("params", CsParams), ("init", CsInitDesc), ("steps", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class CsServeResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32), ("mesh_reused", ctypes.c_int32), ("latency_s", ctypes.c_double),
        ("queue_s", ctypes.c_double), ("mass", ctypes.c_double), ("energy", ctypes.c_double),
        ("max_divb", ctypes.c_double), ("dt_last", ctypes.c_double), ("zone_updates", ctypes.c_int64),
    ]


_lib = None


def load_library() -> ctypes.CDLL:
    """Load libcubesphere_b200.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m cubesphere_b200.build` (needs nvcc)")
    lib = ctypes.CDLL(str(LIB_PATH))
    P, I, D, S = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_size_t
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)
    sig = {
        "cs_geom_ncomp": ([ctypes.c_int], ctypes.c_int),
        "cs_create": ([ctypes.POINTER(CsParams), ctypes.POINTER(P)], ctypes.c_int),
        "cs_destroy": ([P], ctypes.c_int),
        "cs_last_error": ([P], ctypes.c_char_p),
        "cs_params_check": ([ctypes.POINTER(CsParams)], ctypes.c_char_p),
        "cs_box_dims": ([P, ip, ip, ip], ctypes.c_int),
        "cs_mesh_build": ([P], ctypes.c_int),
        "cs_mesh_share": ([P, P], ctypes.c_int),
        "cs_mesh_device_bytes": ([P, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "cs_mesh_build_host": ([P], ctypes.c_int),
        "cs_geometry_get": ([P, ctypes.c_int, dp, S], ctypes.c_int),
        "cs_mask_get": ([P, ip, S], ctypes.c_int),
        "cs_stencil_get": ([P, ip, S], ctypes.c_int),
        "cs_fill_map_get": ([P, ip, ip, ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "cs_sync_map_get": ([P, I, ip, ip, ctypes.POINTER(ctypes.c_int8), ctypes.POINTER(ctypes.c_int8),
                             ctypes.POINTER(ctypes.c_int8), ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "cs_geometry_single_zone": ([I, I, I, I, D, D, I, I, dp, S], ctypes.c_int),
        "cs_init_problem": ([P, ctypes.POINTER(CsInitDesc)], ctypes.c_int),
        "cs_init_problem_host": ([P, ctypes.POINTER(CsInitDesc), dp, dp, dp, dp, dp], ctypes.c_int),
        "cs_state_put": ([P, dp, dp, dp, dp, dp], ctypes.c_int),
        "cs_state_get": ([P, dp, dp, dp, dp, dp], ctypes.c_int),
        "cs_stage": ([P, I, D], ctypes.c_int),
        "cs_step": ([P, D, dp], ctypes.c_int),
        "cs_steps": ([P, ctypes.c_int32, ctypes.c_double, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "cs_evaluate_timestep": ([P, D, dp], ctypes.c_int),
        "cs_synchronize": ([P], ctypes.c_int),
        "cs_update_imex_rk_step_p1": ([P, D], ctypes.c_int),
        "cs_debug_get": ([P, I, dp, S], ctypes.c_int),
        "cs_diag": ([P, dp, dp, dp], ctypes.c_int),
        "cs_get_stream": ([P, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
        "cs_launch_count": ([P, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "cs_profile_begin": ([P], ctypes.c_int),
        "cs_profile_end": ([P, I, ctypes.c_char_p, dp, ctypes.POINTER(ctypes.c_int64), ip], ctypes.c_int),
        "cs_cfl_timestep_noalloc": ([P, P, P, P, I, I, I, D, D, D, D, D, P, dp], ctypes.c_int),
        "cs_estimate_device_bytes": ([ctypes.POINTER(CsParams)], ctypes.c_size_t),
        "cs_serve_create": ([I, D, I, ctypes.POINTER(P)], ctypes.c_int),
        "cs_serve_submit": ([P, ctypes.POINTER(CsRequest), ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "cs_serve_wait": ([P, ctypes.c_int64, ctypes.POINTER(CsServeResult)], ctypes.c_int),
        "cs_serve_state": ([P, ctypes.c_int64, dp, dp, dp, dp, dp], ctypes.c_int),
        "cs_serve_stats": ([P, dp, dp, dp, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "cs_serve_destroy": ([P], ctypes.c_int),
        "cs_batch_create": ([ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)],
                            ctypes.c_int),
        "cs_batch_steps": ([P, ctypes.c_int32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
                           ctypes.c_int),
        "cs_batch_autotune": ([P, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "cs_batch_grid_fraction": ([P, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "cs_batch_last_error": ([P], ctypes.c_char_p),
        "cs_batch_destroy": ([P], ctypes.c_int),
        "cs_twod_rs_ez": ([ctypes.c_int32, ctypes.c_int32, dp, dp], ctypes.c_int),
        "cs_pointwise": ([ctypes.POINTER(CsParams), ctypes.c_int32, ctypes.c_int32, dp, dp], ctypes.c_int),
        "cs_fp64_fma_rate": ([ctypes.c_int32, dp], ctypes.c_int),
        "cs_limit_minmax": ([P, dp, dp], ctypes.c_int),
        "cs_state_put_amr": ([P, ctypes.c_int32, dp, dp, dp, dp, dp], ctypes.c_int),
        "cs_debug_set_wait_error": ([P, ctypes.c_int32], ctypes.c_int),
        "cs_state_get_amr": ([P, ctypes.c_int32, dp, dp, dp, dp, dp], ctypes.c_int),
        "cs_snapshot_save": ([P, ctypes.c_char_p, D, D, ctypes.c_int64], ctypes.c_int),
        "cs_snapshot_load": ([P, ctypes.c_char_p, dp, dp, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "cs_snapshot_write_host": ([ctypes.c_char_p, ctypes.POINTER(CsParams), dp, dp, dp, dp, dp, D, D,
                                    ctypes.c_int64], ctypes.c_int),
        "cs_snapshot_read_host": ([ctypes.c_char_p, ctypes.POINTER(CsParams), dp, dp, dp, dp, dp, dp, dp,
                                   ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    }
    for name in ("cs_fill_ghosts", "cs_limit_all_slopes_p12", "cs_make_facial_fluxes", "cs_make_edge_efields_p1",
                 "cs_build_non_stiff_sources", "cs_cleanup_after_update"):
        sig[name] = ([P], ctypes.c_int)
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


class CsError(RuntimeError):
    pass


class Solve:
    """One resident solve: six panels of (ntp + 2 G + 1)^2 x (nr + 2 G + 1)
    points on the current CUDA device, driven through the C ABI."""

    def __init__(self, params: CsParams | None = None, **kw):
        self.lib = load_library()
        self.params = params if params is not None else make_params(**kw)
        h = ctypes.c_void_p()
        rc = self.lib.cs_create(ctypes.byref(self.params), ctypes.byref(h))
        if rc:
            why = self.lib.cs_params_check(ctypes.byref(self.params)).decode()
            raise CsError(f"cs_create failed ({rc}): {why}")
        self.h = h
        ni, nj, nk = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self.lib.cs_box_dims(self.h, ctypes.byref(ni), ctypes.byref(nj), ctypes.byref(nk))
        self.NI, self.NJ, self.NK = ni.value, nj.value, nk.value
        self.N, self.nr, self.G = self.params.ntp, self.params.nr, self.params.nghost
        self.box = self.NI * self.NJ * self.NK

    # ---------------- plumbing ----------------
    def _check(self, rc: int, what: str) -> None:
        if rc:
            raise CsError(f"{what} failed ({rc}): {self.lib.cs_last_error(self.h).decode()}")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, ncomp: int) -> tuple:
        return (ncomp, 6, self.NK, self.NJ, self.NI)

    def zeros(self, ncomp: int) -> np.ndarray:
        return np.zeros(self.shape(ncomp), dtype=np.float64)

    def interior(self, a: np.ndarray) -> np.ndarray:
        """Interior zones (1..ntp)^2 x (1..nr) of a panel-box array."""
        G, N, nr = self.G, self.N, self.nr
        return a[..., G + 1:G + nr + 1, G + 1:G + N + 1, G + 1:G + N + 1]

    # ---------------- mesh ----------------
    def mesh_build(self, device: bool = True) -> None:
        rc = self.lib.cs_mesh_build(self.h) if device else self.lib.cs_mesh_build_host(self.h)
        self._check(rc, "cs_mesh_build")

    def mesh_share(self, other: "Solve") -> None:
        """Use the resident mesh of `other` (same mesh parameters) instead of building one."""
        self._check(self.lib.cs_mesh_share(self.h, other.h), "cs_mesh_share")

    def mesh_device_bytes(self) -> int:
        """Device bytes held by this solve's mesh (shared with attached solves)."""
        out = ctypes.c_uint64()
        self._check(self.lib.cs_mesh_device_bytes(self.h, ctypes.byref(out)), "cs_mesh_device_bytes")
        return out.value

    def geometry(self, field: str | int) -> np.ndarray:
        f = GEOM[field] if isinstance(field, str) else field
        out = self.zeros(GEOM_NCOMP[f])
        self._check(self.lib.cs_geometry_get(self.h, f, _dptr(out), out.size), "cs_geometry_get")
        return out

    def mask(self) -> np.ndarray:
        out = np.zeros((6, self.NK, self.NJ, self.NI), dtype=np.int32)
        self._check(self.lib.cs_mask_get(self.h, _iptr(out), out.size), "cs_mask_get")
        return out

    def fill_map(self):
        """The ghost-exchange map cs_fill_ghosts applies (cs_fill_map_get):
        arrays src, dst (int32 element offsets into the field arrays) and meta
        (uint8: destination field bits 0-2, source field bits 5-7, negate bit
        3, average bit 4)."""
        n = ctypes.c_int64(0)
        self._check(self.lib.cs_fill_map_get(self.h, None, None, None, ctypes.byref(n)), "cs_fill_map_get")
        src = np.zeros(n.value, dtype=np.int32)
        dst = np.zeros(n.value, dtype=np.int32)
        meta = np.zeros(n.value, dtype=np.uint8)
        self._check(self.lib.cs_fill_map_get(self.h, _iptr(src), _iptr(dst),
                                             meta.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.byref(n)),
                    "cs_fill_map_get")
        return src, dst, meta

    def sync_map(self, which: int):
        """The panel-edge ownership list cs_stage applies (cs_sync_map_get):
        which 0 faces, 1 edges.  Arrays dst, src (int32 offsets), dst_kind,
        src_kind (int8 face direction or EMF component) and sign (int8)."""
        n = ctypes.c_int64(0)
        self._check(self.lib.cs_sync_map_get(self.h, which, None, None, None, None, None, ctypes.byref(n)),
                    "cs_sync_map_get")
        dst, src = np.zeros(n.value, dtype=np.int32), np.zeros(n.value, dtype=np.int32)
        dk, sk, sg = (np.zeros(n.value, dtype=np.int8) for _ in range(3))
        i8 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))
        self._check(self.lib.cs_sync_map_get(self.h, which, _iptr(dst), _iptr(src), i8(dk), i8(sk), i8(sg),
                                             ctypes.byref(n)), "cs_sync_map_get")
        return dst, src, dk, sk, sg

    def stencil(self) -> np.ndarray:
        out = np.zeros((6, 12, 2, self.NJ, self.NI), dtype=np.int32)
        self._check(self.lib.cs_stencil_get(self.h, _iptr(out), out.size), "cs_stencil_get")
        return out

    # ---------------- state ----------------
    def init_problem(self, desc: CsInitDesc | None = None, **kw) -> None:
        d = desc if desc is not None else make_init(**kw)
        self._check(self.lib.cs_init_problem(self.h, ctypes.byref(d)), "cs_init_problem")

    def init_problem_host(self, desc: CsInitDesc | None = None, **kw) -> dict:
        d = desc if desc is not None else make_init(**kw)
        st = self.empty_state()
        self._check(self.lib.cs_init_problem_host(self.h, ctypes.byref(d), *[_dptr(st[k]) for k in STATE_KEYS]),
                    "cs_init_problem_host")
        return st

    def empty_state(self) -> dict:
        return {"U": self.zeros(8), "ent": self.zeros(1), "bxf": self.zeros(1), "byf": self.zeros(1),
                "bzf": self.zeros(1)}

    def put_state(self, st: dict) -> None:
        self._check(self.lib.cs_state_put(self.h, *[_dptr(np.ascontiguousarray(st[k])) for k in STATE_KEYS]),
                    "cs_state_put")

    def get_state(self, out: dict | None = None) -> dict:
        st = out if out is not None else self.empty_state()
        self._check(self.lib.cs_state_get(self.h, *[_dptr(st[k]) for k in STATE_KEYS]), "cs_state_get")
        return st

    # ---------------- the step ----------------
    def stage(self, irk: int, dtcur: float) -> None:
        self._check(self.lib.cs_stage(self.h, irk, dtcur), "cs_stage")

    def step(self, dtcur: float) -> float:
        out = ctypes.c_double()
        self._check(self.lib.cs_step(self.h, dtcur, ctypes.byref(out)), "cs_step")
        return out.value

    def steps(self, nsteps: int, dtcur: float) -> float:
        """nsteps steps (graph replay, device-resident time step); returns the next time step."""
        out = ctypes.c_double()
        self._check(self.lib.cs_steps(self.h, nsteps, dtcur, ctypes.byref(out)), "cs_steps")
        return out.value

    def evaluate_timestep(self, dtcur: float) -> float:
        out = ctypes.c_double()
        self._check(self.lib.cs_evaluate_timestep(self.h, dtcur, ctypes.byref(out)), "cs_evaluate_timestep")
        return out.value

    def synchronize(self) -> None:
        self._check(self.lib.cs_synchronize(self.h), "cs_synchronize")

    # reference routine names
    def fill_ghosts(self):
        self._check(self.lib.cs_fill_ghosts(self.h), "cs_fill_ghosts")

    def limit_all_slopes_p12(self):
        self._check(self.lib.cs_limit_all_slopes_p12(self.h), "cs_limit_all_slopes_p12")

    def make_facial_fluxes(self):
        self._check(self.lib.cs_make_facial_fluxes(self.h), "cs_make_facial_fluxes")

    def make_edge_efields_p1(self):
        self._check(self.lib.cs_make_edge_efields_p1(self.h), "cs_make_edge_efields_p1")

    def build_non_stiff_sources(self):
        self._check(self.lib.cs_build_non_stiff_sources(self.h), "cs_build_non_stiff_sources")

    def update_imex_rk_step_p1(self, dtmove: float):
        self._check(self.lib.cs_update_imex_rk_step_p1(self.h, dtmove), "cs_update_imex_rk_step_p1")

    def cleanup_after_update(self):
        self._check(self.lib.cs_cleanup_after_update(self.h), "cs_cleanup_after_update")

    def debug(self, name: str) -> np.ndarray:
        which, nc = DEBUG[name]
        out = self.zeros(nc)
        self._check(self.lib.cs_debug_get(self.h, which, _dptr(out), out.size), "cs_debug_get")
        return out

    def stream_ptr(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        out = ctypes.c_void_p()
        self._check(self.lib.cs_get_stream(self.h, ctypes.byref(out)), "cs_get_stream")
        return out.value or 0

    def launch_count(self) -> int:
        out = ctypes.c_int64()
        self._check(self.lib.cs_launch_count(self.h, ctypes.byref(out)), "cs_launch_count")
        return out.value

    def profile_begin(self) -> None:
        self._check(self.lib.cs_profile_begin(self.h), "cs_profile_begin")

    def profile_end(self, max_kernels: int = 64) -> dict:
        """{kernel name: (total device ms, launches)} since profile_begin."""
        names = ctypes.create_string_buffer(32 * max_kernels)
        ms = np.zeros(max_kernels)
        cnt = np.zeros(max_kernels, dtype=np.int64)
        n = ctypes.c_int32()
        self._check(self.lib.cs_profile_end(self.h, max_kernels, names, _dptr(ms),
                                            cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(n)),
                    "cs_profile_end")
        raw = names.raw
        out = {}
        for q in range(n.value):
            key = raw[32 * q:32 * q + 32].split(b"\0", 1)[0].decode()
            out[key] = (float(ms[q]), int(cnt[q]))
        return out

    def snapshot_save(self, path: str, time: float, dtcur: float, step: int) -> None:
        self._check(self.lib.cs_snapshot_save(self.h, str(path).encode(), time, dtcur, step), "cs_snapshot_save")

    def snapshot_load(self, path: str) -> tuple:
        """Loads a snapshot into the resident state; returns (time, dtcur, step)."""
        t, d, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        self._check(self.lib.cs_snapshot_load(self.h, str(path).encode(), ctypes.byref(t), ctypes.byref(d),
                                              ctypes.byref(n)), "cs_snapshot_load")
        return t.value, d.value, n.value

    def limit_minmax(self) -> tuple:
        """STEP 10 of the last LIMIT_ALL_SLOPES_P12 (needs CS_FLAG_STEP10):
        (v_min[9], v_max[9]) -- 8 primitives and the normalised divergence."""
        vmin, vmax = np.zeros(9), np.zeros(9)
        self._check(self.lib.cs_limit_minmax(self.h, _dptr(vmin), _dptr(vmax)), "cs_limit_minmax")
        return vmin, vmax

    def diag(self) -> tuple:
        m, e, d = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.cs_diag(self.h, ctypes.byref(m), ctypes.byref(e), ctypes.byref(d)), "cs_diag")
        return m.value, e.value, d.value


STATE_KEYS = ("U", "ent", "bxf", "byf", "bzf")


def geometry_single_zone(isector: int, ntp_global: int, nr_global: int, iscale: int, rmin: float, rmax: float,
                         radial_mesh: str, field: str) -> np.ndarray:
    """Geometry field of the reference quadrature-point test setting (host only)."""
    lib = load_library()
    n1 = ntp_global // iscale + 1
    nk = nr_global // iscale + 1
    f = GEOM[field]
    out = np.zeros((GEOM_NCOMP[f], 6, nk, n1, n1), dtype=np.float64)
    rc = lib.cs_geometry_single_zone(isector, ntp_global, nr_global, iscale, rmin, rmax, RADIAL[radial_mesh], f,
                                     _dptr(out), out.size)
    if rc:
        raise CsError(f"cs_geometry_single_zone failed ({rc})")
    return out


class Batch:
    """Batched form: independent solves advanced together, one CUDA graph
    launch per step for all members (each member's step a child graph)."""

    def __init__(self, members: list):
        self.lib = load_library()
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        h = ctypes.c_void_p()
        rc = self.lib.cs_batch_create(arr, len(self.members), ctypes.byref(h))
        if rc:
            raise CsError(f"cs_batch_create failed ({rc})")
        self.h = h

    def _check(self, rc: int, what: str) -> None:
        if rc:
            raise CsError(f"{what} failed ({rc}): {self.lib.cs_batch_last_error(self.h).decode()}")

    def steps(self, nsteps: int, dts) -> list:
        n = len(self.members)
        din = (ctypes.c_double * n)(*dts)
        dout = (ctypes.c_double * n)()
        self._check(self.lib.cs_batch_steps(self.h, nsteps, din, dout), "cs_batch_steps")
        return list(dout)

    def autotune(self, trial_steps: int = 2) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.cs_batch_autotune(self.h, trial_steps, ctypes.byref(ms)), "cs_batch_autotune")
        return ms.value

    def grid_fraction(self, member: int) -> float:
        f = ctypes.c_double()
        self._check(self.lib.cs_batch_grid_fraction(self.h, member, ctypes.byref(f)), "cs_batch_grid_fraction")
        return f.value

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cs_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop over the C ABI: requests (solves of any size) are admitted
    while device memory allows and run concurrently, each in its own context
    and stream; ``stats`` reports p50 / p99 latency and throughput."""

    def __init__(self, max_active: int = 4, mem_fraction: float = 0.8, keep_state: bool = False):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.cs_serve_create(max_active, mem_fraction, int(keep_state), ctypes.byref(h))
        if rc:
            raise CsError(f"cs_serve_create failed ({rc})")
        self.h = h

    def submit(self, steps: int, params, init) -> int:
        r = CsRequest()
        r.params = params if isinstance(params, CsParams) else make_params(**params)
        r.init = init if isinstance(init, CsInitDesc) else make_init(**init)
        r.steps = steps
        rid = ctypes.c_int64()
        rc = self.lib.cs_serve_submit(self.h, ctypes.byref(r), ctypes.byref(rid))
        if rc:
            raise CsError(f"cs_serve_submit failed ({rc})")
        return rid.value

    def wait(self, rid: int) -> CsServeResult:
        out = CsServeResult()
        self.lib.cs_serve_wait(self.h, rid, ctypes.byref(out))
        return out

    def state(self, rid: int, params: CsParams) -> dict:
        ni = params.ntp + 2 * params.nghost + 1
        nk = params.nr + 2 * params.nghost + 1
        st = {k: np.zeros(((8 if k == "U" else 1), 6, nk, ni, ni)) for k in STATE_KEYS}
        rc = self.lib.cs_serve_state(self.h, rid, *[_dptr(st[k]) for k in STATE_KEYS])
        if rc:
            raise CsError(f"cs_serve_state failed ({rc})")
        return st

    def stats(self) -> dict:
        p50, p99, zu = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n = ctypes.c_int64()
        self.lib.cs_serve_stats(self.h, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(zu), ctypes.byref(n))
        return {"p50_s": p50.value, "p99_s": p99.value, "zone_updates_per_s": zu.value, "completed": n.value}

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cs_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def twod_rs_ez(kind: int, cases: np.ndarray) -> np.ndarray:
    """ESSz of the device multidimensional Riemann solver for each row of
    `cases` (kind 4: 11 inputs, kind 3: 10 inputs; see cs_twod_rs_ez)."""
    a = np.ascontiguousarray(cases, dtype=np.float64)
    out = np.zeros(a.shape[0])
    rc = load_library().cs_twod_rs_ez(kind, a.shape[0], _dptr(a), _dptr(out))
    if rc:
        raise CsError(f"cs_twod_rs_ez failed ({rc})")
    return out


def pointwise(kind: int, cases: np.ndarray, **params) -> np.ndarray:
    """The device pointwise physics on each row of `cases` (see cs_pointwise):
    kind 0 PRIM_TO_CONS (8 prims + entropy -> 8 conserved), 1 CONS_TO_PRIM
    (8 conserved + entropy -> 8 prims, entropy, floor flag, 8 conserved),
    2 the HLL solve (V_L, V_R, ent_L, ent_R -> Fluct_L, Fluct_R, F_L, F_R,
    S_L, S_R, entropy flux); params as for Solve (flags=CS_FLAG_FP32 for
    the precision form)."""
    nin, nout = {0: (9, 8), 1: (9, 18), 2: (18, 35)}[kind]
    a = np.ascontiguousarray(cases, dtype=np.float64).reshape(-1, nin)
    out = np.zeros((a.shape[0], nout))
    p = make_params(**params)
    rc = load_library().cs_pointwise(ctypes.byref(p), kind, a.shape[0], _dptr(a), _dptr(out))
    if rc:
        raise CsError(f"cs_pointwise failed ({rc})")
    return out


def fp64_fma_rate(iters: int = 4096) -> float:
    """Measured FP64 FMA rate of the current device, TFLOP/s."""
    out = ctypes.c_double()
    rc = load_library().cs_fp64_fma_rate(iters, ctypes.byref(out))
    if rc:
        raise CsError(f"cs_fp64_fma_rate failed ({rc})")
    return out.value


def estimate_device_bytes(**params) -> int:
    p = make_params(**params)
    return int(load_library().cs_estimate_device_bytes(ctypes.byref(p)))


def snapshot_write_host(path, params: CsParams, st: dict, time: float, dtcur: float, step: int) -> int:
    """Writes host arrays as a snapshot file (no device); returns the status."""
    lib = load_library()
    return lib.cs_snapshot_write_host(str(path).encode(), ctypes.byref(params),
                                      *[_dptr(np.ascontiguousarray(st[k])) for k in STATE_KEYS], time, dtcur, step)


def snapshot_read_host(path, params: CsParams, st: dict):
    """Reads a snapshot into host arrays; returns (status, time, dtcur, step)."""
    lib = load_library()
    t, d, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
    rc = lib.cs_snapshot_read_host(str(path).encode(), ctypes.byref(params), *[_dptr(st[k]) for k in STATE_KEYS],
                                   ctypes.byref(t), ctypes.byref(d), ctypes.byref(n))
    return rc, t.value, d.value, n.value
