"""ctypes binding of liboracle_b200.so (the C ABI in include/oracle_b200.h).

There is no CPU fallback: if the library or a CUDA device is missing, every
entry point raises RuntimeError.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_size_t, c_void_p
from pathlib import Path

import numpy as np

OB_OK, OB_ERR_ARG, OB_ERR_CUDA, OB_ERR_NONFINITE, OB_ERR_UNSUPPORTED = 0, 1, 2, 3, 4
OB_PREC_F64, OB_PREC_F32 = 0, 1
OB_ADV_NONE, OB_ADV_CENTERED2, OB_ADV_UPWIND5H = 0, 1, 2
OB_COR_NONE, OB_COR_FPLANE, OB_COR_BETA = 0, 1, 2
OB_TEND_ADVECTION, OB_TEND_CORIOLIS, OB_TEND_DAMPING, OB_TEND_HEATING = 1, 2, 4, 8
OB_TEND_DRAG, OB_TEND_SPONGE, OB_TEND_DIFFUSION, OB_TEND_COOLING = 16, 32, 64, 128
OB_DIFF_NONE, OB_DIFF_LAPLACIAN, OB_DIFF_BIHARMONIC = 0, 1, 2
DIAG = dict(max_u=0, max_v=1, max_w=2, max_th=3, phi_min=4, phi_max=5, compat0=6, disc0=9,
            last_compat=12, last_disc=13, blowup=14, stall=15)
DIAG_COUNT = 16

LIB_PATH = Path(__file__).resolve().parent / "liboracle_b200.so"

EXPORTS = (
    "oracle_b200_plan_create", "oracle_b200_plan_destroy", "oracle_b200_plan_scratch_bytes",
    "oracle_b200_step", "oracle_b200_project", "oracle_b200_divergence",
    "oracle_b200_phi_gradient", "oracle_b200_poisson_solve", "oracle_b200_apply_operator",
    "oracle_b200_buoyancy", "oracle_b200_tendency", "oracle_b200_read_diag",
    "oracle_b200_last_error", "oracle_b200_version", "oracle_b200_launch_count",
    "oracle_b200_profile", "oracle_b200_profile_read", "oracle_b200_poisson_solve_noalloc",
    "oracle_b200_set_refinement", "oracle_b200_refine",
    "oracle_b200_tracker_create", "oracle_b200_tracker_destroy", "oracle_b200_track_theta",
    "oracle_b200_track_vorticity", "oracle_b200_step_graph_create",
    "oracle_b200_step_graph_launch", "oracle_b200_step_graph_kernels",
    "oracle_b200_step_graph_destroy", "oracle_b200_vortex_fill", "oracle_b200_plan_release",
    "oracle_b200_intensity_cap", "oracle_b200_vdiag_create", "oracle_b200_vdiag_destroy",
    "oracle_b200_vdiag_speed_max", "oracle_b200_vdiag_vorticity", "oracle_b200_vdiag_ke",
    "oracle_b200_vdiag_rings", "oracle_b200_vdiag_zpos", "oracle_b200_vdiag_centroid",
    "oracle_b200_plan_get_variants", "oracle_b200_plan_set_variants", "oracle_b200_plan_tune",
    "oracle_b200_read_diag_async",
)
# kernel-variant choices of a plan, in OB_VAR_* order (include/oracle_b200.h)
VARIANTS = ("zc2_fx", "zc2_fxs", "zc2_ix", "zc2_fy", "zc2_iy", "zc3_fx", "zc3_fxs", "zc3_ix",
            "zc3_fxd", "zc3_fy", "zc3_fyd", "zc4_fx", "zc4_fxs", "zc4_ix", "zc4_fxd", "zc4_fy",
            "zc4_iy", "slow_xw", "thomas_fast", "rzc2_fx", "rzc2_fy", "zc4_fyd", "zc4_fxsh")
OB_TUNE_FORCE = 1
ABI_VERSION = 2  # OB_ABI_VERSION of the header these tables follow
PROF_CLASSES = ("fx", "fy", "thomas", "iy", "ix", "slow", "diag", "other", "refine",
                "thomas_lw")


class GridDesc(ctypes.Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("nz", c_int), ("Lx", c_double),
                ("Ly", c_double), ("Lz", c_double), ("precision", c_int)]


class ComponentDesc(ctypes.Structure):
    _fields_ = [("buoyancy", c_int), ("projection", c_int), ("advection", c_int),
                ("coriolis", c_int), ("f0", c_double), ("u_env", c_double),
                ("v_env", c_double), ("f_y", POINTER(c_double)), ("damping", c_int),
                ("epsilon", c_double), ("heating", c_int), ("heat_r", POINTER(c_double)),
                ("heat_z", POINTER(c_double)), ("rho0", POINTER(c_double)),
                ("theta0", POINTER(c_double)), ("poisson_diag_every", c_int),
                ("drag", c_int), ("drag_cd", c_double), ("drag_dz", c_double),
                ("drag_u_env", c_double), ("drag_v_env", c_double),
                ("drag_weight", POINTER(c_double)), ("sponge", c_int),
                ("sponge_u_env", c_double), ("sponge_v_env", c_double),
                ("sponge_alpha", POINTER(c_double)), ("sponge_alpha_h", POINTER(c_double)),
                ("diffusion", c_int), ("diff_nu", c_double), ("diff_dx2", c_double),
                ("diff_dy2", c_double), ("cooling", c_int), ("cool_alpha", c_double),
                ("blowup_u_max", c_double)]


class StatePtrs(ctypes.Structure):
    _fields_ = [("u", c_void_p), ("v", c_void_p), ("w", c_void_p),
                ("theta_prime", c_void_p), ("phi", c_void_p)]


class TrackFix(ctypes.Structure):
    _fields_ = [("mean", c_double), ("raw_min", c_double), ("raw_max", c_double),
                ("raw_idx", ctypes.c_longlong), ("raw_nb", c_double * 5),
                ("win_min", c_double), ("win_max", c_double),
                ("win_idx", ctypes.c_longlong), ("win_nb", c_double * 5)]


class VdMax(ctypes.Structure):
    _fields_ = [("value", c_double), ("index", ctypes.c_longlong)]


_lib = None


def load(path: Path | None = None):
    """Load the library (once).  Raises RuntimeError when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p.name} not found: build it with `python -m oraclev8_b200.build` "
            "(the B200 backend has no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    vp = c_void_p
    sig = {
        "oracle_b200_plan_create": ([POINTER(GridDesc), POINTER(ComponentDesc), POINTER(vp)], c_int),
        "oracle_b200_plan_destroy": ([vp], c_int),
        "oracle_b200_plan_release": ([vp, vp], c_int),
        "oracle_b200_plan_scratch_bytes": ([vp], c_size_t),
        "oracle_b200_step": ([vp, POINTER(StatePtrs), POINTER(StatePtrs), c_double, c_int, vp], c_int),
        "oracle_b200_project": ([vp, vp, vp, vp, vp, c_int, vp], c_int),
        "oracle_b200_divergence": ([vp, vp, vp, vp, vp, vp], c_int),
        "oracle_b200_phi_gradient": ([vp, vp, vp, vp, vp, vp], c_int),
        "oracle_b200_poisson_solve": ([vp, vp, vp, c_int, vp], c_int),
        "oracle_b200_apply_operator": ([vp, vp, vp, vp], c_int),
        "oracle_b200_buoyancy": ([vp, vp, vp, vp], c_int),
        "oracle_b200_tendency": ([vp, c_int, POINTER(StatePtrs), vp, vp, vp, vp, c_double, vp], c_int),
        "oracle_b200_intensity_cap": ([vp, vp, c_int, ctypes.c_long, c_double, c_double, c_double,
                                       c_double, vp, vp, vp], c_int),
        "oracle_b200_read_diag": ([vp, POINTER(c_double), c_int, vp], c_int),
        "oracle_b200_last_error": ([], ctypes.c_char_p),
        "oracle_b200_version": ([], c_int),
        "oracle_b200_launch_count": ([vp], ctypes.c_long),
        "oracle_b200_profile": ([vp, c_int], c_int),
        "oracle_b200_profile_read": ([vp, POINTER(c_double), POINTER(ctypes.c_long), c_int], c_int),
        "oracle_b200_poisson_solve_noalloc": ([POINTER(GridDesc), POINTER(c_double), vp, vp, vp], c_int),
        "oracle_b200_set_refinement": ([vp, c_int, c_int], c_int),
        "oracle_b200_refine": ([vp, vp, vp, vp, vp, vp], c_int),
        "oracle_b200_tracker_create": ([c_int, c_int, c_int, POINTER(c_double), POINTER(c_double),
                                        POINTER(c_double), POINTER(vp)], c_int),
        "oracle_b200_tracker_destroy": ([vp], c_int),
        "oracle_b200_track_theta": ([vp, vp, c_int, c_int, c_int, c_double, c_double, c_double,
                                     POINTER(TrackFix), vp], c_int),
        "oracle_b200_track_vorticity": ([vp, vp, vp, c_int, c_double, POINTER(c_double), vp], c_int),
        "oracle_b200_step_graph_create": ([vp, POINTER(StatePtrs), c_double, c_int, POINTER(vp)], c_int),
        "oracle_b200_step_graph_launch": ([vp, vp], c_int),
        "oracle_b200_step_graph_kernels": ([vp], ctypes.c_long),
        "oracle_b200_step_graph_destroy": ([vp], c_int),
        "oracle_b200_vortex_fill": ([c_int, c_int, c_int, c_int, vp, vp, vp, vp, c_int, c_double,
                                     c_double, POINTER(StatePtrs), vp], c_int),
        "oracle_b200_vdiag_create": ([c_int, c_int, c_int, POINTER(vp)], c_int),
        "oracle_b200_vdiag_destroy": ([vp], c_int),
        "oracle_b200_vdiag_speed_max": ([vp, vp, vp, c_int, POINTER(c_int), c_int, c_double,
                                         c_double, POINTER(VdMax), vp], c_int),
        "oracle_b200_vdiag_vorticity": ([vp, vp, vp, c_int, POINTER(c_int), c_int, c_double,
                                         c_double, c_double, c_double, c_double, POINTER(VdMax),
                                         POINTER(c_double), vp], c_int),
        "oracle_b200_vdiag_ke": ([vp, vp, vp, c_int, c_double, c_double, POINTER(c_double), vp],
                                 c_int),
        "oracle_b200_vdiag_rings": ([vp, vp, vp, c_int, POINTER(c_int), c_int, c_double, c_double,
                                     c_double, c_double, POINTER(c_double), c_int, c_double,
                                     POINTER(c_double), vp], c_int),
        "oracle_b200_vdiag_zpos": ([vp, vp, vp, c_int, c_double, vp], c_int),
        "oracle_b200_vdiag_centroid": ([vp, c_int, c_int, c_int, c_int, POINTER(c_double), vp],
                                       c_int),
        "oracle_b200_plan_get_variants": ([vp, POINTER(c_int), c_int], c_int),
        "oracle_b200_plan_set_variants": ([vp, POINTER(c_int), c_int], c_int),
        "oracle_b200_plan_tune": ([vp, c_int, vp], c_int),
        "oracle_b200_read_diag_async": ([vp, vp, c_int, vp], c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    v = lib.oracle_b200_version()
    if v != ABI_VERSION:
        raise RuntimeError(f"{p.name} has ABI version {v}, these bindings need {ABI_VERSION}: "
                           "rebuild it with `python -m oraclev8_b200.build`")
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc == OB_OK:
        return
    msg = _lib.oracle_b200_last_error().decode(errors="replace") if _lib else "?"
    if rc == OB_ERR_ARG:
        raise ValueError(msg)
    raise RuntimeError(f"oracle_b200 error {rc}: {msg}")


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(POINTER(c_double))
