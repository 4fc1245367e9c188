"""Device plan: one compiled configuration of the LH82 step on one grid.

Wraps an ``OraclePlan*`` of the C ABI.  Tensors passed in must be contiguous
CUDA tensors of the plan's dtype (float64 for "fp64", float32 for "fp32").
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _lib as L

PRECISIONS = {"fp64": (L.OB_PREC_F64, torch.float64), "fp32": (L.OB_PREC_F32, torch.float32)}


def require_cuda() -> None:
    if not torch.cuda.is_available():
        raise RuntimeError("the oraclev8_b200 backend needs a CUDA device (no CPU fallback)")


@dataclass
class PlanSpec:
    nx: int
    ny: int
    nz: int
    Lx: float
    Ly: float
    Lz: float
    rho0: np.ndarray
    theta0: np.ndarray
    precision: str = "fp64"
    buoyancy: bool = False
    projection: bool = False
    advection: int = L.OB_ADV_NONE
    coriolis: int = L.OB_COR_NONE
    f0: float = 0.0
    u_env: float = 0.0
    v_env: float = 0.0
    f_y: Optional[np.ndarray] = None
    damping: bool = False
    epsilon: float = 0.0
    heating: bool = False
    heat_r: Optional[np.ndarray] = None
    heat_z: Optional[np.ndarray] = None
    poisson_diag_every: int = 60
    # production slow components (tendency.py:1259-1668)
    drag: bool = False
    drag_cd: float = 0.0
    drag_dz: float = 1.0
    drag_u_env: float = 0.0
    drag_v_env: float = 0.0
    drag_weight: Optional[np.ndarray] = None
    sponge: bool = False
    sponge_u_env: float = 0.0
    sponge_v_env: float = 0.0
    sponge_alpha: Optional[np.ndarray] = None
    sponge_alpha_h: Optional[np.ndarray] = None
    diffusion: int = L.OB_DIFF_NONE
    diff_nu: float = 0.0
    diff_dx2: float = 1.0
    diff_dy2: float = 1.0
    cooling: bool = False
    cool_alpha: float = 0.0
    # max|u| (m/s) above which the device's blow-up flag is raised; 0: only
    # non-finite values raise it (measure_lh82_phase3.py:129-130)
    blowup_u_max: float = 0.0
    # time the kernel forms of each class at creation and keep the fastest
    # (cached per grid, precision, component set and device); False keeps
    # the built-in choice
    autotune: bool = True


def _f64(a):
    return None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class Plan:
    def __init__(self, spec: PlanSpec):
        require_cuda()
        self.lib = L.load()
        if spec.precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {spec.precision!r}")
        self.spec = spec
        self.prec, self.dtype = PRECISIONS[spec.precision]
        self.device = torch.device("cuda", torch.cuda.current_device())
        g = L.GridDesc(spec.nx, spec.ny, spec.nz, spec.Lx, spec.Ly, spec.Lz, self.prec)
        keep = [_f64(spec.rho0), _f64(spec.theta0), _f64(spec.f_y), _f64(spec.heat_r),
                _f64(spec.heat_z), _f64(spec.drag_weight), _f64(spec.sponge_alpha),
                _f64(spec.sponge_alpha_h)]
        rho0, theta0, f_y, heat_r, heat_z, drag_w, sp_a, sp_ah = keep
        self._keep = keep
        if rho0.shape != (spec.nz,) or theta0.shape != (spec.nz,):
            raise ValueError(f"rho0/theta0 must have shape ({spec.nz},)")
        c = L.ComponentDesc(int(spec.buoyancy), int(spec.projection), int(spec.advection),
                            int(spec.coriolis), float(spec.f0), float(spec.u_env),
                            float(spec.v_env), L.dptr(f_y), int(spec.damping),
                            float(spec.epsilon), int(spec.heating), L.dptr(heat_r),
                            L.dptr(heat_z), L.dptr(rho0), L.dptr(theta0),
                            int(spec.poisson_diag_every), int(spec.drag),
                            float(spec.drag_cd), float(spec.drag_dz), float(spec.drag_u_env),
                            float(spec.drag_v_env), L.dptr(drag_w), int(spec.sponge),
                            float(spec.sponge_u_env), float(spec.sponge_v_env), L.dptr(sp_a),
                            L.dptr(sp_ah), int(spec.diffusion), float(spec.diff_nu),
                            float(spec.diff_dx2), float(spec.diff_dy2), int(spec.cooling),
                            float(spec.cool_alpha), float(spec.blowup_u_max))
        h = ctypes.c_void_p()
        L.check(self.lib.oracle_b200_plan_create(ctypes.byref(g), ctypes.byref(c), ctypes.byref(h)))
        self.handle = h
        self.shape = (spec.nx, spec.ny, spec.nz)
        self.wshape = (spec.nx, spec.ny, spec.nz + 1)
        if spec.autotune:
            self.tune()

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.oracle_b200_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    def release(self, stream=None) -> None:
        """Give the plan's device memory back to the pool in the order of
        ``stream`` (default: the current stream) without synchronising; every
        kernel that used the plan must have been queued on that stream or be
        complete.  The plan is unusable afterwards."""
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            s = stream if stream is not None else torch.cuda.current_stream(self.device)
            self.lib.oracle_b200_plan_release(h, ctypes.c_void_p(s.cuda_stream))
            self.handle = None

    # -- helpers -------------------------------------------------------------
    @property
    def scratch_bytes(self) -> int:
        return int(self.lib.oracle_b200_plan_scratch_bytes(self.handle))

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _ptr(self, t: torch.Tensor, shape) -> ctypes.c_void_p:
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"expected a CUDA torch.Tensor, got {type(t).__name__}")
        if t.device.type != "cuda" or t.dtype != self.dtype or not t.is_contiguous():
            raise ValueError(f"expected a contiguous {self.dtype} CUDA tensor, got "
                             f"{t.dtype} on {t.device} (contiguous={t.is_contiguous()})")
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"shape {tuple(t.shape)} does not match expected {tuple(shape)}")
        return ctypes.c_void_p(t.data_ptr())

    def state_ptrs(self, u, v, w, th, phi) -> L.StatePtrs:
        s, ws = self.shape, self.wshape
        return L.StatePtrs(self._ptr(u, s), self._ptr(v, s), self._ptr(w, ws),
                           self._ptr(th, s), self._ptr(phi, s))

    def empty(self, wlevels=False):
        return torch.empty(self.wshape if wlevels else self.shape, dtype=self.dtype,
                           device=self.device)

    # -- entry points ----------------------------------------------------------
    def step(self, ins: L.StatePtrs, outs: L.StatePtrs, dt: float, want_diag: bool):
        L.check(self.lib.oracle_b200_step(self.handle, ctypes.byref(ins), ctypes.byref(outs),
                                          float(dt), int(want_diag), self._stream()))

    @property
    def launches(self) -> int:
        return int(self.lib.oracle_b200_launch_count(self.handle))

    def profile(self, enable: bool) -> None:
        L.check(self.lib.oracle_b200_profile(self.handle, int(enable)))

    def profile_read(self) -> dict:
        n = len(L.PROF_CLASSES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_long * n)()
        L.check(self.lib.oracle_b200_profile_read(self.handle, ms, cnt, n))
        return {c: (float(ms[i]), int(cnt[i])) for i, c in enumerate(L.PROF_CLASSES)}

    def set_refinement(self, passes: int, every: int = 1) -> None:
        """FP64 defect correction of the final projection of every `every`-th
        step (single-precision plans)."""
        L.check(self.lib.oracle_b200_set_refinement(self.handle, int(passes), int(every)))

    def refine(self, u, v, w, phi):
        s = self.shape
        L.check(self.lib.oracle_b200_refine(self.handle, self._ptr(u, s), self._ptr(v, s),
                                            self._ptr(w, self.wshape), self._ptr(phi, s),
                                            self._stream()))

    def step_graph(self, ptrs: L.StatePtrs, dt: float, nsteps: int) -> "StepGraph":
        return StepGraph(self, ptrs, dt, nsteps)

    # -- kernel variants ---------------------------------------------------------
    def variants(self) -> dict:
        """The plan's kernel-form choices, by OB_VAR_* name (0 = form off)."""
        n = len(L.VARIANTS)
        buf = (ctypes.c_int * n)()
        L.check(self.lib.oracle_b200_plan_get_variants(self.handle, buf, n))
        return dict(zip(L.VARIANTS, buf))

    def set_variants(self, **kw) -> None:
        """Change some choices (``plan.set_variants(zc4_ix=8)``); every value is
        checked against the forms the plan's grid and precision allow."""
        cur = self.variants()
        for k, v in kw.items():
            if k not in cur:
                raise ValueError(f"unknown kernel variant {k!r}")
            cur[k] = int(v)
        vals = (ctypes.c_int * len(L.VARIANTS))(*[cur[k] for k in L.VARIANTS])
        L.check(self.lib.oracle_b200_plan_set_variants(self.handle, vals, len(L.VARIANTS)))

    def shared_memory_forms(self) -> None:
        """Turn every register-resident and compile-time-chunk form off: the
        runtime-chunk shared-memory Stockham kernels only."""
        self.set_variants(**{k: 0 for k in L.VARIANTS if k.startswith(("zc3", "zc4"))})

    def tune(self, force: bool = False) -> dict:
        """Time the kernel forms of each class and keep the fastest (cached per
        grid, precision, component set and device); returns the choices."""
        L.check(self.lib.oracle_b200_plan_tune(self.handle, L.OB_TUNE_FORCE if force else 0,
                                               self._stream()))
        return self.variants()

    def read_diag(self) -> np.ndarray:
        """The diagnostics block (synchronises the current stream).  A raised
        blow-up flag is not an error here: it is slot ``DIAG["blowup"]``, and
        the values are returned as computed (NaN maxima propagate as NumPy's
        max does)."""
        buf = (ctypes.c_double * L.DIAG_COUNT)()
        rc = self.lib.oracle_b200_read_diag(self.handle, buf, L.DIAG_COUNT, self._stream())
        if rc != L.OB_ERR_NONFINITE:
            L.check(rc)
        return np.frombuffer(buf, dtype=np.float64).copy()

    def read_diag_async(self, out: torch.Tensor) -> None:
        """Enqueue a copy of the raw diagnostics block into ``out`` (a pinned
        float64 host tensor of at least DIAG_COUNT elements) on the current
        stream, without waiting; ``out[DIAG["blowup"]]`` is the blow-up flag
        once the copy has landed."""
        if out.dtype != torch.float64 or out.device.type != "cpu" or out.numel() < L.DIAG_COUNT:
            raise ValueError("read_diag_async needs a float64 host tensor of DIAG_COUNT elements")
        L.check(self.lib.oracle_b200_read_diag_async(
            self.handle, ctypes.c_void_p(out.data_ptr()), L.DIAG_COUNT, self._stream()))

    def blown_up(self) -> int:
        """The plan's sticky blow-up flag as of its last diagnosed step: 0 none,
        1 a non-finite value, 2 max|u| above ``blowup_u_max``."""
        return int(self.read_diag()[L.DIAG["blowup"]])

    def project(self, u, v, w, phi, log_diag=False):
        s = self.shape
        L.check(self.lib.oracle_b200_project(self.handle, self._ptr(u, s), self._ptr(v, s),
                                             self._ptr(w, self.wshape), self._ptr(phi, s),
                                             int(log_diag), self._stream()))

    def divergence(self, u, v, w, out=None):
        out = self.empty() if out is None else out
        s = self.shape
        L.check(self.lib.oracle_b200_divergence(self.handle, self._ptr(u, s), self._ptr(v, s),
                                                self._ptr(w, self.wshape), self._ptr(out, s),
                                                self._stream()))
        return out

    def phi_gradient(self, phi):
        gx, gy, gz = self.empty(), self.empty(), self.empty(True)
        s = self.shape
        L.check(self.lib.oracle_b200_phi_gradient(self.handle, self._ptr(phi, s),
                                                  self._ptr(gx, s), self._ptr(gy, s),
                                                  self._ptr(gz, self.wshape), self._stream()))
        return gx, gy, gz

    def poisson_solve(self, d, log_diag=False):
        phi = self.empty()
        s = self.shape
        L.check(self.lib.oracle_b200_poisson_solve(self.handle, self._ptr(d, s),
                                                   self._ptr(phi, s), int(log_diag),
                                                   self._stream()))
        return phi

    def apply_operator(self, phi):
        out = self.empty()
        s = self.shape
        L.check(self.lib.oracle_b200_apply_operator(self.handle, self._ptr(phi, s),
                                                    self._ptr(out, s), self._stream()))
        return out

    def buoyancy(self, th):
        dw = self.empty(True)
        L.check(self.lib.oracle_b200_buoyancy(self.handle, self._ptr(th, self.shape),
                                              self._ptr(dw, self.wshape), self._stream()))
        return dw

    def tendency(self, mask, u, v, w, th, dt_slow):
        du, dv, dw, dth = self.empty(), self.empty(), self.empty(True), self.empty()
        phi_dummy = th  # the tendency entry point does not read phi
        sp = self.state_ptrs(u, v, w, th, phi_dummy)
        s = self.shape
        L.check(self.lib.oracle_b200_tendency(self.handle, int(mask), ctypes.byref(sp),
                                              self._ptr(du, s), self._ptr(dv, s),
                                              self._ptr(dw, self.wshape), self._ptr(dth, s),
                                              float(dt_slow), self._stream()))
        return du, dv, dw, dth


class StepGraph:
    """``nsteps`` in-place steps of one state recorded as a CUDA graph
    (oracle_b200_step_graph_create); ``launch`` replays them with one call.
    Holds the plan so that the plan outlives the graph; the state tensors
    behind ``ptrs`` must stay alive while the graph is used."""

    def __init__(self, plan: Plan, ptrs: L.StatePtrs, dt: float, nsteps: int):
        self.plan, self.lib, self.nsteps = plan, plan.lib, int(nsteps)
        h = ctypes.c_void_p()
        L.check(self.lib.oracle_b200_step_graph_create(plan.handle, ctypes.byref(ptrs),
                                                       float(dt), self.nsteps, ctypes.byref(h)))
        self.handle = h
        self.kernels = int(self.lib.oracle_b200_step_graph_kernels(h))

    def launch(self, stream=None) -> None:
        s = stream if stream is not None else torch.cuda.current_stream(self.plan.device)
        L.check(self.lib.oracle_b200_step_graph_launch(self.handle,
                                                       ctypes.c_void_p(s.cuda_stream)))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.oracle_b200_step_graph_destroy(h)
            except Exception:
                pass
            self.handle = None


# ---------------------------------------------------------------------------
# Small cache of operator plans (component-level calls and module functions)
# ---------------------------------------------------------------------------
_CACHE: "dict[tuple, Plan]" = {}
_CACHE_MAX = 8


def _key(spec: PlanSpec) -> tuple:
    def b(a):
        return None if a is None else np.asarray(a, dtype=np.float64).tobytes()
    return (spec.nx, spec.ny, spec.nz, float(spec.Lx), float(spec.Ly), float(spec.Lz),
            spec.precision, b(spec.rho0), b(spec.theta0), spec.buoyancy, spec.projection,
            spec.advection, spec.coriolis, float(spec.f0), float(spec.u_env),
            float(spec.v_env), b(spec.f_y), spec.damping, float(spec.epsilon), spec.heating,
            b(spec.heat_r), b(spec.heat_z), spec.poisson_diag_every, spec.drag,
            float(spec.drag_cd), float(spec.drag_dz), float(spec.drag_u_env),
            float(spec.drag_v_env), b(spec.drag_weight), spec.sponge, float(spec.sponge_u_env),
            float(spec.sponge_v_env), b(spec.sponge_alpha), b(spec.sponge_alpha_h),
            spec.diffusion, float(spec.diff_nu), float(spec.diff_dx2), float(spec.diff_dy2),
            spec.cooling, float(spec.cool_alpha), float(spec.blowup_u_max), spec.autotune)


def cached_plan(spec: PlanSpec) -> Plan:
    k = _key(spec)
    p = _CACHE.get(k)
    if p is None:
        if len(_CACHE) >= _CACHE_MAX:
            _CACHE.pop(next(iter(_CACHE)))
        p = Plan(spec)
        _CACHE[k] = p
    return p


def precision_of(t: torch.Tensor) -> str:
    if t.dtype == torch.float64:
        return "fp64"
    if t.dtype == torch.float32:
        return "fp32"
    raise ValueError(f"unsupported dtype {t.dtype}; use float64 or float32")
