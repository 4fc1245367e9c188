"""WS-RK3 integrator of the LH82 core on the B200 backend.

Same interface as oracle_v8/solver/integrator.py:140-311:
``RK3Integrator(config, base).step(state, dt, step_number) -> (State,
StepDiagnostics)``.  The OperatorConfig is compiled once into a device plan;
each step is one call into the C ABI, which enqueues the Strang slow half
steps, the three fast stages and their five projections on the current CUDA
stream.  The six StepDiagnostics reductions run on the device; the host reads
them (one synchronisation) only on the steps ``ORACLE_DIAG_EVERY`` selects,
exactly as the reference does (integrator.py:287-300).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np
import torch

from .. import _lib as L
from .._plan import Plan, PlanSpec
from .. import backend
from ..backend import asarray, to_numpy, wrap_base
from .tendency import (State, cooling_fields, diffusion_fields, drag_fields,
                       sponge_fields)

_DIAG_EVERY = max(1, int(os.environ.get("ORACLE_DIAG_EVERY", "1")))


@dataclass
class StepDiagnostics:
    """integrator.py:83-132."""
    step: int
    t: float
    dt: float
    stage_compat_residuals: list = field(default_factory=list)
    stage_disc_op_residuals: list = field(default_factory=list)
    max_u: float = 0.0
    max_v: float = 0.0
    max_w: float = 0.0
    max_theta_prime: float = 0.0
    surface_phi_min: float = 0.0
    surface_phi_max: float = 0.0
    # not in the reference's dataclass: the device's sticky blow-up flag
    # (0 none, 1 a non-finite value, 2 max|u| above the integrator's
    # blowup_u_max) as of this step
    blowup: int = 0


_UNSUPPORTED_SLOTS = ("pressure_gradient",)


def compile_config(config, base, precision: str, poisson_diag_every: int | None = None,
                   grid=None) -> PlanSpec:
    """Translate an OperatorConfig into a device PlanSpec.  Components the B200
    step does not implement raise NotImplementedError (no silent fallback)."""
    for slot in _UNSUPPORTED_SLOTS:
        if getattr(config, slot, None) is not None:
            raise NotImplementedError(
                f"OperatorConfig.{slot} is not implemented on the oraclev8_b200 backend")
    proj = config.projection
    adv = config.advection
    if grid is None:
        src = proj if proj is not None else adv
        if src is None:
            raise ValueError("cannot infer the grid: the config has neither a projection "
                             "nor an advection component")
        if proj is not None:
            grid = (proj.nx, proj.ny, proj.nz, proj.Lx, proj.Ly, proj.Lz)
        else:
            if getattr(adv, "_grid", None) is None:
                raise RuntimeError("AdvectionComponent is unconfigured")
            grid = adv._grid
    nx, ny, nz, Lx, Ly, Lz = grid
    if poisson_diag_every is None:
        poisson_diag_every = max(1, int(os.environ.get("ORACLE_POISSON_DIAG_EVERY", "60")))
    spec = PlanSpec(nx=int(nx), ny=int(ny), nz=int(nz), Lx=float(Lx), Ly=float(Ly),
                    Lz=float(Lz), rho0=np.asarray(to_numpy(base.rho0), dtype=np.float64),
                    theta0=np.asarray(to_numpy(base.theta0), dtype=np.float64),
                    precision=precision, buoyancy=config.buoyancy is not None,
                    projection=proj is not None, poisson_diag_every=int(poisson_diag_every))
    if adv is not None:
        if getattr(adv, "_grid", None) is None and getattr(adv, "_dx", None) is None:
            raise RuntimeError("AdvectionComponent is unconfigured")
        spec.advection = (L.OB_ADV_UPWIND5H if adv.scheme == "upwind5h"
                          else L.OB_ADV_CENTERED2)
    cor = config.coriolis
    if cor is not None:
        spec.coriolis = L.OB_COR_BETA if cor._mode == "beta_plane" else L.OB_COR_FPLANE
        spec.f0 = float(cor._f0)
        spec.u_env = float(cor._u_env)
        spec.v_env = float(cor._v_env)
        if spec.coriolis == L.OB_COR_BETA:
            fy = getattr(cor, "f_y", None)
            if fy is None:  # reference object: device (1, ny, 1) array
                fy = np.asarray(to_numpy(cor._f_y)).reshape(-1)
            spec.f_y = np.asarray(fy, dtype=np.float64)
    dmp = config.divergence_damping
    if dmp is not None:
        if getattr(dmp, "name", "") != "helmholtz_divergence_damping":
            raise NotImplementedError(f"{type(dmp).__name__} is not implemented on the "
                                      "oraclev8_b200 backend")
        spec.damping = True
        spec.epsilon = float(dmp._epsilon)
    heat = config.diabatic_heating
    if heat is not None:
        if not hasattr(heat, "heat_factors"):
            raise NotImplementedError("diabatic heating must be the oraclev8_b200 "
                                      "DiabaticHeatingComponent (separable factors)")
        spec.heating = True
        spec.heat_r, spec.heat_z = heat.heat_factors
    # production components (operator_config.py:100-103); their attribute
    # names are the reference's, so either side's objects compile alike
    z = None
    if config.surface_drag is not None or config.sponge_damping is not None:
        z = np.asarray(to_numpy(base.z), dtype=np.float64).reshape(-1)
        if z.shape != (int(nz),):
            raise ValueError(f"base.z has shape {z.shape}, expected ({nz},)")
    if config.surface_drag is not None:
        _set(spec, drag_fields(config.surface_drag, z))
    if config.sponge_damping is not None:
        _set(spec, sponge_fields(config.sponge_damping, z))
    if config.horiz_diffusion is not None:
        _set(spec, diffusion_fields(config.horiz_diffusion))
    if config.newtonian_cooling is not None:
        _set(spec, cooling_fields(config.newtonian_cooling))
    return spec


def _set(spec: PlanSpec, fields: dict) -> None:
    for k, v in fields.items():
        setattr(spec, k, v)


class RK3Integrator:
    """integrator.py:140-311."""
    _STAGE_ALPHAS = (1.0 / 3.0, 1.0 / 2.0, 1.0)

    def __init__(self, config, base, precision: str | None = None,
                 refine_passes: int | None = None, refine_every: int = 1,
                 blowup_u_max: float = 0.0, autotune: bool = True) -> None:
        """precision: "fp64", "fp32" or "fp32r".  "fp32r" is the FP32 step
        followed, every ``refine_every`` steps, by ``refine_passes`` (default 1)
        defect corrections of the final projection whose residual divergence
        is formed in FP64.  blowup_u_max > 0 also raises the device's blow-up
        flag (``StepDiagnostics.blowup``) when max|u| exceeds it; non-finite
        values always do.  Steps never raise on it, as the reference's step
        does not: a harness tests the flag (measure_lh82_phase3.py:129-130).
        autotune: time the kernel forms of each class for this grid once per
        process and keep the fastest (``plan.variants()`` shows the choice)."""
        self.config = config
        self.base = wrap_base(base)
        self.precision = precision or backend.PRECISION
        if self.precision not in ("fp64", "fp32", "fp32r"):
            raise ValueError(f"precision must be fp64, fp32 or fp32r, got {self.precision!r}")
        plan_prec = "fp64" if self.precision == "fp64" else "fp32"
        if refine_passes is None:
            refine_passes = 1 if self.precision == "fp32r" else 0
        self.spec = compile_config(config, self.base, plan_prec)
        self.spec.blowup_u_max = float(blowup_u_max)
        self.spec.autotune = bool(autotune)
        self.plan = Plan(self.spec)
        self.refine_passes, self.refine_every = int(refine_passes), int(refine_every)
        if self.refine_passes:
            self.plan.set_refinement(self.refine_passes, self.refine_every)
        self.dtype = self.plan.dtype
        self._fast = self.spec.buoyancy and self.spec.projection

    # -- helpers ---------------------------------------------------------------
    def _dev(self, a, wlevels=False):
        t = asarray(a, dtype=self.dtype)
        shape = self.plan.wshape if wlevels else self.plan.shape
        if tuple(t.shape) != shape:
            raise ValueError(f"state field shape {tuple(t.shape)} does not match the grid {shape}")
        return t

    def _want_diag(self, step_number: int) -> bool:
        de = _DIAG_EVERY
        return de == 1 or step_number % de == 0 or (step_number + 1) % de == 0

    def _diagnostics(self, step_number, t, dt, want) -> StepDiagnostics:
        dg = StepDiagnostics(step=step_number, t=t, dt=dt)
        if not want:
            nan = float("nan")
            dg.max_u = dg.max_v = dg.max_w = dg.max_theta_prime = nan
            dg.surface_phi_min = dg.surface_phi_max = nan
            return dg
        d = self.plan.read_diag()
        D = L.DIAG
        dg.max_u, dg.max_v = float(d[D["max_u"]]), float(d[D["max_v"]])
        dg.max_w, dg.max_theta_prime = float(d[D["max_w"]]), float(d[D["max_th"]])
        dg.surface_phi_min, dg.surface_phi_max = float(d[D["phi_min"]]), float(d[D["phi_max"]])
        dg.blowup = int(d[D["blowup"]])
        if self._fast:
            dg.stage_compat_residuals = [float(d[D["compat0"] + s]) for s in range(3)]
            dg.stage_disc_op_residuals = [float(d[D["disc0"] + s]) for s in range(3)]
        return dg

    # -- public interface ------------------------------------------------------
    def step(self, state: State, dt: float, step_number: int = 0):
        """Advance one full RK3 step; returns a new State at t + dt (t is
        advanced only by the fast stages, integrator.py:339-340, 489)."""
        u, v = self._dev(state.u), self._dev(state.v)
        w = self._dev(state.w, wlevels=True)
        th, phi = self._dev(state.theta_prime), self._dev(state.projection_potential)
        out = State(torch.empty_like(u), torch.empty_like(v), torch.empty_like(w),
                    torch.empty_like(th), torch.empty_like(phi),
                    state.t + dt if self._fast else state.t)
        want = self._want_diag(step_number)
        self.plan.step(self.plan.state_ptrs(u, v, w, th, phi),
                       self.plan.state_ptrs(out.u, out.v, out.w, out.theta_prime,
                                            out.projection_potential), dt, want)
        return out, self._diagnostics(step_number, state.t, dt, want)

    def step_(self, state: State, dt: float, want_diag: bool = False):
        """In-place step on device tensors of the plan's dtype (no allocation,
        no synchronisation); returns the state.  Diagnostics, when requested,
        are left on the device for ``read_diagnostics``."""
        ptrs = self.plan.state_ptrs(state.u, state.v, state.w, state.theta_prime,
                                    state.projection_potential)
        self.plan.step(ptrs, ptrs, dt, want_diag)
        if self._fast:
            state.t = state.t + dt
        return state

    def capture(self, state: State, dt: float, nsteps: int = 1):
        """Record ``nsteps`` in-place steps of ``state`` (device tensors of the
        plan's dtype) as a CUDA graph; ``graph.launch(stream)`` then advances
        the state by nsteps * dt with one host call.  The model time
        ``state.t`` is not advanced by graph launches (the caller owns it)."""
        ptrs = self.plan.state_ptrs(state.u, state.v, state.w, state.theta_prime,
                                    state.projection_potential)
        return self.plan.step_graph(ptrs, dt, nsteps)

    def read_diagnostics(self, step_number: int = 0, t: float = 0.0, dt: float = 0.0):
        return self._diagnostics(step_number, t, dt, True)
