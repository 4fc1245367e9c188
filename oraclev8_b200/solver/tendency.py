"""Step components of the LH82 core on the B200 backend.

Mirrors oracle_v8/solver/tendency.py: the same classes, constructor
signatures, shape contracts and exception types.  State fields are CUDA
torch tensors; every ``compute_tendency`` / ``apply_projection`` runs the
sm_100a kernels through the C ABI.  The integrator does not call these
methods on its hot path: it compiles the whole OperatorConfig into one device
plan (see integrator.py).
"""
from __future__ import annotations

import abc
import ctypes
from dataclasses import dataclass
from enum import Enum
from typing import Optional

import numpy as np
import torch

from .. import _lib as L
from .._plan import PlanSpec, cached_plan, precision_of
from ..backend import to_numpy


class StateVar(str, Enum):
    """tendency.py:60-76."""
    U = "u"
    V = "v"
    W = "w"
    THETA_PRIME = "theta_prime"
    PROJECTION_POTENTIAL = "projection_potential"


class StepStage(Enum):
    """tendency.py:84-116."""
    PRE_PROJECTION = "pre_projection"
    PROJECTION = "projection"
    POST_PROJECTION = "post_projection"
    SLOW = "slow"
    DIAGNOSTIC = "diagnostic"


@dataclass
class State:
    """Prognostic state (tendency.py:145-172): u, v, theta', phi are (nx, ny, nz),
    w is (nx, ny, nz+1) with explicit surface/lid values."""
    u: torch.Tensor
    v: torch.Tensor
    w: torch.Tensor
    theta_prime: torch.Tensor
    projection_potential: torch.Tensor
    t: float


@dataclass
class Tendency:
    """tendency.py:175-255."""
    du_dt: Optional[torch.Tensor] = None
    dv_dt: Optional[torch.Tensor] = None
    dw_dt: Optional[torch.Tensor] = None
    dtheta_prime_dt: Optional[torch.Tensor] = None

    @classmethod
    def zeros_like(cls, state: State) -> "Tendency":
        return cls(torch.zeros_like(state.u), torch.zeros_like(state.v),
                   torch.zeros_like(state.w), torch.zeros_like(state.theta_prime))

    def add_(self, other: "Tendency") -> "Tendency":
        for f in ("du_dt", "dv_dt", "dw_dt", "dtheta_prime_dt"):
            o = getattr(other, f)
            if o is None:
                continue
            c = getattr(self, f)
            if c is None:
                setattr(self, f, o.clone())
            else:
                c += o
        return self

    def validate_against_state(self, state: State) -> None:
        for tn, sn in (("du_dt", "u"), ("dv_dt", "v"), ("dw_dt", "w"),
                       ("dtheta_prime_dt", "theta_prime")):
            tv = getattr(self, tn)
            if tv is None:
                continue
            sv = getattr(state, sn)
            if tuple(tv.shape) != tuple(sv.shape):
                raise ValueError(f"Tendency.{tn} shape {tuple(tv.shape)} does not match "
                                 f"State.{sn} shape {tuple(sv.shape)}")


# ---------------------------------------------------------------------------
# Component hierarchy (tendency.py:263-385)
# ---------------------------------------------------------------------------

class StepComponent(abc.ABC):
    name: str = "abstract"
    stage: StepStage = StepStage.SLOW

    @abc.abstractmethod
    def reads(self) -> tuple: ...

    @abc.abstractmethod
    def writes(self) -> tuple: ...

    def to_log_dict(self) -> dict:
        return {"name": self.name, "stage": self.stage.value,
                "reads": [v.value for v in self.reads()],
                "writes": [v.value for v in self.writes()],
                "class": type(self).__name__, "kind": self._kind()}

    def _kind(self) -> str:
        if isinstance(self, TendencyComponent):
            return "tendency"
        if isinstance(self, ProjectionComponent):
            return "projection"
        if isinstance(self, DiagnosticComponent):
            return "diagnostic"
        return "unknown"

    def __repr__(self) -> str:
        return f"<{type(self).__name__}: {self.name} ({self.stage.value})>"


class TendencyComponent(StepComponent):
    @abc.abstractmethod
    def compute_tendency(self, state, equation_set, staggering, base, dt) -> Tendency: ...


class ProjectionComponent(StepComponent):
    stage = StepStage.PROJECTION

    @abc.abstractmethod
    def apply_projection(self, state, equation_set, staggering, base, dt) -> State: ...


class DiagnosticComponent(StepComponent):
    stage = StepStage.DIAGNOSTIC

    @abc.abstractmethod
    def compute_diagnostic(self, state, equation_set, staggering, base) -> dict: ...

    def writes(self) -> tuple:
        return ()


# ---------------------------------------------------------------------------
# Plans for component-level calls
# ---------------------------------------------------------------------------

def _profiles(base, nz):
    if base is None:
        one = np.ones(nz)
        return one, 300.0 * one
    return (np.asarray(to_numpy(base.rho0), dtype=np.float64),
            np.asarray(to_numpy(base.theta0), dtype=np.float64))


def _plan_for(state_like: torch.Tensor, base=None, Lx=1.0, Ly=1.0, Lz=1.0, rho0=None,
              **components):
    nx, ny, nz = (int(s) for s in state_like.shape)
    r, t = _profiles(base, nz)
    if rho0 is not None:
        r = np.asarray(to_numpy(rho0), dtype=np.float64)
    spec = PlanSpec(nx=nx, ny=ny, nz=nz, Lx=float(Lx), Ly=float(Ly), Lz=float(Lz), rho0=r,
                    theta0=t, precision=precision_of(state_like), **components)
    return cached_plan(spec)


def _lengths_from_k(kx, ky, nx, ny):
    kx = np.asarray(to_numpy(kx), dtype=np.float64)
    ky = np.asarray(to_numpy(ky), dtype=np.float64)
    return 2.0 * np.pi / kx[1], 2.0 * np.pi / ky[1]


# ---------------------------------------------------------------------------
# Shared operators (tendency.py:393-500)
# ---------------------------------------------------------------------------

def anelastic_divergence(u, v, w, rho_bar_full, rho_bar_half, kx, ky, dz):
    """d = div(rho u) with the projection's own discrete operator
    (tendency.py:393-437).  rho_bar_half must be the Lorenz average of
    rho_bar_full with boundary copies (tendency.py:748-754)."""
    nx, ny, nz = (int(s) for s in u.shape)
    Lx, Ly = _lengths_from_k(kx, ky, nx, ny)
    p = _plan_for(u, Lx=Lx, Ly=Ly, Lz=float(dz) * nz, rho0=rho_bar_full)
    return p.divergence(u.contiguous(), v.contiguous(), w.contiguous())


def _phi_gradient(phi, kx, ky, dz):
    """(dphi/dx, dphi/dy on full levels, dphi/dz on nz+1 half levels) —
    tendency.py:440-500."""
    nx, ny, nz = (int(s) for s in phi.shape)
    Lx, Ly = _lengths_from_k(kx, ky, nx, ny)
    p = _plan_for(phi, Lx=Lx, Ly=Ly, Lz=float(dz) * nz)
    return p.phi_gradient(phi.contiguous())


# ---------------------------------------------------------------------------
# Concrete components
# ---------------------------------------------------------------------------

class BuoyancyComponent(TendencyComponent):
    """dw/dt += g theta'/theta0 on half levels (tendency.py:508-552)."""
    name = "buoyancy"
    stage = StepStage.PRE_PROJECTION

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        b_half = equation_set.compute_buoyancy_tendency(state.theta_prime, base, staggering)
        if tuple(b_half.shape) != tuple(state.w.shape):
            raise ValueError(
                f"equation_set.compute_buoyancy_tendency returned shape {tuple(b_half.shape)}, "
                f"expected state.w.shape = {tuple(state.w.shape)}.")
        return Tendency(dw_dt=b_half)

    def reads(self):
        return (StateVar.THETA_PRIME,)

    def writes(self):
        return (StateVar.W,)


class PressureGradientComponent(TendencyComponent):
    """-grad(phi) as a tendency (tendency.py:555-674).  Forbidden alongside the
    projection by OperatorConfig; usable on its own."""
    name = "pressure_gradient"
    stage = StepStage.PRE_PROJECTION

    def __init__(self, nx=None, ny=None, nz=None, Lx=None, Ly=None, Lz=None):
        self._grid = None
        if nx is not None and Lx is not None:
            self._grid = (nx, ny, nz, float(Lx), float(Ly), float(Lz))

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        if self._grid is None:
            raise RuntimeError(
                "PressureGradientComponent.compute_tendency called on an unconfigured "
                "instance.  Supply grid parameters at construction:\n"
                "    PressureGradientComponent(nx=..., ny=..., nz=..., Lx=..., Ly=..., Lz=...)")
        nx, ny, nz, Lx, Ly, Lz = self._grid
        p = _plan_for(state.projection_potential, base, Lx, Ly, Lz)
        gx, gy, gz = p.phi_gradient(state.projection_potential.contiguous())
        if tuple(gx.shape) != tuple(state.u.shape) or tuple(gz.shape) != tuple(state.w.shape):
            raise ValueError("phi gradient shapes do not match the state; check the grid")
        return Tendency(du_dt=-gx, dv_dt=-gy, dw_dt=-gz)

    def reads(self):
        return (StateVar.PROJECTION_POTENTIAL,)

    def writes(self):
        return (StateVar.U, StateVar.V, StateVar.W)


@dataclass
class PoissonSolveResult:
    """poisson.py:74-95."""
    phi: object
    compatibility_residual: float
    discrete_operator_residual: float
    n_wavenumbers_solved: int


class AnelasticProjection(ProjectionComponent):
    """Project onto div(rho u) = 0 (tendency.py:677-832)."""
    name = "anelastic_projection"

    def __init__(self, nx: int, ny: int, nz: int, Lx: float, Ly: float, Lz: float):
        from .poisson import VariableCoefficientPoissonSolver
        self._solver = VariableCoefficientPoissonSolver(nx, ny, nz, Lx, Ly, Lz)
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self._dx, self._dy, self._dz = Lx / nx, Ly / ny, Lz / nz
        self.last_solve = None
        self._solve_count = 0

    def apply_projection(self, state, equation_set, staggering, base, dt):
        """Correct (u, v, w) and store phi; rebinds new tensors on ``state``
        like the reference (tendency.py:781-788)."""
        import os
        p = _plan_for(state.u, base, self.Lx, self.Ly, self.Lz)
        self._solve_count += 1
        de = max(1, int(os.environ.get("ORACLE_POISSON_DIAG_EVERY", "60")))
        log = de == 1 or self._solve_count % de == 1
        u, v, w = state.u.clone(), state.v.clone(), state.w.clone()
        phi = torch.empty_like(u)
        p.project(u, v, w, phi, log_diag=log)
        if log:
            d = p.read_diag()
            compat, disc = float(d[L.DIAG["last_compat"]]), float(d[L.DIAG["last_disc"]])
        else:
            compat = disc = 0.0
        self.last_solve = PoissonSolveResult(phi, compat, disc, self.nx * self.ny)
        state.u, state.v, state.w = u, v, w
        state.projection_potential = phi
        return state

    def reads(self):
        return (StateVar.U, StateVar.V, StateVar.W)

    def writes(self):
        return (StateVar.U, StateVar.V, StateVar.W, StateVar.PROJECTION_POTENTIAL)


class AdvectionComponent(TendencyComponent):
    """Advective form for theta' and momentum; WS5 ('upwind5h') or centred
    ('centered2') in x, y, centred in z (tendency.py:835-1068)."""
    name = "advection"
    stage = StepStage.SLOW

    def __init__(self, nx=None, ny=None, nz=None, Lx=None, Ly=None, Lz=None,
                 scheme: str = "centered2"):
        if scheme not in ("centered2", "upwind5h"):
            raise ValueError(f"AdvectionComponent scheme must be 'centered2' or 'upwind5h', "
                             f"got {scheme!r}")
        self.scheme = scheme
        self._grid = None
        self._nz = nz
        if nx is not None and Lx is not None:
            self._grid = (int(nx), int(ny), int(nz), float(Lx), float(Ly), float(Lz))
            self._dx, self._dy, self._dz = Lx / nx, Ly / ny, Lz / nz

    @property
    def scheme_code(self) -> int:
        return L.OB_ADV_UPWIND5H if self.scheme == "upwind5h" else L.OB_ADV_CENTERED2

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        if self._grid is None:
            raise RuntimeError(
                "AdvectionComponent.compute_tendency called on an unconfigured instance.  "
                "Provide grid parameters:\n"
                "    AdvectionComponent(nx=..., ny=..., nz=..., Lx=..., Ly=..., Lz=...)")
        _, _, _, Lx, Ly, Lz = self._grid
        p = _plan_for(state.u, base, Lx, Ly, Lz, advection=self.scheme_code)
        du, dv, dw, dth = p.tendency(L.OB_TEND_ADVECTION, state.u, state.v, state.w,
                                     state.theta_prime, float(dt))
        return Tendency(du_dt=du, dv_dt=dv, dw_dt=dw, dtheta_prime_dt=dth)

    def reads(self):
        return (StateVar.U, StateVar.V, StateVar.W, StateVar.THETA_PRIME)

    def writes(self):
        return (StateVar.U, StateVar.V, StateVar.W, StateVar.THETA_PRIME)


class CoriolisComponent(TendencyComponent):
    """f-plane / beta-plane Coriolis on the perturbation velocity
    (tendency.py:1071-1256)."""
    name = "coriolis"
    stage = StepStage.SLOW
    _OMEGA = 7.2921e-5
    _R_EARTH = 6.371e6

    def __init__(self, f: float = 5e-5, mode: str = "f_plane", beta: float = None,
                 Ly: float = None, ny: int = None, y0: float = None, u_env: float = 0.0,
                 v_env: float = 0.0, periodic_taper: bool = False) -> None:
        self._f0 = f
        self._mode = mode
        self._u_env = float(u_env)
        self._v_env = float(v_env)
        if mode == "beta_plane":
            if Ly is None or ny is None:
                raise ValueError("CoriolisComponent beta_plane mode requires Ly and ny.")
            if beta is None:
                lat = np.arcsin(np.clip(f / (2.0 * self._OMEGA), -1.0, 1.0))
                beta = 2.0 * self._OMEGA * np.cos(lat) / self._R_EARTH
            self._beta = float(beta)
            dy = Ly / ny
            y_ref = y0 if y0 is not None else Ly / 2.0
            y = (np.arange(ny) + 0.5) * dy
            dev = self._beta * (y - y_ref)
            if periodic_taper:
                n_taper = max(1, int(round(0.20 * ny)))
                taper = np.ones(ny)
                for i in range(n_taper):
                    t = np.sin(np.pi * (i + 0.5) / (2.0 * n_taper)) ** 2
                    taper[i] = t
                    taper[ny - 1 - i] = t
                dev = dev * taper
            self._f_y_host = np.float64(f) + dev
        else:
            self._beta = None
            self._f_y_host = None

    @property
    def f(self):
        return self._f0

    @property
    def mode(self):
        return self._mode

    @property
    def beta(self):
        return self._beta

    @property
    def f_y(self):
        """f(y) at cell centres, shape (ny,), FP64 host array (None on the f-plane)."""
        return self._f_y_host

    def mode_code(self) -> int:
        return L.OB_COR_BETA if self._mode == "beta_plane" else L.OB_COR_FPLANE

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        if self._mode == "beta_plane" and state.u.shape[1] != len(self._f_y_host):
            raise ValueError("CoriolisComponent ny does not match the state")
        p = _plan_for(state.u, base, coriolis=self.mode_code(), f0=float(self._f0),
                      u_env=self._u_env, v_env=self._v_env, f_y=self._f_y_host)
        du, dv, _, _ = p.tendency(L.OB_TEND_CORIOLIS, state.u, state.v, state.w,
                                  state.theta_prime, float(dt))
        return Tendency(du_dt=du, dv_dt=dv)

    def set_env(self, u_env: float, v_env: float) -> None:
        """tendency.py:1236-1250."""
        self._u_env = float(u_env)
        self._v_env = float(v_env)

    def reads(self):
        return (StateVar.U, StateVar.V)

    def writes(self):
        return (StateVar.U, StateVar.V)


class DiabaticHeatingComponent(TendencyComponent):
    """Static annular eyewall heating (tendency.py:1671-1738).  Stored as the
    separable factors Q_max f_r(x, y) and f_z(z); their product is formed in
    the kernel in the reference's order, (Q_max f_r) f_z."""
    name = "diabatic_heating"
    stage = StepStage.SLOW

    def __init__(self, Q_max, r_eyewall, width_r, z_peak, width_z, nx, ny, nz, Lx, Ly, Lz,
                 x_c=None, y_c=None) -> None:
        dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
        x_c = x_c if x_c is not None else Lx / 2.0
        y_c = y_c if y_c is not None else Ly / 2.0
        x = (np.arange(nx) + 0.5) * dx
        y = (np.arange(ny) + 0.5) * dy
        z = (np.arange(nz) + 0.5) * dz
        X, Y = np.meshgrid(x, y, indexing="ij")
        r = np.sqrt((X - x_c) ** 2 + (Y - y_c) ** 2)
        f_r = np.exp(-((r - r_eyewall) / width_r) ** 2)
        f_z = np.exp(-((z - z_peak) / width_z) ** 2)
        self._heat_r = float(Q_max) * f_r
        self._heat_z = f_z
        self._Q_max = float(Q_max)
        self._grid = (nx, ny, nz)

    @property
    def heat_factors(self):
        return self._heat_r, self._heat_z

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        if tuple(state.theta_prime.shape) != self._grid:
            raise ValueError("DiabaticHeatingComponent grid does not match the state")
        p = _plan_for(state.u, base, heating=True, heat_r=self._heat_r, heat_z=self._heat_z)
        _, _, _, dth = p.tendency(L.OB_TEND_HEATING, state.u, state.v, state.w,
                                  state.theta_prime, float(dt))
        return Tendency(dtheta_prime_dt=dth)

    def reads(self):
        return ()

    def writes(self):
        return (StateVar.THETA_PRIME,)


class HelmholtzDivergenceDampingComponent(TendencyComponent):
    """Damp the divergent (irrotational) horizontal flow by epsilon per slow
    half step, fully spectral (tendency.py:1741-1845)."""
    name = "helmholtz_divergence_damping"
    stage = StepStage.SLOW

    def __init__(self, epsilon: float, Lx: float, Ly: float, nx: int, ny: int) -> None:
        self._epsilon = float(epsilon)
        self._dx, self._dy = Lx / nx, Ly / ny
        self._grid = (int(nx), int(ny), float(Lx), float(Ly))

    @property
    def epsilon(self):
        return self._epsilon

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        nx, ny, Lx, Ly = self._grid
        p = _plan_for(state.u, base, Lx, Ly, 1.0, damping=True, epsilon=self._epsilon)
        du, dv, _, _ = p.tendency(L.OB_TEND_DAMPING, state.u, state.v, state.w,
                                  state.theta_prime, float(dt))
        return Tendency(du_dt=du, dv_dt=dv)

    def reads(self):
        return (StateVar.U, StateVar.V)

    def writes(self):
        return (StateVar.U, StateVar.V)


# ---------------------------------------------------------------------------
# Production slow components (tendency.py:1259-1668) and the intensity cap.
# Each stores the reference's constructor arguments under the reference's
# attribute names, so that compile_config reads a reference object and one of
# these alike (the *_fields helpers below).
# ---------------------------------------------------------------------------

def _base_z(base, nz):
    if base is None or getattr(base, "z", None) is None:
        raise ValueError("this component needs the base state's z levels")
    z = np.asarray(to_numpy(base.z), dtype=np.float64).reshape(-1)
    if z.shape != (nz,):
        raise ValueError(f"base.z has shape {z.shape}, expected ({nz},)")
    return z


def drag_fields(comp, z) -> dict:
    """PlanSpec fields of a SurfaceDragComponent (tendency.py:1318-1338): the
    level spacing and the vertical weight exactly as the reference forms them."""
    dz = float(z[1] - z[0]) if len(z) > 1 else float(z[0])
    weight = np.maximum(0.0, 1.0 - z / float(comp._H_bl))
    return dict(drag=True, drag_cd=float(comp._Cd), drag_dz=dz, drag_u_env=float(comp._u_env),
                drag_v_env=float(comp._v_env), drag_weight=weight)


def sponge_fields(comp, z) -> dict:
    """PlanSpec fields of a SpongeDampingComponent: its full- and half-level
    damping rates (tendency.py:1478-1498)."""
    z_sp, Lz, amax = float(comp._z_sponge), float(comp._Lz), float(comp._alpha_max)
    alpha = np.zeros_like(z)
    above = z > z_sp
    if np.any(above):
        alpha[above] = amax * ((z[above] - z_sp) / (Lz - z_sp)) ** 2
    nz = len(z)
    ah = np.zeros(nz + 1)
    ah[1:-1] = 0.5 * (alpha[:-1] + alpha[1:])
    ah[0] = alpha[0]
    ah[-1] = alpha[-1]
    return dict(sponge=True, sponge_u_env=float(comp._u_env), sponge_v_env=float(comp._v_env),
                sponge_alpha=alpha, sponge_alpha_h=ah)


def diffusion_fields(comp) -> dict:
    """PlanSpec fields of a HorizontalDiffusionComponent (nu_H, Laplacian) or
    a HyperDiffusionComponent (nu4, biharmonic)."""
    if hasattr(comp, "_nu4"):
        return dict(diffusion=L.OB_DIFF_BIHARMONIC, diff_nu=float(comp._nu4),
                    diff_dx2=float(comp._dx2), diff_dy2=float(comp._dy2))
    return dict(diffusion=L.OB_DIFF_LAPLACIAN, diff_nu=float(comp._nu_H),
                diff_dx2=float(comp._dx2), diff_dy2=float(comp._dy2))


def cooling_fields(comp) -> dict:
    return dict(cooling=True, cool_alpha=float(comp._alpha))


class SurfaceDragComponent(TendencyComponent):
    """Bulk aerodynamic drag on the perturbation wind (u - u_env, v - v_env)
    with the rate Cd |V'(k=0)| / dz tapered linearly to zero at H_bl
    (tendency.py:1259-1357)."""
    name = "surface_drag"
    stage = StepStage.SLOW

    def __init__(self, Cd: float = 1.5e-3, H_bl: float = 1000.0, u_env: float = 0.0,
                 v_env: float = 0.0) -> None:
        self._Cd = float(Cd)
        self._H_bl = float(H_bl)
        self._u_env = float(u_env)
        self._v_env = float(v_env)

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        z = _base_z(base, int(state.u.shape[2]))
        p = _plan_for(state.u, base, **drag_fields(self, z))
        du, dv, _, _ = p.tendency(L.OB_TEND_DRAG, state.u, state.v, state.w,
                                  state.theta_prime, float(dt))
        return Tendency(du_dt=du, dv_dt=dv)

    def set_env(self, u_env: float, v_env: float) -> None:
        """tendency.py:1340-1351."""
        self._u_env = float(u_env)
        self._v_env = float(v_env)

    def reads(self):
        return (StateVar.U, StateVar.V)

    def writes(self):
        return (StateVar.U, StateVar.V)


class SpongeDampingComponent(TendencyComponent):
    """Rayleigh damping of the perturbations toward the environment near the
    lid, quadratic in height above z_sp = Lz (1 - sponge_fraction)
    (tendency.py:1417-1514)."""
    name = "sponge_damping"
    stage = StepStage.SLOW

    def __init__(self, Lz: float = 10_000.0, alpha_max: float = 0.01,
                 sponge_fraction: float = 0.3, u_env: float = 0.0, v_env: float = 0.0) -> None:
        self._Lz = Lz
        self._alpha_max = alpha_max
        self._z_sponge = Lz * (1.0 - sponge_fraction)
        self._u_env = u_env
        self._v_env = v_env

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        z = _base_z(base, int(state.u.shape[2]))
        p = _plan_for(state.u, base, **sponge_fields(self, z))
        du, dv, dw, dth = p.tendency(L.OB_TEND_SPONGE, state.u, state.v, state.w,
                                     state.theta_prime, float(dt))
        return Tendency(du_dt=du, dv_dt=dv, dw_dt=dw, dtheta_prime_dt=dth)

    def reads(self):
        return (StateVar.U, StateVar.V, StateVar.W, StateVar.THETA_PRIME)

    def writes(self):
        return (StateVar.U, StateVar.V, StateVar.W, StateVar.THETA_PRIME)


class HorizontalDiffusionComponent(TendencyComponent):
    """Second-order horizontal Laplacian diffusion of u, v, periodic
    5-point stencil (tendency.py:1517-1566)."""
    name = "horizontal_diffusion"
    stage = StepStage.SLOW

    def __init__(self, nu_H: float, Lx: float, Ly: float, nx: int, ny: int) -> None:
        self._nu_H = float(nu_H)
        self._dx2 = (Lx / nx) ** 2
        self._dy2 = (Ly / ny) ** 2

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        p = _plan_for(state.u, base, **diffusion_fields(self))
        du, dv, _, _ = p.tendency(L.OB_TEND_DIFFUSION, state.u, state.v, state.w,
                                  state.theta_prime, float(dt))
        return Tendency(du_dt=du, dv_dt=dv)

    def reads(self):
        return (StateVar.U, StateVar.V)

    def writes(self):
        return (StateVar.U, StateVar.V)


class HyperDiffusionComponent(TendencyComponent):
    """Fourth-order (biharmonic) horizontal diffusion of u, v as two
    applications of the 5-point Laplacian (tendency.py:1569-1627)."""
    name = "hyper_diffusion"
    stage = StepStage.SLOW

    def __init__(self, nu4: float, Lx: float, Ly: float, nx: int, ny: int) -> None:
        self._nu4 = float(nu4)
        self._dx2 = (Lx / nx) ** 2
        self._dy2 = (Ly / ny) ** 2

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        p = _plan_for(state.u, base, **diffusion_fields(self))
        du, dv, _, _ = p.tendency(L.OB_TEND_DIFFUSION, state.u, state.v, state.w,
                                  state.theta_prime, float(dt))
        return Tendency(du_dt=du, dv_dt=dv)

    def reads(self):
        return (StateVar.U, StateVar.V)

    def writes(self):
        return (StateVar.U, StateVar.V)


class NewtonianCoolingComponent(TendencyComponent):
    """Relaxation of theta' toward zero on the time scale tau
    (tendency.py:1630-1668)."""
    name = "newtonian_cooling"
    stage = StepStage.SLOW

    def __init__(self, tau: float = 3600.0) -> None:
        self._alpha = 1.0 / float(tau)

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        p = _plan_for(state.u, base, **cooling_fields(self))
        _, _, _, dth = p.tendency(L.OB_TEND_COOLING, state.u, state.v, state.w,
                                  state.theta_prime, float(dt))
        return Tendency(dtheta_prime_dt=dth)

    def reads(self):
        return (StateVar.THETA_PRIME,)

    def writes(self):
        return (StateVar.THETA_PRIME,)


class IntensityCapComponent(TendencyComponent):
    """Perturbation-wind speed limiter (tendency.py:1360-1414): relaxes
    |V'| toward v_cap where it exceeds it, preserving direction.  Not an
    OperatorConfig slot: the reference's run loop adds dt times this
    tendency to the state after each step (run_storm.py:168-172)."""
    name = "intensity_cap"
    stage = StepStage.SLOW

    def __init__(self, v_cap: float = 70.0, tau: float = 300.0, u_env: float = 0.0,
                 v_env: float = 0.0) -> None:
        self._v_cap = float(v_cap)
        self._tau = float(tau)
        self._u_env = float(u_env)
        self._v_env = float(v_env)

    def compute_tendency(self, state, equation_set, staggering, base, dt):
        u, v = state.u, state.v
        if not (isinstance(u, torch.Tensor) and u.is_cuda):
            raise TypeError("IntensityCapComponent reads device fields (CUDA torch tensors)")
        if u.dtype not in (torch.float64, torch.float32) or v.dtype != u.dtype:
            raise ValueError("u and v must share a float64 or float32 dtype")
        if tuple(v.shape) != tuple(u.shape):
            raise ValueError("u and v must have the same shape")
        u, v = u.contiguous(), v.contiguous()
        du, dv = torch.empty_like(u), torch.empty_like(v)
        lib = L.load()
        prec = L.OB_PREC_F64 if u.dtype == torch.float64 else L.OB_PREC_F32
        stream = torch.cuda.current_stream(u.device).cuda_stream
        L.check(lib.oracle_b200_intensity_cap(
            ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(v.data_ptr()), prec, u.numel(),
            self._v_cap, self._tau, self._u_env, self._v_env, ctypes.c_void_p(du.data_ptr()),
            ctypes.c_void_p(dv.data_ptr()), ctypes.c_void_p(stream)))
        return Tendency(du_dt=du, dv_dt=dv)

    def set_env(self, u_env: float, v_env: float) -> None:
        """tendency.py:1405-1408."""
        self._u_env = float(u_env)
        self._v_env = float(v_env)

    def reads(self):
        return (StateVar.U, StateVar.V)

    def writes(self):
        return (StateVar.U, StateVar.V)
