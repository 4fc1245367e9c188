"""The production configuration of the LH82 runs (production_config.py):
the storm-agnostic physics constants (lines 24-54), the base-state builder
(lines 94-109) and the two OperatorConfig factories (lines 116-150) the run
loop builds its integrators from."""
from __future__ import annotations

import numpy as np

from .constants import C_P, GRAVITY, P_REF, R_D

# Physics constants, identical for every storm (production_config.py:24-54).
DT = 30.0               # s
DIAG_EVERY = 60         # steps
N_PREBAL = 5            # projection-only pre-balance iterations
RMAX_RUN_M = 75_000.0
R_ENV_M = 500_000.0
TAPER_START_M = 200_000.0
TAPER_START_FRAC = TAPER_START_M / R_ENV_M
WIND_TAPER = True
NU4 = 3.0e11            # m^4/s, biharmonic diffusion
EPSILON = 0.5           # Helmholtz divergence damping per slow half step
TAU_COOL = 1800.0       # s, Newtonian cooling
CD = 1.5e-3             # surface drag coefficient
H_BL = 1000.0           # m, drag boundary-layer depth
VMAX_CAP_MS = 70.0      # m/s ceiling on |V'|, applied by the run loop after each step
TAU_CAP = 300.0         # s
LZ = 20_000.0
NZ = 32
DX = 15_625.0           # m
STANDARD_NX = (256, 320, 384, 448, 512)
TAPER_FRAC = 0.8


def build_base_state(nz: int = 32, Lz: float = 20_000.0):
    """Return (z_centers, rho0, theta0) for the standard anelastic base state:
    theta0 = 300 exp(N^2 z / g) with N = 0.01 s^-1, Exner function integrated
    by the trapezoid rule from the surface, rho0 = p / (R_d theta0 Pi).  FP64,
    host side, built once per run."""
    dz = Lz / nz
    z = (np.arange(nz) + 0.5) * dz
    theta0 = 300.0 * np.exp(0.01 ** 2 * z / GRAVITY)
    Pi = np.zeros(nz)
    Pi[0] = 1.0 - (GRAVITY / C_P) * z[0] / theta0[0]
    for k in range(nz - 1):
        dl = z[k + 1] - z[k]
        Pi[k + 1] = Pi[k] - (GRAVITY / C_P) * (dl / 2.0) * (1.0 / theta0[k] + 1.0 / theta0[k + 1])
    p0 = P_REF * Pi ** (C_P / R_D)
    rho0 = p0 / (R_D * theta0 * Pi)
    return z, rho0, theta0


class BaseState:
    """Plain holder with the (z, rho0, theta0) attributes the integrator reads."""

    def __init__(self, nz: int, Lz: float):
        self.z, self.rho0, self.theta0 = build_base_state(nz=nz, Lz=Lz)
        self.integration_scheme = "trapezoid"


def build_prebal_config(nx, ny, nz, Lx, Ly, Lz):
    """Projection-only configuration of the pre-balance iterations
    (production_config.py:116-125)."""
    from .grid import LorenzStaggering
    from .solver import AnelasticProjection, LH82AnelasticEquationSet, OperatorConfig
    return OperatorConfig(equation_set=LH82AnelasticEquationSet(),
                          staggering=LorenzStaggering(),
                          projection=AnelasticProjection(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly,
                                                         Lz=Lz))


def build_production_config(nx, ny, nz, Lx, Ly, Lz, f, u_env, v_env):
    """The production physics (production_config.py:128-150): centred
    advection, beta-plane Coriolis with the periodic taper, biharmonic
    diffusion, Helmholtz divergence damping, Newtonian cooling and surface
    drag, with the projection; no buoyancy (barotropic).  Per storm only the
    grid, f and the steering wind change."""
    from .grid import LorenzStaggering
    from .solver import (AdvectionComponent, AnelasticProjection, CoriolisComponent,
                         HelmholtzDivergenceDampingComponent, HyperDiffusionComponent,
                         LH82AnelasticEquationSet, NewtonianCoolingComponent, OperatorConfig,
                         SurfaceDragComponent)
    return OperatorConfig(
        equation_set=LH82AnelasticEquationSet(),
        staggering=LorenzStaggering(),
        advection=AdvectionComponent(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz),
        coriolis=CoriolisComponent(f=f, mode="beta_plane", Ly=Ly, ny=ny, u_env=u_env,
                                   v_env=v_env, periodic_taper=True),
        horiz_diffusion=HyperDiffusionComponent(nu4=NU4, Lx=Lx, Ly=Ly, nx=nx, ny=ny),
        divergence_damping=HelmholtzDivergenceDampingComponent(epsilon=EPSILON, Lx=Lx, Ly=Ly,
                                                               nx=nx, ny=ny),
        newtonian_cooling=NewtonianCoolingComponent(tau=TAU_COOL),
        surface_drag=SurfaceDragComponent(Cd=CD, H_bl=H_BL, u_env=u_env, v_env=v_env),
        projection=AnelasticProjection(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz),
    )
