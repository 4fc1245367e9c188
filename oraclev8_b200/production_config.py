"""Base-state builder of the LH82 runs (production_config.py:94-109)."""
from __future__ import annotations

import numpy as np

from .constants import C_P, GRAVITY, P_REF, R_D


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
