"""Variable-coefficient anelastic Poisson solver on the B200 backend.

Mirrors oracle_v8/solver/poisson.py:98-383: div(rho grad phi) = d, periodic
in x, y (real FFT), rigid lid in z (Thomas per wavenumber column), zero mode
solved on its reduced system with phi(0,0,0) = 0.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _lib as L
from .._plan import PlanSpec, cached_plan, precision_of
from ..backend import to_numpy
from .tendency import PoissonSolveResult


class VariableCoefficientPoissonSolver:
    def __init__(self, nx: int, ny: int, nz: int, Lx: float, Ly: float, Lz: float):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.dx, self.dy, self.dz = Lx / nx, Ly / ny, Lz / nz
        self.kx = 2.0 * np.pi * np.fft.fftfreq(nx, d=self.dx)
        self.ky = 2.0 * np.pi * np.fft.fftfreq(ny, d=self.dy)
        KX, KY = np.meshgrid(self.kx, self.ky, indexing="ij")
        self.k_sq = KX ** 2 + KY ** 2

    def _plan(self, like: torch.Tensor, rho_bar_full, rho_bar_half=None):
        rf = np.asarray(to_numpy(rho_bar_full), dtype=np.float64)
        if rho_bar_half is not None:
            rh = np.asarray(to_numpy(rho_bar_half), dtype=np.float64)
            exp = np.empty(self.nz + 1)
            exp[1:-1] = 0.5 * (rf[:-1] + rf[1:])
            exp[0], exp[-1] = rf[0], rf[-1]
            if not np.array_equal(rh, exp):
                raise ValueError("rho_bar_half must be the Lorenz average of rho_bar_full "
                                 "with boundary copies (tendency.py:748-754)")
        spec = PlanSpec(nx=self.nx, ny=self.ny, nz=self.nz, Lx=self.Lx, Ly=self.Ly,
                        Lz=self.Lz, rho0=rf, theta0=np.full(self.nz, 300.0),
                        precision=precision_of(like))
        return cached_plan(spec)

    def apply_operator(self, phi, rho_bar_full, rho_bar_half):
        """div(rho grad phi) with the solver's stencil (poisson.py:139-200)."""
        return self._plan(phi, rho_bar_full, rho_bar_half).apply_operator(phi.contiguous())

    def solve(self, d, rho_bar_full, rho_bar_half, log_diagnostics: bool = True):
        """poisson.py:202-277."""
        p = self._plan(d, rho_bar_full, rho_bar_half)
        phi = p.poisson_solve(d.contiguous(), log_diag=log_diagnostics)
        if log_diagnostics:
            dg = p.read_diag()
            compat = float(dg[L.DIAG["last_compat"]])
            disc = float(dg[L.DIAG["last_disc"]])
        else:
            compat = disc = 0.0
        return PoissonSolveResult(phi, compat, disc, self.nx * self.ny)
