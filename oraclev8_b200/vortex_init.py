"""Holland (1980) balanced vortex initial state (oracle_v8/vortex_init.py:75-411).

The radial gradient-wind integral and the hydrostatic theta' profiles are
FP64 NumPy tables on the host (O(n_radial nz + nx ny)); the per-cell
interpolation and wind expansion run on the device (``oracle_b200_vortex_fill``)
with numpy's rounding, so both paths give the same fields.  ``wind_decay_top`` selects the
linear wind structure max(0, 1 - z/top) the beta-drift workloads use in place
of exp(-z/H_wind).
"""
from __future__ import annotations

import numpy as np

from .constants import GRAVITY
from .backend import asarray, to_numpy


class HollandVortexInit:
    def __init__(self, Vmax, Rmax, B=1.5, f=5e-5, R_env=None, u_env=0.0, v_env=0.0,
                 n_radial=4000, z_peak=8_000.0, sigma_z=4_000.0, H_wind=15_000.0,
                 wind_taper=False, taper_start_frac=0.5, wind_decay_top=None):
        self.Vmax, self.Rmax, self.B, self.f = float(Vmax), float(Rmax), float(B), float(f)
        self.R_env = float(R_env) if R_env is not None else 10.0 * Rmax
        self.u_env, self.v_env = float(u_env), float(v_env)
        self.n_radial = int(n_radial)
        self.z_peak, self.sigma_z, self.H_wind = float(z_peak), float(sigma_z), float(H_wind)
        self.wind_taper = bool(wind_taper)
        self.taper_start_frac = float(taper_start_frac)
        self.wind_decay_top = None if wind_decay_top is None else float(wind_decay_top)
        self._r1d = np.linspace(0.0, self.R_env, self.n_radial)

    def tangential_wind(self, r):
        """V = Vmax sqrt(x e^{1-x}), x = (Rmax/r)^B, V(0) = 0 (vortex_init.py:169-189)."""
        r_safe = np.where(r > 0.0, r, 1.0)
        x = (self.Rmax / r_safe) ** self.B
        Vt = self.Vmax * np.sqrt(x * np.exp(1.0 - x))
        Vt = np.where(r > 0.0, Vt, 0.0)
        if self.wind_taper:
            r0 = self.taper_start_frac * self.R_env
            frac = np.clip((r - r0) / max(self.R_env - r0, 1e-9), 0.0, 1.0)
            Vt = Vt * 0.5 * (1.0 + np.cos(np.pi * frac))
        return Vt

    def vertical_structure(self, z):
        """The warm core's Gaussian S(z) = exp(-(z - z_peak)^2 / (2 sigma_z^2))
        (vortex_init.py:191-204)."""
        return np.exp(-0.5 * ((np.asarray(z) - self.z_peak) / self.sigma_z) ** 2)

    def surface_pressure_deficit(self, rho_bar_surface):
        """P'(r = 0) at the surface in Pa, negative for a cyclone
        (vortex_init.py:376-382)."""
        return float(self._pressure_deficit_1d(rho_bar_surface, 1.0)[0])

    def peak_wind_check(self):
        """(radius, speed) of the largest tangential wind on the radial grid
        (vortex_init.py:384-391)."""
        vt = self.tangential_wind(self._r1d)
        i = int(np.argmax(vt))
        return float(self._r1d[i]), float(vt[i])

    def summary(self):
        """The reference's one-line log of the vortex (vortex_init.py:393-411)."""
        _, _ = self.peak_wind_check()
        p_min = self.surface_pressure_deficit(rho_bar_surface=1.15)
        if self.wind_taper:
            taper = (f"wind_taper=ON start={self.taper_start_frac * self.R_env / 1000:.0f} km "
                     f"(frac={self.taper_start_frac:.2f})  ")
        else:
            taper = "wind_taper=OFF  "
        return (f"HollandVortex: Vmax={self.Vmax:.0f} m/s  Rmax={self.Rmax / 1000:.0f} km  "
                f"B={self.B:.2f}  f={self.f:.2e}  R_env={self.R_env / 1000:.0f} km  {taper}"
                f"P_min~{p_min:.0f} Pa  z_peak={self.z_peak / 1000:.0f} km  "
                f"sz={self.sigma_z / 1000:.0f} km  u_env={self.u_env:.1f}  "
                f"v_env={self.v_env:.1f} m/s")

    def wind_vertical_structure(self, z):
        if self.wind_decay_top is not None:
            return np.maximum(0.0, 1.0 - z / self.wind_decay_top)
        return np.exp(-z / self.H_wind)

    def _pressure_deficit_1d(self, rho_z, S_z):
        """Inward trapezoid of dP/dr = rho (V^2/r + f V) (vortex_init.py:223-255).
        The reference's recurrence P[i] = P[i+1] - term[i] (from P = 0 at the
        outer edge) is a strictly sequential running sum of -term from the
        outside in, which numpy's cumulative sum evaluates in the same order
        (add.accumulate is sequential), so the values are identical."""
        r = self._r1d
        if getattr(self, "_vt1d", None) is None:
            self._vt1d = self.tangential_wind(r)
        Vt = self._vt1d * S_z
        r_safe = np.where(r > 0.0, r, 1.0)
        dPdr = rho_z * (np.where(r > 0.0, Vt ** 2 / r_safe, 0.0) + self.f * Vt)
        dr = r[1] - r[0]
        P = np.zeros(self.n_radial)
        terms = 0.5 * (dPdr[:-1] + dPdr[1:]) * dr
        P[:-1] = np.cumsum(-terms[::-1])[::-1]
        return P

    def _tables(self, nx, ny, nz, Lx, Ly, base, x_c, y_c):
        """Column tables (r, V_t(r), sin, cos) and theta' radial profiles
        (vortex_init.py:261-329), FP64 on the host: O(nx ny + n_radial nz)."""
        x_c = x_c if x_c is not None else Lx / 2.0
        y_c = y_c if y_c is not None else Ly / 2.0
        dx, dy = Lx / nx, Ly / ny
        x = (np.arange(nx) + 0.5) * dx
        y = (np.arange(ny) + 0.5) * dy
        X, Y = np.meshgrid(x, y, indexing="ij")
        dX, dY = X - x_c, Y - y_c
        R2d = np.sqrt(dX ** 2 + dY ** 2)
        PHI = np.arctan2(dY, dX)
        z = np.asarray(to_numpy(base.z), dtype=np.float64)
        rho0 = np.asarray(to_numpy(base.rho0), dtype=np.float64)
        theta0 = np.asarray(to_numpy(base.theta0), dtype=np.float64)
        S = self.wind_vertical_structure(z)
        Pp = np.zeros((self.n_radial, nz))
        for k in range(nz):
            Pp[:, k] = self._pressure_deficit_1d(float(rho0[k]), float(S[k]))
        dP = np.empty_like(Pp)
        dP[:, 1:-1] = (Pp[:, 2:] - Pp[:, :-2]) / (z[2:] - z[:-2])[None, :]
        dP[:, 0] = (Pp[:, 1] - Pp[:, 0]) / (z[1] - z[0])
        dP[:, -1] = (Pp[:, -1] - Pp[:, -2]) / (z[-1] - z[-2])
        theta_rad = (theta0[None, :] / (rho0[None, :] * GRAVITY)) * dP
        return R2d, self.tangential_wind(R2d), np.sin(PHI), np.cos(PHI), S, theta_rad

    def build_state(self, nx, ny, nz, Lx, Ly, base, x_c=None, y_c=None, device=True,
                    dtype=None):
        """Balanced State (vortex_init.py:261-370).  ``device=True`` expands the
        host tables into the device fields with one kernel (identical values to
        the host path); ``device=False`` returns host NumPy fields.  ``dtype``:
        device dtype (default the backend's)."""
        from .solver.tendency import State
        R2d, Vt0, sin_phi, cos_phi, S, theta_rad = self._tables(nx, ny, nz, Lx, Ly, base,
                                                                x_c, y_c)
        if device:
            return self._fill_device(nx, ny, nz, R2d, Vt0, sin_phi, cos_phi, S, theta_rad,
                                     dtype)
        rf = R2d.ravel()
        th = np.empty((nx, ny, nz))
        for k in range(nz):
            th[:, :, k] = np.interp(rf, self._r1d, theta_rad[:, k]).reshape(nx, ny)
        u = np.empty((nx, ny, nz))
        v = np.empty((nx, ny, nz))
        for k in range(nz):
            Vt = Vt0 * float(S[k])
            u[:, :, k] = -Vt * sin_phi + self.u_env
            v[:, :, k] = +Vt * cos_phi + self.v_env
        w = np.zeros((nx, ny, nz + 1))
        phi = np.zeros((nx, ny, nz))
        return State(u, v, w, th, phi, 0.0)

    def _fill_device(self, nx, ny, nz, R2d, Vt0, sin_phi, cos_phi, S, theta_rad, dtype):
        import ctypes

        import torch

        from . import _lib as L
        from .backend import DTYPE, _device
        from .solver.tendency import State
        dev = _device()
        dtype = dtype or DTYPE
        lib = L.load()
        f64 = dict(dtype=torch.float64, device=dev)
        col = torch.as_tensor(np.stack([R2d, Vt0, sin_phi, cos_phi], axis=-1).reshape(-1),
                              **f64)
        S_d = torch.as_tensor(np.ascontiguousarray(S, dtype=np.float64), **f64)
        rr = torch.as_tensor(self._r1d, **f64)
        tab = torch.as_tensor(np.ascontiguousarray(theta_rad), **f64)
        u = torch.empty((nx, ny, nz), dtype=dtype, device=dev)
        v, th, phi = torch.empty_like(u), torch.empty_like(u), torch.empty_like(u)
        w = torch.empty((nx, ny, nz + 1), dtype=dtype, device=dev)
        prec = {torch.float64: L.OB_PREC_F64, torch.float32: L.OB_PREC_F32}[dtype]
        ptrs = L.StatePtrs(*(ctypes.c_void_p(t.data_ptr()) for t in (u, v, w, th, phi)))
        vp = lambda t: ctypes.c_void_p(t.data_ptr())
        L.check(lib.oracle_b200_vortex_fill(
            nx, ny, nz, prec, vp(col), vp(S_d), vp(rr), vp(tab), int(self.n_radial),
            self.u_env, self.v_env, ctypes.byref(ptrs),
            ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
        return State(u, v, w, th, phi, 0.0)
