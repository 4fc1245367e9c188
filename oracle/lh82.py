"""NumPy restatement of the Oracle V8 LH82 anelastic step (TEST ORACLE ONLY).

Every function here restates one piece of the reference algorithm with the
same floating-point operation order, so that on identical inputs it reproduces
the reference's FP64 NumPy outputs bit for bit (pinned by
``tests/test_oracle_golden.py``).  Citations are ``path:line`` inside the
reference project (justingwatford-dev/Oraclev8).

This module is test infrastructure: the CUDA product path never calls it.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

# constants.py:25-28
GRAVITY = 9.81
R_D = 287.04
C_P = 1004.5
P_REF = 100_000.0

# tendency.py:1125-1126 (CoriolisComponent._OMEGA / _R_EARTH)
OMEGA = 7.2921e-5
R_EARTH = 6.371e6


# ---------------------------------------------------------------------------
# Base state and grid helpers
# ---------------------------------------------------------------------------

def build_base_state(nz: int, Lz: float):
    """(z, rho0, theta0) — production_config.py:94-109."""
    dz = Lz / nz
    z = (np.arange(nz) + 0.5) * dz
    theta0 = 300.0 * np.exp(0.01 ** 2 * z / GRAVITY)
    Pi = np.zeros(nz)
    Pi[0] = 1.0 - (GRAVITY / C_P) * z[0] / theta0[0]
    for k in range(nz - 1):
        dl = z[k + 1] - z[k]
        Pi[k + 1] = Pi[k] - (GRAVITY / C_P) * (dl / 2.0) * (
            1.0 / theta0[k] + 1.0 / theta0[k + 1])
    p0 = P_REF * Pi ** (C_P / R_D)
    rho0 = p0 / (R_D * theta0 * Pi)
    return z, rho0, theta0


def rho_half_levels(rho_full):
    """Half-level rho: interior mean, boundary copies — tendency.py:748-754."""
    nz = rho_full.shape[0]
    rh = np.zeros(nz + 1)
    rh[1:-1] = 0.5 * (rho_full[:-1] + rho_full[1:])
    rh[0] = rho_full[0]
    rh[-1] = rho_full[-1]
    return rh


def wavenumbers(nx, ny, Lx, Ly):
    """kx, ky = 2*pi*fftfreq(n, d) — poisson.py:126-127."""
    kx = 2.0 * np.pi * np.fft.fftfreq(nx, d=Lx / nx)
    ky = 2.0 * np.pi * np.fft.fftfreq(ny, d=Ly / ny)
    return kx, ky


# ---------------------------------------------------------------------------
# State
# ---------------------------------------------------------------------------

@dataclass
class State:
    """Prognostic state — tendency.py:145-172 (w has nz+1 half levels)."""
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    theta_prime: np.ndarray
    projection_potential: np.ndarray
    t: float = 0.0

    def copy(self) -> "State":
        return State(self.u.copy(), self.v.copy(), self.w.copy(),
                     self.theta_prime.copy(),
                     self.projection_potential.copy(), self.t)


# ---------------------------------------------------------------------------
# Fast component: buoyancy
# ---------------------------------------------------------------------------

def buoyancy_half(theta_prime, theta0):
    """b = g*theta'/theta0 on full levels, Lorenz-averaged to half levels with
    zero surface/lid — equation_set.py:255-263, staggering.py:201-208."""
    b_full = GRAVITY * theta_prime / theta0
    shp = b_full.shape[:-1] + (b_full.shape[-1] + 1,)
    out = np.zeros(shp, dtype=b_full.dtype)
    out[..., 1:-1] = 0.5 * (b_full[..., :-1] + b_full[..., 1:])
    out[..., 0] = 0.0
    out[..., -1] = 0.0
    return out


# ---------------------------------------------------------------------------
# Slow component: advection (tendency.py:835-1062)
# ---------------------------------------------------------------------------

def _cx(f, dx):
    return (np.roll(f, -1, axis=0) - np.roll(f, 1, axis=0)) / (2.0 * dx)


def _cy(f, dy):
    return (np.roll(f, -1, axis=1) - np.roll(f, 1, axis=1)) / (2.0 * dy)


def _cz(f, dz):
    """One-sided at ends, centred inside — tendency.py:922-938."""
    g = np.empty_like(f)
    g[:, :, 1:-1] = (f[:, :, 2:] - f[:, :, :-2]) / (2.0 * dz)
    g[:, :, 0] = (f[:, :, 1] - f[:, :, 0]) / dz
    g[:, :, -1] = (f[:, :, -1] - f[:, :, -2]) / dz
    return g


def _upwind5(q, a, d, axis):
    """Wicker-Skamarock 5th-order upwind derivative — tendency.py:940-959.
    a >= 0 selects the positive-biased stencil (tie at a == 0 included)."""
    qm3 = np.roll(q, 3, axis); qm2 = np.roll(q, 2, axis); qm1 = np.roll(q, 1, axis)
    qp1 = np.roll(q, -1, axis); qp2 = np.roll(q, -2, axis); qp3 = np.roll(q, -3, axis)
    d_pos = (-2.0 * qm3 + 15.0 * qm2 - 60.0 * qm1 + 20.0 * q + 30.0 * qp1 - 3.0 * qp2) / (60.0 * d)
    d_neg = (2.0 * qp3 - 15.0 * qp2 + 60.0 * qp1 - 20.0 * q - 30.0 * qm1 + 3.0 * qm2) / (60.0 * d)
    return np.where(a >= 0.0, d_pos, d_neg)


def advection_tendency(u, v, w, th, theta0, dx, dy, dz, scheme="upwind5h"):
    """(du, dv, dw, dtheta') — AdvectionComponent.compute_tendency,
    tendency.py:965-1062."""
    nz = u.shape[2]
    w_c = 0.5 * (w[:, :, :-1] + w[:, :, 1:])
    u_h = np.empty_like(w)
    u_h[:, :, 1:-1] = 0.5 * (u[:, :, :-1] + u[:, :, 1:])
    u_h[:, :, 0] = u[:, :, 0]
    u_h[:, :, -1] = u[:, :, -1]
    v_h = np.empty_like(w)
    v_h[:, :, 1:-1] = 0.5 * (v[:, :, :-1] + v[:, :, 1:])
    v_h[:, :, 0] = v[:, :, 0]
    v_h[:, :, -1] = v[:, :, -1]
    if scheme == "upwind5h":
        ddx = lambda q, a: _upwind5(q, a, dx, 0)
        ddy = lambda q, a: _upwind5(q, a, dy, 1)
    elif scheme == "centered2":
        ddx = lambda q, a: _cx(q, dx)
        ddy = lambda q, a: _cy(q, dy)
    else:
        raise ValueError(scheme)
    dth0 = np.empty(nz)
    dth0[1:-1] = (theta0[2:] - theta0[:-2]) / (2.0 * dz)
    dth0[0] = (theta0[1] - theta0[0]) / dz
    dth0[-1] = (theta0[-1] - theta0[-2]) / dz
    dth = -(u * ddx(th, u) + v * ddy(th, v) + w_c * (_cz(th, dz) + dth0[None, None, :]))
    du = -(u * ddx(u, u) + v * ddy(u, v) + w_c * _cz(u, dz))
    dv = -(u * ddx(v, u) + v * ddy(v, v) + w_c * _cz(v, dz))
    dw = -(u_h * ddx(w, u_h) + v_h * ddy(w, v_h) + w * _cz(w, dz))
    dw[:, :, 0] = 0.0
    dw[:, :, -1] = 0.0
    return du, dv, dw, dth


# ---------------------------------------------------------------------------
# Slow component: Coriolis (tendency.py:1128-1234)
# ---------------------------------------------------------------------------

def coriolis_profile(f, mode="beta_plane", beta=None, Ly=None, ny=None, y0=None,
                     periodic_taper=False):
    """f(y) at cell centres (ny,), or None for the f-plane —
    tendency.py:1153-1203."""
    if mode != "beta_plane":
        return None
    if beta is None:
        lat = np.arcsin(np.clip(f / (2.0 * OMEGA), -1.0, 1.0))
        beta = 2.0 * OMEGA * np.cos(lat) / R_EARTH
    beta = float(beta)
    dy = Ly / ny
    y_ref = y0 if y0 is not None else Ly / 2.0
    y = (np.arange(ny) + 0.5) * dy
    dev = beta * (y - y_ref)
    if periodic_taper:
        n_taper = max(1, int(round(0.20 * ny)))
        taper = np.ones(ny)
        for i in range(n_taper):
            t = np.sin(np.pi * (i + 0.5) / (2.0 * n_taper)) ** 2
            taper[i] = t
            taper[ny - 1 - i] = t
        dev = dev * taper
    return np.float64(f) + dev


def coriolis_tendency(u, v, f0, f_y, u_env=0.0, v_env=0.0):
    """du = f (v - v_env), dv = -f (u - u_env) — tendency.py:1220-1234."""
    u_p = u - float(u_env)
    v_p = v - float(v_env)
    if f_y is None:
        return +f0 * v_p, -f0 * u_p
    fy = f_y[None, :, None]
    return +fy * v_p, -fy * u_p


# ---------------------------------------------------------------------------
# Slow component: prescribed diabatic heating (tendency.py:1712-1732)
# ---------------------------------------------------------------------------

def heating_field(Q_max, r_eyewall, width_r, z_peak, width_z, nx, ny, nz,
                  Lx, Ly, Lz, x_c=None, y_c=None):
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
    return float(Q_max) * f_r[:, :, None] * f_z[None, None, :]


# ---------------------------------------------------------------------------
# Slow component: Helmholtz divergence damping (tendency.py:1777-1839)
# ---------------------------------------------------------------------------

def helmholtz_tendency(u, v, epsilon, dt, Lx, Ly):
    nx, ny = u.shape[0], u.shape[1]
    dx, dy = Lx / nx, Ly / ny
    kx = np.fft.fftfreq(nx, d=dx) * (2.0 * np.pi)
    ky = np.fft.fftfreq(ny, d=dy) * (2.0 * np.pi)
    Kx, Ky = np.meshgrid(kx, ky, indexing="ij")
    K2 = Kx ** 2 + Ky ** 2
    K2[0, 0] = 1.0
    K2_inv = np.where(K2 > 0, -1.0 / K2, 0.0)
    iKx = 1j * Kx
    iKy = 1j * Ky
    u_hat = np.fft.fft2(u, axes=(0, 1))
    v_hat = np.fft.fft2(v, axes=(0, 1))
    D_hat = iKx[:, :, None] * u_hat + iKy[:, :, None] * v_hat
    psi_hat = D_hat * K2_inv[:, :, None]
    u_div = np.real(np.fft.ifft2(iKx[:, :, None] * psi_hat, axes=(0, 1)))
    v_div = np.real(np.fft.ifft2(iKy[:, :, None] * psi_hat, axes=(0, 1)))
    eps = float(epsilon)
    return -(eps / dt) * u_div, -(eps / dt) * v_div


# ---------------------------------------------------------------------------
# Shared operators (tendency.py:393-500)
# ---------------------------------------------------------------------------

# ---------------------------------------------------------------------------
# Production slow components (tendency.py:1259-1668) and the intensity cap
# ---------------------------------------------------------------------------

def surface_drag_tendency(u, v, z, Cd=1.5e-3, H_bl=1000.0, u_env=0.0, v_env=0.0):
    """SurfaceDragComponent — tendency.py:1318-1338: bulk drag on the
    perturbation wind, rate Cd |V'(k=0)| / dz tapered linearly to 0 at H_bl."""
    dz = float(z[1] - z[0]) if len(z) > 1 else float(z[0])
    u_p = u - u_env
    v_p = v - v_env
    V_sfc = np.sqrt(u_p[:, :, 0] ** 2 + v_p[:, :, 0] ** 2)
    alpha_sfc = Cd * V_sfc / dz
    weight = np.maximum(0.0, 1.0 - z / H_bl)
    alpha = alpha_sfc[:, :, None] * weight[None, None, :]
    return -alpha * u_p, -alpha * v_p


def sponge_profiles(z, Lz=10_000.0, alpha_max=0.01, sponge_fraction=0.3):
    """SpongeDampingComponent._alpha_full and the half-level profile —
    tendency.py:1478-1498."""
    z_sp = Lz * (1.0 - sponge_fraction)
    alpha = np.zeros_like(z)
    above = z > z_sp
    if np.any(above):
        alpha[above] = alpha_max * ((z[above] - z_sp) / (Lz - z_sp)) ** 2
    nz = len(z)
    ah = np.zeros(nz + 1)
    ah[1:-1] = 0.5 * (alpha[:-1] + alpha[1:])
    ah[0] = alpha[0]
    ah[-1] = alpha[-1]
    return alpha, ah


def sponge_tendency(u, v, w, th, z, Lz=10_000.0, alpha_max=0.01, sponge_fraction=0.3,
                    u_env=0.0, v_env=0.0):
    """SpongeDampingComponent.compute_tendency — tendency.py:1489-1508."""
    alpha, ah = sponge_profiles(z, Lz, alpha_max, sponge_fraction)
    return (-alpha[None, None, :] * (u - u_env), -alpha[None, None, :] * (v - v_env),
            -ah[None, None, :] * w, -alpha[None, None, :] * th)


def laplacian_h(f, dx2, dy2):
    """Periodic 5-point horizontal Laplacian — tendency.py:1551-1558 and
    HyperDiffusionComponent._laplacian (tendency.py:1608-1613)."""
    return ((np.roll(f, -1, axis=0) - 2.0 * f + np.roll(f, +1, axis=0)) / dx2
            + (np.roll(f, -1, axis=1) - 2.0 * f + np.roll(f, +1, axis=1)) / dy2)


def horizontal_diffusion_tendency(u, v, nu_H, Lx, Ly, nx, ny):
    """HorizontalDiffusionComponent — tendency.py:1548-1562."""
    dx2, dy2 = (Lx / nx) ** 2, (Ly / ny) ** 2
    return nu_H * laplacian_h(u, dx2, dy2), nu_H * laplacian_h(v, dx2, dy2)


def hyper_diffusion_tendency(u, v, nu4, Lx, Ly, nx, ny):
    """HyperDiffusionComponent — tendency.py:1615-1621 (two Laplacians)."""
    dx2, dy2 = (Lx / nx) ** 2, (Ly / ny) ** 2
    bu = laplacian_h(laplacian_h(u, dx2, dy2), dx2, dy2)
    bv = laplacian_h(laplacian_h(v, dx2, dy2), dx2, dy2)
    return -float(nu4) * bu, -float(nu4) * bv


def newtonian_cooling_tendency(th, tau=3600.0):
    """NewtonianCoolingComponent — tendency.py:1658-1662."""
    return -(1.0 / float(tau)) * th


def intensity_cap_tendency(u, v, v_cap=70.0, tau=300.0, u_env=0.0, v_env=0.0):
    """IntensityCapComponent.compute_tendency — tendency.py:1396-1403."""
    u_p = u - u_env
    v_p = v - v_env
    spd = np.sqrt(u_p ** 2 + v_p ** 2)
    excess = np.maximum(0.0, spd - v_cap)
    alpha = excess / (tau * np.maximum(spd, 1e-6))
    return -alpha * u_p, -alpha * v_p


def anelastic_divergence(u, v, w, rho_full, rho_half, kx, ky, dz):
    """d = div(rho u) — tendency.py:393-437."""
    rho_u = rho_full[None, None, :] * u
    rho_v = rho_full[None, None, :] * v
    ikx = 1j * kx[:, None, None]
    iky = 1j * ky[None, :, None]
    rho_u_hat = np.fft.fft2(rho_u, axes=(0, 1))
    rho_v_hat = np.fft.fft2(rho_v, axes=(0, 1))
    d_hat = ikx * rho_u_hat + iky * rho_v_hat
    horiz = np.real(np.fft.ifft2(d_hat, axes=(0, 1)))
    lower = rho_half[None, None, :-1] * w[:, :, :-1]
    upper = rho_half[None, None, 1:] * w[:, :, 1:]
    vert = (upper - lower) / dz
    return horiz + vert


def phi_gradient(phi, kx, ky, dz):
    """Spectral d/dx, d/dy on full levels; (phi[k]-phi[k-1])/dz on interior
    half levels, zero at surface and lid — tendency.py:440-500."""
    phi_hat = np.fft.fft2(phi, axes=(0, 1))
    ikx = 1j * kx[:, None, None]
    iky = 1j * ky[None, :, None]
    dx_ = np.real(np.fft.ifft2(ikx * phi_hat, axes=(0, 1)))
    dy_ = np.real(np.fft.ifft2(iky * phi_hat, axes=(0, 1)))
    nx, ny, nz = phi.shape
    dz_ = np.zeros((nx, ny, nz + 1), dtype=phi.dtype)
    dz_[:, :, 1:-1] = (phi[:, :, 1:] - phi[:, :, :-1]) / dz
    return dx_, dy_, dz_


# ---------------------------------------------------------------------------
# Variable-coefficient Poisson solver (poisson.py:98-383)
# ---------------------------------------------------------------------------

class Poisson:
    """FFT(x,y) + cached Thomas(z) solve of div(rho grad phi) = d with the
    zero mode solved on a reduced system — poisson.py:98-383."""

    def __init__(self, nx, ny, nz, Lx, Ly, Lz):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dz = Lz / nz
        self.kx, self.ky = wavenumbers(nx, ny, Lx, Ly)
        KX, KY = np.meshgrid(self.kx, self.ky, indexing="ij")
        self.k_sq = KX ** 2 + KY ** 2
        self._cache = None

    def thomas_factors(self, rho_full, rho_half):
        """Cached coefficients and forward-elimination factors —
        poisson.py:279-332."""
        if self._cache is not None and self._cache["refs"][0] is rho_full \
                and self._cache["refs"][1] is rho_half:
            return self._cache
        dz2 = self.dz ** 2
        rl = rho_half[:-1] / dz2
        ru = rho_half[1:] / dz2
        nz = self.nz
        ksq = self.k_sq.reshape(self.nx * self.ny)[1:]
        a = rl.copy(); a[0] = 0.0; a[-1] = rl[-1]
        c = ru.copy(); c[-1] = 0.0
        b = (-(rl[None, :] + ru[None, :]) - ksq[:, None] * rho_full[None, :])
        b[:, 0] = -ru[0] - ksq * rho_full[0]
        b[:, -1] = -rl[-1] - ksq * rho_full[-1]
        inv = np.empty_like(b)
        cp = np.empty_like(b)
        inv[:, 0] = 1.0 / b[:, 0]
        cp[:, 0] = c[0] * inv[:, 0]
        for k in range(1, nz):
            den = b[:, k] - a[k] * cp[:, k - 1]
            inv[:, k] = 1.0 / den
            if k < nz - 1:
                cp[:, k] = c[k] * inv[:, k]
        a0 = rl[1:].copy(); b0 = -(rl[1:] + ru[1:]); c0 = ru[1:].copy()
        a0[0] = 0.0; a0[-1] = rl[-1]; c0[-1] = 0.0; b0[-1] = -rl[-1]
        n0 = nz - 1
        inv0 = np.empty(n0); cp0 = np.empty(n0)
        inv0[0] = 1.0 / b0[0]; cp0[0] = c0[0] * inv0[0]
        for k in range(1, n0):
            den = b0[k] - a0[k] * cp0[k - 1]
            inv0[k] = 1.0 / den
            cp0[k] = c0[k] * inv0[k] if k < n0 - 1 else 0.0
        self._cache = dict(refs=(rho_full, rho_half), a=a, cp=cp, inv=inv,
                           a0=a0, cp0=cp0, inv0=inv0)
        return self._cache

    def apply_operator(self, phi, rho_full, rho_half):
        """div(rho grad phi) with the solver's stencil — poisson.py:139-200."""
        phi_hat = np.fft.fft2(phi, axes=(0, 1))
        lap = np.real(np.fft.ifft2(-self.k_sq[:, :, None] * phi_hat, axes=(0, 1)))
        horiz = rho_full[None, None, :] * lap
        dz2 = self.dz ** 2
        flux = rho_half[None, None, 1:-1] * (phi[:, :, 1:] - phi[:, :, :-1])
        vert = np.empty_like(phi)
        vert[:, :, 0] = flux[:, :, 0] / dz2
        vert[:, :, 1:-1] = (flux[:, :, 1:] - flux[:, :, :-1]) / dz2
        vert[:, :, -1] = -flux[:, :, -1] / dz2
        return horiz + vert

    def solve(self, d, rho_full, rho_half, log_diagnostics=False):
        """Returns (phi, compat_residual, disc_residual) — poisson.py:202-277."""
        d_hat = np.fft.fft2(d, axes=(0, 1))
        compat = (float(np.abs(np.sum(d_hat[0, 0, :]) * self.dz))
                  if log_diagnostics else 0.0)
        d_hat[0, 0, :] -= np.sum(d_hat[0, 0, :]) / self.nz
        cache = self.thomas_factors(rho_full, rho_half)
        phi_hat = self._solve_batch(d_hat, cache)
        phi = np.real(np.fft.ifft2(phi_hat, axes=(0, 1)))
        if log_diagnostics:
            r = self.apply_operator(phi, rho_full, rho_half) - d
            r -= np.mean(r)
            disc = float(np.sqrt(np.mean(r ** 2)))
        else:
            disc = 0.0
        return phi, compat, disc

    def _solve_batch(self, d_hat, cache):
        """poisson.py:334-365, zero mode poisson.py:367-383."""
        n = self.nx * self.ny
        nz = self.nz
        flat = d_hat.reshape(n, nz)
        rhs = flat[1:, :]
        a, cp, inv = cache["a"], cache["cp"], cache["inv"]
        dp = np.empty_like(rhs)
        dp[:, 0] = rhs[:, 0] * inv[:, 0]
        for k in range(1, nz):
            dp[:, k] = (rhs[:, k] - a[k] * dp[:, k - 1]) * inv[:, k]
        x = np.empty_like(rhs)
        x[:, -1] = dp[:, -1]
        for k in range(nz - 2, -1, -1):
            x[:, k] = dp[:, k] - cp[:, k] * x[:, k + 1]
        out = np.empty_like(flat)
        out[0, :] = self._zero_mode(flat[0, :], cache)
        out[1:, :] = x
        return out.reshape(self.nx, self.ny, nz)

    @staticmethod
    def _zero_mode(dz_h, cache):
        a0, cp0, inv0 = cache["a0"], cache["cp0"], cache["inv0"]
        n0 = len(inv0)
        rhs = dz_h[1:]
        dp = np.empty(n0, dtype=dz_h.dtype)
        dp[0] = rhs[0] * inv0[0]
        for k in range(1, n0):
            dp[k] = (rhs[k] - a0[k] * dp[k - 1]) * inv0[k]
        x = np.empty(n0, dtype=dz_h.dtype)
        x[-1] = dp[-1]
        for k in range(n0 - 2, -1, -1):
            x[k] = dp[k] - cp0[k] * x[k + 1]
        out = np.zeros(len(dz_h), dtype=dz_h.dtype)
        out[1:] = x
        return out


# ---------------------------------------------------------------------------
# Projection (tendency.py:717-790)
# ---------------------------------------------------------------------------

class Projection:
    def __init__(self, nx, ny, nz, Lx, Ly, Lz, diag_every=60):
        self.solver = Poisson(nx, ny, nz, Lx, Ly, Lz)
        self.dz = Lz / nz
        self.diag_every = max(1, int(diag_every))
        self.count = 0
        self.last = (0.0, 0.0)
        self._rho = None

    def rho_pair(self, rho_full):
        if self._rho is None or self._rho[0] is not rho_full:
            self._rho = (rho_full, rho_half_levels(rho_full))
        return self._rho

    def apply(self, st: State, rho_full) -> State:
        """In-place u,v,w correction and phi store — tendency.py:717-790."""
        rf, rh = self.rho_pair(rho_full)
        s = self.solver
        d = anelastic_divergence(st.u, st.v, st.w, rf, rh, s.kx, s.ky, self.dz)
        self.count += 1
        de = self.diag_every
        phi, compat, disc = s.solve(d, rf, rh,
                                    log_diagnostics=(de == 1 or self.count % de == 1))
        self.last = (compat, disc)
        gx, gy, gz = phi_gradient(phi, s.kx, s.ky, self.dz)
        st.u = st.u - gx
        st.v = st.v - gy
        st.w = st.w - gz
        st.projection_potential = phi
        return st


# ---------------------------------------------------------------------------
# Step configuration and RK3 integrator (integrator.py:140-505)
# ---------------------------------------------------------------------------

@dataclass
class StepConfig:
    """Which components are active, in OperatorConfig slot order
    (operator_config.py:147-160): buoyancy | projection | advection |
    coriolis | surface_drag | sponge_damping | horiz_diffusion |
    newtonian_cooling | divergence_damping | diabatic_heating."""
    nx: int
    ny: int
    nz: int
    Lx: float
    Ly: float
    Lz: float
    buoyancy: bool = True
    projection: bool = True
    advection: Optional[str] = "upwind5h"      # scheme name or None
    coriolis: Optional[dict] = None            # kwargs of CoriolisComponent
    damping_epsilon: Optional[float] = None    # HelmholtzDivergenceDamping
    heating: Optional[dict] = None             # kwargs of DiabaticHeatingComponent (no grid)
    drag: Optional[dict] = None                # kwargs of SurfaceDragComponent
    sponge: Optional[dict] = None              # kwargs of SpongeDampingComponent (Lz = grid's)
    laplacian: Optional[float] = None          # HorizontalDiffusionComponent nu_H
    hyper: Optional[float] = None              # HyperDiffusionComponent nu4
    cooling: Optional[float] = None            # NewtonianCoolingComponent tau
    poisson_diag_every: int = 60


@dataclass
class StepDiag:
    """StepDiagnostics — integrator.py:83-132."""
    step: int
    t: float
    dt: float
    stage_compat: list = field(default_factory=list)
    stage_disc: list = field(default_factory=list)
    max_u: float = 0.0
    max_v: float = 0.0
    max_w: float = 0.0
    max_theta_prime: float = 0.0
    surface_phi_min: float = 0.0
    surface_phi_max: float = 0.0


class Integrator:
    """WS-RK3 with Strang-split slow terms — integrator.py:140-505."""
    ALPHAS = (1.0 / 3.0, 1.0 / 2.0, 1.0)

    def __init__(self, cfg: StepConfig, z, rho0, theta0):
        self.cfg = cfg
        self.z, self.rho0, self.theta0 = z, rho0, theta0
        self.dx = cfg.Lx / cfg.nx
        self.dy = cfg.Ly / cfg.ny
        self.dz = cfg.Lz / cfg.nz
        self.proj = Projection(cfg.nx, cfg.ny, cfg.nz, cfg.Lx, cfg.Ly, cfg.Lz,
                               cfg.poisson_diag_every) if cfg.projection else None
        if cfg.coriolis is not None:
            c = dict(cfg.coriolis)
            self.f0 = float(c.get("f", 5e-5))
            self.u_env = float(c.get("u_env", 0.0))
            self.v_env = float(c.get("v_env", 0.0))
            self.f_y = coriolis_profile(self.f0, c.get("mode", "f_plane"), c.get("beta"),
                                        c.get("Ly"), c.get("ny"), c.get("y0"),
                                        c.get("periodic_taper", False))
        self.Q = None
        if cfg.heating is not None:
            self.Q = heating_field(nx=cfg.nx, ny=cfg.ny, nz=cfg.nz, Lx=cfg.Lx,
                                   Ly=cfg.Ly, Lz=cfg.Lz, **cfg.heating)

    def slow_active(self):
        c = self.cfg
        return bool(c.advection or c.coriolis is not None
                    or c.damping_epsilon is not None or c.heating is not None
                    or c.drag is not None or c.sponge is not None
                    or c.laplacian is not None or c.hyper is not None
                    or c.cooling is not None)

    def slow_writes_momentum(self):
        c = self.cfg
        return bool(c.advection or c.coriolis is not None or c.damping_epsilon is not None
                    or c.drag is not None or c.sponge is not None
                    or c.laplacian is not None or c.hyper is not None)

    def slow_tendency(self, st: State, dt_slow: float):
        """Summed slow tendency in slot order — integrator.py:346-357."""
        c = self.cfg
        du = np.zeros_like(st.u); dv = np.zeros_like(st.v)
        dw = np.zeros_like(st.w); dth = np.zeros_like(st.theta_prime)
        if c.advection:
            a = advection_tendency(st.u, st.v, st.w, st.theta_prime, self.theta0,
                                   self.dx, self.dy, self.dz, c.advection)
            du += a[0]; dv += a[1]; dw += a[2]; dth += a[3]
        if c.coriolis is not None:
            cu, cv = coriolis_tendency(st.u, st.v, self.f0, self.f_y, self.u_env, self.v_env)
            du += cu; dv += cv
        if c.drag is not None:
            gu, gv = surface_drag_tendency(st.u, st.v, self.z, **c.drag)
            du += gu; dv += gv
        if c.sponge is not None:
            su, sv, sw, sth = sponge_tendency(st.u, st.v, st.w, st.theta_prime, self.z,
                                              Lz=c.Lz, **c.sponge)
            du += su; dv += sv; dw += sw; dth += sth
        if c.laplacian is not None:
            lu, lv = horizontal_diffusion_tendency(st.u, st.v, c.laplacian, c.Lx, c.Ly,
                                                   c.nx, c.ny)
            du += lu; dv += lv
        if c.hyper is not None:
            bu, bv = hyper_diffusion_tendency(st.u, st.v, c.hyper, c.Lx, c.Ly, c.nx, c.ny)
            du += bu; dv += bv
        if c.cooling is not None:
            dth += newtonian_cooling_tendency(st.theta_prime, c.cooling)
        if c.damping_epsilon is not None:
            hu, hv = helmholtz_tendency(st.u, st.v, c.damping_epsilon, dt_slow, c.Lx, c.Ly)
            du += hu; dv += hv
        if self.Q is not None:
            dth += self.Q
        return du, dv, dw, dth

    def apply_slow(self, st: State, dt_slow: float) -> State:
        """integrator.py:317-392."""
        if not self.slow_active():
            return st
        du, dv, dw, dth = self.slow_tendency(st, dt_slow)
        out = State(st.u + dt_slow * du, st.v + dt_slow * dv, st.w + dt_slow * dw,
                    st.theta_prime + dt_slow * dth, st.projection_potential, st.t)
        if self.slow_writes_momentum() and self.proj is not None:
            self.proj.apply(out, self.rho0)
        return out

    def rk3_stage(self, st_n: State, st_eval: State, alpha: float, dt: float):
        """integrator.py:398-505 (buoyancy is the only fast component)."""
        sdt = alpha * dt
        du = np.zeros_like(st_n.u); dv = np.zeros_like(st_n.v)
        dw = np.zeros_like(st_n.w); dth = np.zeros_like(st_n.theta_prime)
        if self.cfg.buoyancy:
            dw += buoyancy_half(st_eval.theta_prime, self.theta0)
        prov = State(st_n.u + sdt * du, st_n.v + sdt * dv, st_n.w + sdt * dw,
                     st_n.theta_prime + sdt * dth,
                     st_eval.projection_potential.copy(), st_n.t + sdt)
        self.proj.apply(prov, self.rho0)
        return prov, self.proj.last[0], self.proj.last[1]

    def step(self, st: State, dt: float, step_number: int = 0, diag_every: int = 1):
        """integrator.py:189-311."""
        dg = StepDiag(step=step_number, t=st.t, dt=dt)
        st = self.apply_slow(st, dt * 0.5)
        st_n = st
        stage = st_n
        if self.cfg.buoyancy:
            for alpha in self.ALPHAS:
                stage, cpt, dsc = self.rk3_stage(st_n, stage, alpha, dt)
                dg.stage_compat.append(cpt)
                dg.stage_disc.append(dsc)
        else:
            stage = st_n
            if self.proj is not None:
                self.proj.apply(stage, self.rho0)
        phi_fast = stage.projection_potential.copy()
        stage = self.apply_slow(stage, dt * 0.5)
        if (diag_every == 1 or step_number % diag_every == 0
                or (step_number + 1) % diag_every == 0):
            phi_c = phi_fast - np.mean(phi_fast)
            dg.max_u = float(np.max(np.abs(stage.u)))
            dg.max_v = float(np.max(np.abs(stage.v)))
            dg.max_w = float(np.max(np.abs(stage.w)))
            dg.max_theta_prime = float(np.max(np.abs(stage.theta_prime)))
            dg.surface_phi_min = float(np.min(phi_c[:, :, 0]))
            dg.surface_phi_max = float(np.max(phi_c[:, :, 0]))
        else:
            nan = float("nan")
            dg.max_u = dg.max_v = dg.max_w = dg.max_theta_prime = nan
            dg.surface_phi_min = dg.surface_phi_max = nan
        return stage, dg


# ---------------------------------------------------------------------------
# Holland vortex initialisation (vortex_init.py:75-370)
# ---------------------------------------------------------------------------

class Holland:
    """Holland (1980) balanced vortex — vortex_init.py:92-370.  ``wind_decay_top``
    replaces the exp(-z/H) wind structure (vortex_init.py:206-217) with the
    linear decay max(0, 1 - z/top) used by the β-drift workloads."""

    def __init__(self, Vmax, Rmax, B=1.5, f=5e-5, R_env=None, u_env=0.0, v_env=0.0,
                 n_radial=4000, H_wind=15_000.0, wind_taper=False,
                 taper_start_frac=0.5, wind_decay_top=None):
        self.Vmax = float(Vmax); self.Rmax = float(Rmax); self.B = float(B)
        self.f = float(f)
        self.R_env = float(R_env) if R_env is not None else 10.0 * Rmax
        self.u_env = float(u_env); self.v_env = float(v_env)
        self.n_radial = int(n_radial); self.H_wind = float(H_wind)
        self.wind_taper = bool(wind_taper)
        self.taper_start_frac = float(taper_start_frac)
        self.wind_decay_top = wind_decay_top
        self.r1d = np.linspace(0.0, self.R_env, self.n_radial)

    def tangential_wind(self, r):
        """vortex_init.py:169-189."""
        r_safe = np.where(r > 0.0, r, 1.0)
        x = (self.Rmax / r_safe) ** self.B
        Vt = self.Vmax * np.sqrt(x * np.exp(1.0 - x))
        Vt = np.where(r > 0.0, Vt, 0.0)
        if self.wind_taper:
            r0 = self.taper_start_frac * self.R_env
            frac = np.clip((r - r0) / max(self.R_env - r0, 1e-9), 0.0, 1.0)
            Vt = Vt * 0.5 * (1.0 + np.cos(np.pi * frac))
        return Vt

    def wind_vertical_structure(self, z):
        if self.wind_decay_top is not None:
            return np.maximum(0.0, 1.0 - z / float(self.wind_decay_top))
        return np.exp(-z / self.H_wind)

    def pressure_deficit_1d(self, rho_z, S_z):
        """vortex_init.py:223-255."""
        r = self.r1d
        Vt = self.tangential_wind(r) * S_z
        r_safe = np.where(r > 0.0, r, 1.0)
        dPdr = rho_z * (np.where(r > 0.0, Vt ** 2 / r_safe, 0.0) + self.f * Vt)
        dr = r[1] - r[0]
        P = np.zeros(self.n_radial)
        for i in range(self.n_radial - 2, -1, -1):
            P[i] = P[i + 1] - 0.5 * (dPdr[i] + dPdr[i + 1]) * dr
        return P

    def build_state(self, nx, ny, nz, Lx, Ly, z, rho0, theta0, x_c=None, y_c=None):
        """vortex_init.py:261-370."""
        x_c = x_c if x_c is not None else Lx / 2.0
        y_c = y_c if y_c is not None else Ly / 2.0
        dx = Lx / nx; dy = Ly / ny
        x = (np.arange(nx) + 0.5) * dx
        y = (np.arange(ny) + 0.5) * dy
        X, Y = np.meshgrid(x, y, indexing="ij")
        dX = X - x_c; dY = Y - y_c
        R2d = np.sqrt(dX ** 2 + dY ** 2)
        PHI = np.arctan2(dY, dX)
        S = self.wind_vertical_structure(z)
        Pp = np.zeros((self.n_radial, nz))
        for k in range(nz):
            Pp[:, k] = self.pressure_deficit_1d(float(rho0[k]), float(S[k]))
        dP = np.empty_like(Pp)
        dP[:, 1:-1] = (Pp[:, 2:] - Pp[:, :-2]) / (z[2:] - z[:-2])[None, :]
        dP[:, 0] = (Pp[:, 1] - Pp[:, 0]) / (z[1] - z[0])
        dP[:, -1] = (Pp[:, -1] - Pp[:, -2]) / (z[-1] - z[-2])
        theta_rad = (theta0[None, :] / (rho0[None, :] * GRAVITY)) * dP
        r_flat = R2d.ravel()
        th = np.empty((nx, ny, nz))
        for k in range(nz):
            th[:, :, k] = np.interp(r_flat, self.r1d, theta_rad[:, k]).reshape(nx, ny)
        sin_phi = np.sin(PHI); cos_phi = np.cos(PHI)
        u = np.zeros((nx, ny, nz)); v = np.zeros((nx, ny, nz))
        for k in range(nz):
            Vt = self.tangential_wind(R2d) * float(S[k])
            u[:, :, k] = -Vt * sin_phi + self.u_env
            v[:, :, k] = +Vt * cos_phi + self.v_env
        return State(u, v, np.zeros((nx, ny, nz + 1)), th, np.zeros((nx, ny, nz)), 0.0)


# ---------------------------------------------------------------------------
# Storm tracker (storm_tracker.py:64-394)
# ---------------------------------------------------------------------------

R0_CELLS = 10.0  # storm_tracker.py:59


def theta_prime_proxy(theta_prime, z, rho0, theta0):
    """p_sfc = -trapz(rho0 g theta'/theta0, z), mean removed —
    storm_tracker.py:64-73."""
    b = GRAVITY * theta_prime / theta0[None, None, :]
    integrand = rho0[None, None, :] * b
    trap = getattr(np, "trapezoid", None) or np.trapz
    p = -trap(integrand, z, axis=2)
    return p - np.mean(p)


def gaussian_weight(p, nx, ny, dx, last_pos, r0=R0_CELLS):
    """storm_tracker.py:76-98."""
    if last_pos is None:
        return p
    ixl = last_pos[0] / dx
    iyl = last_pos[1] / dx
    ix = np.arange(nx, dtype=float).reshape(-1, 1)
    iy = np.arange(ny, dtype=float).reshape(1, -1)
    r2 = (ix - ixl) ** 2 + (iy - iyl) ** 2
    return p * np.exp(-r2 / (2.0 * r0 ** 2))


def smooth3(f):
    """storm_tracker.py:102-112."""
    f = (np.roll(f, 1, axis=0) + 2.0 * f + np.roll(f, -1, axis=0)) * 0.25
    f = (np.roll(f, 1, axis=1) + 2.0 * f + np.roll(f, -1, axis=1)) * 0.25
    return f


def vorticity_centre(u, v, nx, ny, dx, last_pos=None, r0=R0_CELLS):
    """storm_tracker.py:115-188."""
    nzh = u.shape[2] // 2
    ul = u[:, :, :nzh]; vl = v[:, :, :nzh]
    dvdx = (np.roll(vl, -1, axis=0) - np.roll(vl, 1, axis=0)) / (2.0 * dx)
    dudy = (np.roll(ul, -1, axis=1) - np.roll(ul, 1, axis=1)) / (2.0 * dx)
    zeta = dvdx - dudy
    zcol = np.mean(np.maximum(zeta, 0.0), axis=2)
    ix = np.arange(nx, dtype=np.float64)[:, None]
    iy = np.arange(ny, dtype=np.float64)[None, :]
    if last_pos is None:
        total = float(np.sum(zcol))
        if total < 1e-14:
            return nx * dx / 2.0, ny * dx / 2.0
        xc = float(np.sum(ix * zcol) / total) * dx + 0.5 * dx
        yc = float(np.sum(iy * zcol) / total) * dx + 0.5 * dx
        return xc, yc
    r2 = (ix - last_pos[0] / dx) ** 2 + (iy - last_pos[1] / dx) ** 2
    zw = smooth3(zcol) * np.exp(-r2 / (2.0 * r0 ** 2))
    if float(np.max(zw)) < 1e-14:
        return last_pos[0], last_pos[1]
    idx = int(np.argmax(zw))
    ix0, iy0 = divmod(idx, ny)
    w = 2
    i0, i1 = max(0, ix0 - w), min(nx, ix0 + w + 1)
    j0, j1 = max(0, iy0 - w), min(ny, iy0 + w + 1)
    patch = np.maximum(zw[i0:i1, j0:j1], 0.0)
    ptot = float(np.sum(patch))
    if ptot < 1e-14:
        xcc, ycc = float(ix0), float(iy0)
    else:
        ii = np.arange(i0, i1, dtype=np.float64)[:, None]
        jj = np.arange(j0, j1, dtype=np.float64)[None, :]
        xcc = float(np.sum(ii * patch) / ptot)
        ycc = float(np.sum(jj * patch) / ptot)
    return (xcc + 0.5) * dx, (ycc + 0.5) * dx


def masked_argmin(p, nx, ny, margin):
    """storm_tracker.py:191-203."""
    q = p.copy()
    q[:margin, :] = q.max()
    q[-margin:, :] = q.max()
    q[:, :margin] = q.max()
    q[:, -margin:] = q.max()
    idx = int(np.argmin(q))
    return divmod(idx, ny)


def parabolic_refine(p, ix, iy):
    """storm_tracker.py:206-227."""
    nx_, ny_ = p.shape

    def off(a, b, c):
        d = a - 2.0 * b + c
        if abs(d) < 1e-30:
            return 0.0
        return float(np.clip(0.5 * (a - c) / d, -0.5, 0.5))

    ox = off(p[ix - 1, iy], p[ix, iy], p[ix + 1, iy]) if 0 < ix < nx_ - 1 else 0.0
    oy = off(p[ix, iy - 1], p[ix, iy], p[ix, iy + 1]) if 0 < iy < ny_ - 1 else 0.0
    return ix + ox, iy + oy


def find_storm_centre(st: State, z, rho0, theta0, nx, ny, dx, last_pos=None,
                      max_jump_cells=5, interior_margin=0.12, v_env_ms=0.0,
                      u_env_ms=0.0, dt_output_s=1800.0, last_raw_pos=None,
                      reacq_jump_cells=None, subcell=True):
    """Returns ((x, y), method, theta_raw_m) — storm_tracker.py:232-394."""
    margin = max(int(interior_margin * nx), 3)
    p = theta_prime_proxy(st.theta_prime, z, rho0, theta0)
    ixr, iyr = masked_argmin(p, nx, ny, margin)
    fxr, fyr = parabolic_refine(p, ixr, iyr) if subcell else (float(ixr), float(iyr))
    raw = ((fxr + 0.5) * dx, (fyr + 0.5) * dx)
    p = gaussian_weight(p, nx, ny, dx, last_pos)
    ix, iy = masked_argmin(p, nx, ny, margin)
    fx, fy = parabolic_refine(p, ix, iy) if subcell else (float(ix), float(iy))
    x_new = (fx + 0.5) * dx
    y_new = (fy + 0.5) * dx
    method = "theta_prime"
    if last_pos is not None:
        lix = last_pos[0] / dx
        liy = last_pos[1] / dx
        dist = np.sqrt((ix - lix) ** 2 + (iy - liy) ** 2)
        if dist > max_jump_cells:
            reacq = reacq_jump_cells if reacq_jump_cells is not None else max_jump_cells
            done = False
            if last_raw_pos is not None:
                rj = np.sqrt((ixr - last_raw_pos[0] / dx) ** 2 + (iyr - last_raw_pos[1] / dx) ** 2)
                if rj <= reacq:
                    x_new, y_new = raw
                    method = "theta_reacq"
                    done = True
            if not done:
                x_new, y_new = vorticity_centre(st.u, st.v, nx, ny, dx, last_pos=last_pos)
                method = "vorticity"
                vd = np.sqrt((x_new / dx - lix) ** 2 + (y_new / dx - liy) ** 2)
                if vd > max_jump_cells * 2:
                    if v_env_ms != 0.0 or u_env_ms != 0.0:
                        x_new = last_pos[0] + u_env_ms * dt_output_s
                        y_new = last_pos[1] + v_env_ms * dt_output_s
                    else:
                        x_new, y_new = last_pos[0], last_pos[1]
                    method = "extrapolated"
    return (x_new, y_new), method, raw
