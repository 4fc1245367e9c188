"""CPU restatement of the vortex diagnostics read-outs (test infrastructure).

Follows oracle_v8/diagnostics.py:40-260 (intensity, ventilation flow,
vorticity centre, budgets, the one-call wrapper and its log line) and the
sub-cell centre refinement of oracle_v8/run_translation_test.py:115-161, in
NumPy on host arrays, with the reference's array operations so that the
results agree bit for bit with the reference's NumPy path.  Only the tests,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` use it; the
product never imports it.

Pinned against ``tests/golden/diagnostics.npz`` (outputs of the unmodified
reference, made by ``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import numpy as np


def _cell_centres(nx, ny, dx, dy):
    """diagnostics.py:40-44: x as (nx, 1), y as (1, ny)."""
    return ((np.arange(nx) + 0.5) * dx)[:, None], ((np.arange(ny) + 0.5) * dy)[None, :]


def radius(nx, ny, dx, dy, cx_m, cy_m):
    """diagnostics.py:47-50 (no periodic wrap)."""
    x, y = _cell_centres(nx, ny, dx, dy)
    return np.sqrt((x - cx_m) ** 2 + (y - cy_m) ** 2)


def level_band(nz, z, z_lo_m, z_hi_m):
    """diagnostics.py:53-59: levels with z in [z_lo, z_hi]; all levels when
    the base state has no z."""
    if z is None:
        return np.ones(nz, dtype=bool)
    zz = np.asarray(z)[:nz]
    return (zz >= z_lo_m) & (zz <= z_hi_m)


def _low_level_winds(u, v, band):
    return np.mean(u[:, :, band], axis=2), np.mean(v[:, :, band], axis=2)


def _zeta(u_ll, v_ll, dx, dy):
    """Centred periodic relative vorticity of a 2-D wind (diagnostics.py:176-178)."""
    dvdx = (np.roll(v_ll, -1, axis=0) - np.roll(v_ll, 1, axis=0)) / (2 * dx)
    dudy = (np.roll(u_ll, -1, axis=1) - np.roll(u_ll, 1, axis=1)) / (2 * dy)
    return dvdx - dudy


def low_level_vmax(u, v, z, cx_m, cy_m, dx, dy, u_env=0.0, v_env=0.0, z_top_m=3000.0):
    """diagnostics.py:65-98."""
    nx, ny, nz = u.shape
    spd = np.sqrt((u - u_env) ** 2 + (v - v_env) ** 2)
    band = level_band(nz, z, 0.0, z_top_m)
    if not band.any():
        band = np.zeros(nz, dtype=bool)
        band[0] = True
    masked = np.where(band[None, None, :], spd, -1.0)
    flat = int(np.argmax(masked))
    ix, rem = divmod(flat, ny * nz)
    iy, iz = divmod(rem, nz)
    r = radius(nx, ny, dx, dy, cx_m, cy_m)
    return {"vmax_lowlvl": float(masked[ix, iy, iz]), "r_vmax_km": float(r[ix, iy]) / 1e3,
            "z_vmax_m": float(np.asarray(z)[iz]) if z is not None else float(iz)}


def vmax_3d(u, v, z, u_env=0.0, v_env=0.0):
    """diagnostics.py:101-112."""
    nz = u.shape[2]
    spd = np.sqrt((u - u_env) ** 2 + (v - v_env) ** 2)
    flat = int(np.argmax(spd))
    iz = flat % nz
    return {"vmax_3d": float(spd.reshape(-1)[flat]),
            "z_vmax3d_m": float(np.asarray(z)[iz]) if z is not None else float(iz)}


def ventilation_flow(u, v, cx_m, cy_m, dx, dy, z=None, r_vent_m=150e3, z_lo_m=0.0,
                     z_hi_m=12000.0, u_env=None, v_env=None, n_bins=12):
    """diagnostics.py:118-166: ring-binned azimuthal mean of the deep-layer
    Cartesian wind, rings averaged; a disk mean when no ring holds a cell."""
    nx, ny, nz = u.shape
    band = level_band(nz, z, z_lo_m, z_hi_m)
    if not band.any():
        band = np.ones(nz, dtype=bool)
    u_dl, v_dl = _low_level_winds(u, v, band)
    r = radius(nx, ny, dx, dy, cx_m, cy_m)
    edges = np.linspace(0.0, r_vent_m, n_bins + 1)
    us, vs = [], []
    for lo, hi in zip(edges[:-1], edges[1:]):
        ring = (r >= lo) & (r < hi)
        if ring.any():
            us.append(np.mean(u_dl[ring]))
            vs.append(np.mean(v_dl[ring]))
    if us:
        uv, vv = float(np.mean(np.stack(us))), float(np.mean(np.stack(vs)))
    else:
        disk = r < r_vent_m
        uv, vv = float(np.mean(u_dl[disk])), float(np.mean(v_dl[disk]))
    out = {"u_vent": uv, "v_vent": vv}
    if u_env is not None and v_env is not None:
        out["u_gyre"] = uv - float(u_env)
        out["v_gyre"] = vv - float(v_env)
    return out


def vorticity_center(u, v, cx_m, cy_m, dx, dy, z=None, window_m=200e3, z_top_m=3000.0):
    """diagnostics.py:172-191: argmax of the low-level vorticity inside the
    window (first index; index 0 when the window holds no cell)."""
    nx, ny, nz = u.shape
    band = level_band(nz, z, 0.0, z_top_m)
    zeta = _zeta(*_low_level_winds(u, v, band), dx, dy)
    r = radius(nx, ny, dx, dy, cx_m, cy_m)
    flat = int(np.argmax(np.where(r < window_m, zeta, -np.inf)))
    ix, iy = divmod(flat, ny)
    x, y = _cell_centres(nx, ny, dx, dy)
    return {"xv_m": float(x[ix, 0]), "yv_m": float(y[0, iy])}


def center_separation_km(theta_xy_m, vort_xy_m):
    """diagnostics.py:194-198."""
    a = theta_xy_m[0] - vort_xy_m[0]
    b = theta_xy_m[1] - vort_xy_m[1]
    return float((a ** 2 + b ** 2) ** 0.5) / 1e3


def perturbation_ke(u, v, u_env=0.0, v_env=0.0):
    """diagnostics.py:203-207."""
    return {"pert_ke": float(0.5 * np.mean((u - u_env) ** 2 + (v - v_env) ** 2))}


def enstrophy(u, v, dx, dy, z=None, z_top_m=3000.0):
    """diagnostics.py:210-220."""
    band = level_band(u.shape[2], z, 0.0, z_top_m)
    zeta = _zeta(*_low_level_winds(u, v, band), dx, dy)
    return {"enstrophy": float(0.5 * np.mean(zeta ** 2))}


def compute_diagnostics(u, v, z, cx_m, cy_m, dx, dy, u_env=0.0, v_env=0.0, theta_xy_m=None,
                        r_vent_m=120e3):
    """diagnostics.py:226-254: everything anchored on the vorticity centre."""
    d = dict(vorticity_center(u, v, cx_m, cy_m, dx, dy, z=z))
    cxv, cyv = d["xv_m"], d["yv_m"]
    d.update(low_level_vmax(u, v, z, cxv, cyv, dx, dy, u_env, v_env))
    d.update(vmax_3d(u, v, z, u_env, v_env))
    d.update(ventilation_flow(u, v, cxv, cyv, dx, dy, z=z, r_vent_m=r_vent_m, u_env=u_env,
                              v_env=v_env))
    if theta_xy_m is not None:
        d["sep_km"] = center_separation_km(theta_xy_m, (cxv, cyv))
    d.update(perturbation_ke(u, v, u_env, v_env))
    d.update(enstrophy(u, v, dx, dy, z=z))
    return d


def format_diag_line(d):
    """diagnostics.py:257-270, the compact log line."""
    s = (f"Vmax'={d['vmax_lowlvl']:5.1f}@{d['r_vmax_km']:4.0f}km/"
         f"{d['z_vmax_m'] / 1e3:3.1f}km  vent=[{d['u_vent']:+.2f},{d['v_vent']:+.2f}]")
    if "v_gyre" in d:
        s += f" gyre=[{d['u_gyre']:+.2f},{d['v_gyre']:+.2f}]"
    if "sep_km" in d:
        s += f"  sep={d['sep_km']:4.0f}km"
    s += f"  KE={d['pert_ke']:.0f}"
    return s


def subcell_refine(u, v, x_m, y_m, dx, patch=9):
    """run_translation_test.py:115-161: zeta^2-weighted centroid of the
    smoothed positive low-level vorticity over a (2 patch + 1)^2 patch, two
    iterations; the seed back when it is not finite or the patch is empty."""
    nzh = u.shape[2] // 2
    ulo, vlo = u[:, :, :nzh], v[:, :, :nzh]
    dvdx = (np.roll(vlo, -1, axis=0) - np.roll(vlo, 1, axis=0)) / (2.0 * dx)
    dudy = (np.roll(ulo, -1, axis=1) - np.roll(ulo, 1, axis=1)) / (2.0 * dx)
    zp = np.mean(np.maximum(dvdx - dudy, 0.0), axis=2)
    zp = (np.roll(zp, 1, 0) + 2.0 * zp + np.roll(zp, -1, 0)) * 0.25
    zp = (np.roll(zp, 1, 1) + 2.0 * zp + np.roll(zp, -1, 1)) * 0.25
    nx, ny = zp.shape
    xc, yc = x_m / dx - 0.5, y_m / dx - 0.5
    if not (np.isfinite(xc) and np.isfinite(yc)):
        return x_m, y_m
    for _ in range(2):
        i0, j0 = int(round(xc)), int(round(yc))
        sx = slice(max(i0 - patch, 0), min(i0 + patch + 1, nx))
        sy = slice(max(j0 - patch, 0), min(j0 + patch + 1, ny))
        w = zp[sx, sy] ** 2
        tot = float(np.sum(w))
        if not np.isfinite(tot) or tot < 1e-20:
            return x_m, y_m
        xc = float(np.sum(np.arange(sx.start, sx.stop, dtype=np.float64)[:, None] * w) / tot)
        yc = float(np.sum(np.arange(sy.start, sy.stop, dtype=np.float64)[None, :] * w) / tot)
    return (xc + 0.5) * dx, (yc + 0.5) * dx
