"""Vortex diagnostics read-outs on the B200 backend: the counterpart of
oracle_v8/diagnostics.py (same function names, arguments and returned keys)
and of the sub-cell centre refinement in oracle_v8/run_translation_test.py
(``subcell_refine``, also exported as ``_subcell_refine``).

The field work runs on the GPU through the C ABI (``oracle_b200_vdiag_*``):
- the level-band column means, in NumPy's summation order for a
  boolean-indexed band;
- the periodic centred vorticity;
- the windowed and banded argmax reductions, in numpy.argmax's order;
- the kinetic-energy, enstrophy and ring sums;
- the refinement's positive-vorticity field with its smoothing, and the
  patch sums of each centroid iteration.

The host keeps the reference's scalar logic and its Python slice rules.
State fields are CUDA tensors (float64 or float32; arithmetic in double).
There is no CPU path: host arrays raise TypeError.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib as L

_WORK: "dict[tuple, _Workspace]" = {}
_WORK_MAX = 8


class _Workspace:
    """Device scratch of the reductions for one grid."""

    def __init__(self, nx, ny, nz):
        self.lib = L.load()
        self.nx, self.ny, self.nz = nx, ny, nz
        h = ctypes.c_void_p()
        L.check(self.lib.oracle_b200_vdiag_create(nx, ny, nz, ctypes.byref(h)))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.oracle_b200_vdiag_destroy(h)
            except Exception:
                pass
            self.handle = None


def _fields(state):
    u, v = state.u, state.v
    for t in (u, v):
        if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
            raise TypeError("the diagnostics read device fields (CUDA torch tensors); "
                            "the B200 backend has no CPU fallback")
    if u.dim() != 3 or tuple(v.shape) != tuple(u.shape):
        raise ValueError("u and v must be (nx, ny, nz) fields of one shape")
    if u.dtype != v.dtype or u.dtype not in (torch.float64, torch.float32):
        raise ValueError("u and v must share a float64 or float32 dtype")
    prec = L.OB_PREC_F64 if u.dtype == torch.float64 else L.OB_PREC_F32
    return u.contiguous(), v.contiguous(), prec


def _workspace(u) -> _Workspace:
    nx, ny, nz = (int(s) for s in u.shape)
    key = (u.device.index, nx, ny, nz)
    w = _WORK.get(key)
    if w is None:
        if len(_WORK) >= _WORK_MAX:
            _WORK.pop(next(iter(_WORK)))
        w = _WORK[key] = _Workspace(nx, ny, nz)
    return w


def _stream(u):
    return ctypes.c_void_p(torch.cuda.current_stream(u.device).cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _base_z(base):
    z = getattr(base, "z", None) if base is not None else None
    if z is None:
        return None
    if isinstance(z, torch.Tensor):
        z = z.detach().cpu().numpy()
    return np.asarray(z)


def _band(nz, z, z_lo_m, z_hi_m):
    """diagnostics.py:53-59: the levels with z in [z_lo, z_hi] (all levels
    without a z), as ascending indices."""
    if z is None:
        return np.ones(nz, dtype=bool)
    zz = z[:nz]
    return (zz >= z_lo_m) & (zz <= z_hi_m)


def _levels(mask):
    idx = np.flatnonzero(mask).astype(np.int32)
    return idx, idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(idx)


def _centres(i, d):
    return (i + 0.5) * d


# ---------------------------------------------------------------------------
# intensity
# ---------------------------------------------------------------------------

def _speed_max(state, mask, u_env, v_env):
    u, v, prec = _fields(state)
    w = _workspace(u)
    keep, lev, n = _levels(mask)
    out = L.VdMax()
    L.check(w.lib.oracle_b200_vdiag_speed_max(w.handle, _ptr(u), _ptr(v), prec, lev, n,
                                              float(u_env), float(v_env), ctypes.byref(out),
                                              _stream(u)))
    return out.value, int(out.index)


def low_level_vmax(state, base, cx_m, cy_m, dx, dy, u_env=0.0, v_env=0.0, z_top_m=3000.0):
    """Max perturbation |V'| in the lowest z_top_m with its radius (km) from
    (cx_m, cy_m) and its height (diagnostics.py:65-98)."""
    nx, ny, nz = (int(s) for s in state.u.shape)
    z = _base_z(base)
    band = _band(nz, z, 0.0, z_top_m)
    if not band.any():
        band = np.zeros(nz, dtype=bool)
        band[0] = True
    vmax, flat = _speed_max(state, band, u_env, v_env)
    iz = flat % nz
    iy = (flat // nz) % ny
    ix = flat // (nz * ny)
    # the distance as np.sqrt((x - cx)**2 + (y - cy)**2) forms it (NumPy
    # squares by multiplying)
    a, b = _centres(ix, dx) - cx_m, _centres(iy, dy) - cy_m
    r = math.sqrt(a * a + b * b)
    return {"vmax_lowlvl": vmax, "r_vmax_km": float(r) / 1e3,
            "z_vmax_m": float(z[iz]) if z is not None else float(iz)}


def vmax_3d(state, base, u_env=0.0, v_env=0.0):
    """Max perturbation |V'| anywhere with its height (diagnostics.py:101-112)."""
    nz = int(state.u.shape[2])
    vmax, flat = _speed_max(state, np.ones(nz, dtype=bool), u_env, v_env)
    z = _base_z(base)
    iz = flat % nz
    return {"vmax_3d": vmax, "z_vmax3d_m": float(z[iz]) if z is not None else float(iz)}


# ---------------------------------------------------------------------------
# ventilation flow
# ---------------------------------------------------------------------------

def ventilation_flow(state, cx_m, cy_m, dx, dy, base=None, r_vent_m=150e3, z_lo_m=0.0,
                     z_hi_m=12000.0, u_env=None, v_env=None, n_bins=12):
    """Azimuthal mean of the deep-layer Cartesian wind over rings out to
    r_vent_m, rings averaged; the disk mean when no ring holds a cell
    (diagnostics.py:118-166)."""
    u, v, prec = _fields(state)
    nz = int(u.shape[2])
    band = _band(nz, _base_z(base), z_lo_m, z_hi_m) if base is not None \
        else np.ones(nz, dtype=bool)
    if not band.any():
        band = np.ones(nz, dtype=bool)
    n_bins = int(n_bins)
    edges = np.ascontiguousarray(np.linspace(0.0, r_vent_m, n_bins + 1), dtype=np.float64)
    w = _workspace(u)
    keep, lev, n = _levels(band)
    sums = np.zeros(3 * (n_bins + 1))
    L.check(w.lib.oracle_b200_vdiag_rings(
        w.handle, _ptr(u), _ptr(v), prec, lev, n, float(dx), float(dy), float(cx_m),
        float(cy_m), L.dptr(edges), n_bins, float(r_vent_m), L.dptr(sums), _stream(u)))
    sums = sums.reshape(n_bins + 1, 3)
    rings = [(su / c, sv / c) for c, su, sv in sums[:n_bins] if c > 0]
    if rings:
        u_vent = float(np.mean(np.array([r[0] for r in rings])))
        v_vent = float(np.mean(np.array([r[1] for r in rings])))
    else:
        c, su, sv = sums[n_bins]
        u_vent = su / c if c > 0 else float("nan")
        v_vent = sv / c if c > 0 else float("nan")
    out = {"u_vent": float(u_vent), "v_vent": float(v_vent)}
    if u_env is not None and v_env is not None:
        out["u_gyre"] = out["u_vent"] - float(u_env)
        out["v_gyre"] = out["v_vent"] - float(v_env)
    return out


# ---------------------------------------------------------------------------
# vorticity centre, budgets
# ---------------------------------------------------------------------------

def _vorticity(state, base, dx, dy, cx_m, cy_m, window_m, z_top_m):
    u, v, prec = _fields(state)
    nz = int(u.shape[2])
    band = _band(nz, _base_z(base), 0.0, z_top_m) if base is not None \
        else np.ones(nz, dtype=bool)
    if not band.any():
        # NumPy's mean over no level is NaN everywhere, so argmax returns the
        # first cell inside the window (cell 0 when none is), and the
        # enstrophy is NaN
        nx, ny = int(u.shape[0]), int(u.shape[1])
        a = (np.arange(nx) + 0.5) * dx - cx_m
        b = (np.arange(ny) + 0.5) * dy - cy_m
        inside = np.flatnonzero(np.sqrt((a * a)[:, None] + (b * b)[None, :]) < window_m)
        return (int(inside[0]) if inside.size else 0), float("nan")
    w = _workspace(u)
    keep, lev, n = _levels(band)
    best, sq = L.VdMax(), ctypes.c_double()
    L.check(w.lib.oracle_b200_vdiag_vorticity(
        w.handle, _ptr(u), _ptr(v), prec, lev, n, float(dx), float(dy), float(cx_m),
        float(cy_m), float(window_m), ctypes.byref(best), ctypes.byref(sq), _stream(u)))
    return int(best.index), sq.value


def vorticity_center(state, cx_m, cy_m, dx, dy, base=None, window_m=200e3, z_top_m=3000.0):
    """Low-level relative-vorticity maximum inside r < window_m about
    (cx_m, cy_m) (diagnostics.py:172-191)."""
    ny = int(state.u.shape[1])
    flat, _ = _vorticity(state, base, dx, dy, cx_m, cy_m, window_m, z_top_m)
    ix, iy = divmod(flat, ny)
    return {"xv_m": float(_centres(ix, dx)), "yv_m": float(_centres(iy, dy))}


def center_separation_km(theta_xy_m, vort_xy_m):
    """Distance (km) between the theta' and vorticity centres (diagnostics.py:194-198)."""
    a = theta_xy_m[0] - vort_xy_m[0]
    b = theta_xy_m[1] - vort_xy_m[1]
    return float((a ** 2 + b ** 2) ** 0.5) / 1e3


def perturbation_ke(state, u_env=0.0, v_env=0.0):
    """0.5 <(u')^2 + (v')^2> (diagnostics.py:203-207)."""
    u, v, prec = _fields(state)
    w = _workspace(u)
    s = ctypes.c_double()
    L.check(w.lib.oracle_b200_vdiag_ke(w.handle, _ptr(u), _ptr(v), prec, float(u_env),
                                       float(v_env), ctypes.byref(s), _stream(u)))
    return {"pert_ke": float(0.5 * (s.value / u.numel()))}


def enstrophy(state, dx, dy, base=None, z_top_m=3000.0):
    """0.5 <zeta^2> of the low-level wind (diagnostics.py:210-220)."""
    nx, ny = int(state.u.shape[0]), int(state.u.shape[1])
    _, sq = _vorticity(state, base, dx, dy, 0.0, 0.0, 0.0, z_top_m)
    return {"enstrophy": float(0.5 * (sq / (nx * ny)))}


def compute_diagnostics(state, base, cx_m, cy_m, dx, dy, u_env=0.0, v_env=0.0,
                        theta_xy_m=None, r_vent_m=120e3):
    """All read-outs, anchored on the vorticity centre (diagnostics.py:226-254)."""
    d = {}
    vc = vorticity_center(state, cx_m, cy_m, dx, dy, base=base)
    d.update(vc)
    cxv, cyv = vc["xv_m"], vc["yv_m"]
    d.update(low_level_vmax(state, base, cxv, cyv, dx, dy, u_env, v_env))
    d.update(vmax_3d(state, base, u_env, v_env))
    d.update(ventilation_flow(state, cxv, cyv, dx, dy, base=base, r_vent_m=r_vent_m,
                              u_env=u_env, v_env=v_env))
    if theta_xy_m is not None:
        d["sep_km"] = center_separation_km(theta_xy_m, (cxv, cyv))
    d.update(perturbation_ke(state, u_env, v_env))
    d.update(enstrophy(state, dx, dy, base=base))
    return d


def format_diag_line(d):
    """The compact one-line log (diagnostics.py:257-270)."""
    s = (f"Vmax'={d['vmax_lowlvl']:5.1f}@{d['r_vmax_km']:4.0f}km/"
         f"{d['z_vmax_m'] / 1e3:3.1f}km  vent=[{d['u_vent']:+.2f},{d['v_vent']:+.2f}]")
    if "v_gyre" in d:
        s += f" gyre=[{d['u_gyre']:+.2f},{d['v_gyre']:+.2f}]"
    if "sep_km" in d:
        s += f"  sep={d['sep_km']:4.0f}km"
    s += f"  KE={d['pert_ke']:.0f}"
    return s


# ---------------------------------------------------------------------------
# sub-cell centre refinement (run_translation_test.py:115-161)
# ---------------------------------------------------------------------------

def subcell_refine(state, x_m, y_m, dx, patch=9):
    """Replace a cell-resolution centre by the zeta^2-weighted centroid of the
    smoothed positive low-level vorticity over a (2 patch + 1)^2 patch, two
    iterations, each recentred on the last; the seed comes back for a
    non-finite seed or an empty or zero patch."""
    u, v, prec = _fields(state)
    nx, ny, nz = (int(s) for s in u.shape)
    w = _workspace(u)
    L.check(w.lib.oracle_b200_vdiag_zpos(w.handle, _ptr(u), _ptr(v), prec, float(dx),
                                         _stream(u)))
    xc, yc = x_m / dx - 0.5, y_m / dx - 0.5
    if not (np.isfinite(xc) and np.isfinite(yc)):
        return x_m, y_m
    out = np.zeros(3)
    for _ in range(2):
        i0, j0 = int(round(xc)), int(round(yc))
        sx = slice(max(i0 - patch, 0), min(i0 + patch + 1, nx))
        sy = slice(max(j0 - patch, 0), min(j0 + patch + 1, ny))
        rx, ry = range(nx)[sx], range(ny)[sy]  # the rows NumPy's slice selects
        if len(rx) and len(ry):
            L.check(w.lib.oracle_b200_vdiag_centroid(w.handle, rx.start, rx.stop, ry.start,
                                                     ry.stop, L.dptr(out), _stream(u)))
            tot = float(out[0])
        else:
            tot = 0.0
        if not np.isfinite(tot) or tot < 1e-20:
            return x_m, y_m
        # the index vectors are np.arange(start, stop) of the raw slices; a
        # length that differs from the selected rows fails to broadcast
        if len(range(sx.start, sx.stop)) != len(rx) or len(range(sy.start, sy.stop)) != len(ry):
            raise ValueError("operands could not be broadcast together (patch slice wrapped)")
        xc = float(out[1] / tot)
        yc = float(out[2] / tot)
    return (xc + 0.5) * dx, (yc + 0.5) * dx


_subcell_refine = subcell_refine
