"""Storm-centre tracker on the B200 backend: the counterpart of
oracle_v8/storm_tracker.py (``find_storm_centre``, storm_tracker.py:232-394).

The field work runs on the GPU through the C ABI (``oracle_b200_track_theta``,
``oracle_b200_track_vorticity``):
- the theta' surface-pressure proxy, a warp-per-column trapezoid integral;
- its domain mean;
- the Gaussian window;
- the masked argmin reductions;
- the positive-vorticity column means.

Only a few scalars come back: the argmin cells with their 5-point
neighbourhoods, or, on the rare vorticity fall-back, one (nx, ny) plane.
The decision logic stays on the host, as in the reference: parabolic
sub-cell refine, continuity gate, raw re-acquisition, vorticity fall-back
and dead reckoning.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib as L
from .backend import to_numpy

R0_CELLS = 10.0  # Gaussian window radius in cells (storm_tracker.py:59)

_TRACKERS: "dict[tuple, _Tracker]" = {}
_TRACKERS_MAX = 8


class _Tracker:
    """Device profiles and reduction scratch for one grid and base state."""

    def __init__(self, nx, ny, nz, z, rho0, theta0):
        self.lib = L.load()
        self.nx, self.ny, self.nz = nx, ny, nz
        keep = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in (z, rho0, theta0)]
        for a in keep:
            if a.shape != (nz,):
                raise ValueError(f"base-state profiles must have shape ({nz},), got {a.shape}")
        h = ctypes.c_void_p()
        L.check(self.lib.oracle_b200_tracker_create(nx, ny, nz, *(L.dptr(a) for a in keep),
                                                    ctypes.byref(h)))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.oracle_b200_tracker_destroy(h)
            except Exception:
                pass
            self.handle = None

    def _field(self, t, shape):
        if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
            raise TypeError("the tracker reads device fields (CUDA torch tensors); "
                            "the B200 backend has no CPU fallback")
        if tuple(t.shape) != shape:
            raise ValueError(f"field shape {tuple(t.shape)} does not match the grid {shape}")
        if t.dtype == torch.float64:
            prec = L.OB_PREC_F64
        elif t.dtype == torch.float32:
            prec = L.OB_PREC_F32
        else:
            raise ValueError(f"unsupported dtype {t.dtype}")
        t = t.contiguous()
        return t, prec

    def _stream(self, t):
        return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)

    def theta_fix(self, theta_prime, margin, last_cells=None, r0=R0_CELLS) -> L.TrackFix:
        th, prec = self._field(theta_prime, (self.nx, self.ny, self.nz))
        fix = L.TrackFix()
        lx, ly = last_cells if last_cells is not None else (0.0, 0.0)
        L.check(self.lib.oracle_b200_track_theta(
            self.handle, ctypes.c_void_p(th.data_ptr()), prec, int(margin),
            int(last_cells is not None), float(lx), float(ly), float(r0), ctypes.byref(fix),
            self._stream(th)))
        if not math.isfinite(fix.mean):
            raise RuntimeError("non-finite theta' field: no storm centre can be located")
        return fix

    def vorticity_column(self, u, v, dx) -> np.ndarray:
        shape = (self.nx, self.ny, self.nz)
        u, prec = self._field(u, shape)
        v, prec_v = self._field(v, shape)
        if prec != prec_v:
            raise ValueError("u and v must have the same dtype")
        out = np.empty((self.nx, self.ny), dtype=np.float64)
        L.check(self.lib.oracle_b200_track_vorticity(
            self.handle, ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(v.data_ptr()), prec,
            float(dx), L.dptr(out), self._stream(u)))
        return out


def _tracker_for(nx, ny, nz, base_w) -> _Tracker:
    prof = [np.asarray(to_numpy(getattr(base_w, k)), dtype=np.float64)
            for k in ("z", "rho0", "theta0")]
    key = (nx, ny, nz) + tuple(a.tobytes() for a in prof)
    t = _TRACKERS.get(key)
    if t is None:
        if len(_TRACKERS) >= _TRACKERS_MAX:
            _TRACKERS.pop(next(iter(_TRACKERS)))
        t = _Tracker(nx, ny, nz, *prof)
        _TRACKERS[key] = t
    return t


def _parabolic_offset(a, b, c):
    """Vertex of the parabola through (-1, a), (0, b), (1, c), clipped to half
    a cell (storm_tracker.py:217-222)."""
    d = a - 2.0 * b + c
    if abs(d) < 1e-30:
        return 0.0
    return float(np.clip(0.5 * (a - c) / d, -0.5, 0.5))


def _refine(nb, ix, iy, nx, ny):
    """Sub-cell position from the 5-point neighbourhood nb = f(ix, iy),
    f(ix-1, iy), f(ix+1, iy), f(ix, iy-1), f(ix, iy+1) (storm_tracker.py:206-227)."""
    ox = _parabolic_offset(nb[1], nb[0], nb[2]) if 0 < ix < nx - 1 else 0.0
    oy = _parabolic_offset(nb[3], nb[0], nb[4]) if 0 < iy < ny - 1 else 0.0
    return ix + ox, iy + oy


def _smooth3(f):
    """1-2-1 smoothing along x then y, periodic (storm_tracker.py:102-112)."""
    f = (np.roll(f, 1, axis=0) + 2.0 * f + np.roll(f, -1, axis=0)) * 0.25
    return (np.roll(f, 1, axis=1) + 2.0 * f + np.roll(f, -1, axis=1)) * 0.25


def _vorticity_centre(zcol, nx, ny, dx, last_pos, r0=R0_CELLS):
    """Host part of the vorticity fall-back (storm_tracker.py:141-188) on the
    device-computed column means ``zcol``: global centre of mass on a first
    call; otherwise the arg-max of the smoothed, windowed field refined by the
    centre of mass of its 5 x 5 patch."""
    ix = np.arange(nx, dtype=np.float64)[:, None]
    iy = np.arange(ny, dtype=np.float64)[None, :]
    if last_pos is None:
        total = float(np.sum(zcol))
        if total < 1e-14:
            return nx * dx / 2.0, ny * dx / 2.0
        return (float(np.sum(ix * zcol) / total) * dx + 0.5 * dx,
                float(np.sum(iy * zcol) / total) * dx + 0.5 * dx)
    r2 = (ix - last_pos[0] / dx) ** 2 + (iy - last_pos[1] / dx) ** 2
    zw = _smooth3(zcol) * np.exp(-r2 / (2.0 * r0 ** 2))
    if float(np.max(zw)) < 1e-14:
        return last_pos[0], last_pos[1]
    i, j = divmod(int(np.argmax(zw)), ny)
    i0, i1 = max(0, i - 2), min(nx, i + 3)
    j0, j1 = max(0, j - 2), min(ny, j + 3)
    patch = np.maximum(zw[i0:i1, j0:j1], 0.0)
    ptot = float(np.sum(patch))
    if ptot < 1e-14:
        xc, yc = float(i), float(j)
    else:
        xc = float(np.sum(np.arange(i0, i1, dtype=np.float64)[:, None] * patch) / ptot)
        yc = float(np.sum(np.arange(j0, j1, dtype=np.float64)[None, :] * patch) / ptot)
    return (xc + 0.5) * dx, (yc + 0.5) * dx


def find_storm_centre(state, base_w, nx, ny, dx, last_pos=None, max_jump_cells=5,
                      interior_margin=0.12, v_env_ms=0.0, u_env_ms=0.0, dt_output_s=1800.0,
                      return_diag=False, last_raw_pos=None, reacq_jump_cells=None,
                      subcell=True):
    """Storm centre (x_m, y_m) from the SW corner, and the method that gave it
    ('theta_prime' | 'theta_reacq' | 'vorticity' | 'extrapolated'); with
    ``return_diag`` also {'theta_raw_m': raw unwindowed theta' centre}.
    Same arguments and results as storm_tracker.py:232-394."""
    nz = int(state.theta_prime.shape[2])
    tr = _tracker_for(nx, ny, nz, base_w)
    margin = max(int(interior_margin * nx), 3)
    last_cells = None if last_pos is None else (last_pos[0] / dx, last_pos[1] / dx)
    fix = tr.theta_fix(state.theta_prime, margin, last_cells)

    # raw (unwindowed) fix: a diagnostic that also drives re-acquisition
    ixr, iyr = divmod(int(fix.raw_idx), ny)
    fxr, fyr = _refine(fix.raw_nb, ixr, iyr, nx, ny) if subcell else (float(ixr), float(iyr))
    theta_raw_m = ((fxr + 0.5) * dx, (fyr + 0.5) * dx)

    ix, iy = divmod(int(fix.win_idx), ny)
    fx, fy = _refine(fix.win_nb, ix, iy, nx, ny) if subcell else (float(ix), float(iy))
    x_new, y_new = (fx + 0.5) * dx, (fy + 0.5) * dx
    method = "theta_prime"

    if last_pos is not None:
        lix, liy = last_cells
        if np.sqrt((ix - lix) ** 2 + (iy - liy) ** 2) > max_jump_cells:
            reacq = max_jump_cells if reacq_jump_cells is None else reacq_jump_cells
            if last_raw_pos is not None and np.sqrt(
                    (ixr - last_raw_pos[0] / dx) ** 2 + (iyr - last_raw_pos[1] / dx) ** 2) <= reacq:
                (x_new, y_new), method = theta_raw_m, "theta_reacq"
            else:
                zcol = tr.vorticity_column(state.u, state.v, dx)
                x_new, y_new = _vorticity_centre(zcol, nx, ny, dx, last_pos)
                method = "vorticity"
                if np.sqrt((x_new / dx - lix) ** 2 + (y_new / dx - liy) ** 2) > 2 * max_jump_cells:
                    if v_env_ms != 0.0 or u_env_ms != 0.0:
                        x_new = last_pos[0] + u_env_ms * dt_output_s
                        y_new = last_pos[1] + v_env_ms * dt_output_s
                    else:
                        x_new, y_new = last_pos[0], last_pos[1]
                    method = "extrapolated"
    if return_diag:
        return (x_new, y_new), method, {"theta_raw_m": theta_raw_m}
    return (x_new, y_new), method
