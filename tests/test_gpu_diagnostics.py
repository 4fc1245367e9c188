"""Vortex diagnostics read-outs on the GPU against the reference's outputs.

Every recorded call of oracle_v8/diagnostics.py and of the sub-cell refinement
of run_translation_test.py (tests/golden/diagnostics.npz) is replayed through
``oraclev8_b200.diagnostics`` on device fields:
* vorticity_center, low_level_vmax and vmax_3d are argmax reductions over
  values formed in the reference's operation order: equal bit for bit;
* the ring, kinetic-energy, enstrophy and centroid sums are device trees:
  within 1e-12 of the reference, relative;
* FP32 fields: the same calls against the oracle on the FP32 values widened
  to double (the device computes in double), with the same bars.
"""
import types
import warnings

import numpy as np
import pytest
import torch

from oracle import vortex_diag as VD
from tests.diag_cases import diag_states, replay, same
from tests.gpu_helpers import dev

pytestmark = pytest.mark.gpu

EXACT = {"vorticity_center", "low_level_vmax", "vmax_3d"}
EXACT_KEYS = {"xv_m", "yv_m", "vmax_lowlvl", "r_vmax_km", "z_vmax_m", "vmax_3d", "z_vmax3d_m",
              "sep_km"}
RTOL = 1e-12


class _Device:
    """The device module in the oracle's keyword form (u, v, z arrays)."""

    def __init__(self, dtype):
        self.dtype = dtype

    def _st(self, u, v):
        return types.SimpleNamespace(u=dev(u, self.dtype), v=dev(v, self.dtype))

    @staticmethod
    def _base(z):
        return None if z is None else types.SimpleNamespace(z=z)

    def compute_diagnostics(self, u, v, z, cx, cy, dx, dy, ue, ve, theta_xy_m=None,
                            r_vent_m=120e3):
        from oraclev8_b200 import diagnostics as D
        return D.compute_diagnostics(self._st(u, v), self._base(z), cx, cy, dx, dy, ue, ve,
                                     theta_xy_m=theta_xy_m, r_vent_m=r_vent_m)

    def format_diag_line(self, d):
        from oraclev8_b200 import diagnostics as D
        return D.format_diag_line(d)

    def vorticity_center(self, u, v, cx, cy, dx, dy, z=None, window_m=200e3, z_top_m=3000.0):
        from oraclev8_b200 import diagnostics as D
        return D.vorticity_center(self._st(u, v), cx, cy, dx, dy, base=self._base(z),
                                  window_m=window_m, z_top_m=z_top_m)

    def low_level_vmax(self, u, v, z, cx, cy, dx, dy, ue, ve, z_top_m=3000.0):
        from oraclev8_b200 import diagnostics as D
        return D.low_level_vmax(self._st(u, v), self._base(z), cx, cy, dx, dy, ue, ve,
                                z_top_m=z_top_m)

    def vmax_3d(self, u, v, z, ue, ve):
        from oraclev8_b200 import diagnostics as D
        return D.vmax_3d(self._st(u, v), self._base(z), ue, ve)

    def ventilation_flow(self, u, v, cx, cy, dx, dy, z=None, **kw):
        from oraclev8_b200 import diagnostics as D
        return D.ventilation_flow(self._st(u, v), cx, cy, dx, dy, base=self._base(z), **kw)

    def perturbation_ke(self, u, v, ue, ve):
        from oraclev8_b200 import diagnostics as D
        return D.perturbation_ke(self._st(u, v), ue, ve)

    def enstrophy(self, u, v, dx, dy, z=None, z_top_m=3000.0):
        from oraclev8_b200 import diagnostics as D
        return D.enstrophy(self._st(u, v), dx, dy, base=self._base(z), z_top_m=z_top_m)

    def subcell_refine(self, u, v, x, y, dx, patch=9):
        from oraclev8_b200 import diagnostics as D
        return D._subcell_refine(self._st(u, v), x, y, dx, patch=patch)


def _check(got, want, fn):
    if fn in EXACT:
        return same(got, want)
    if fn == "compute_diagnostics":
        return (set(got) == set(want)
                and all(same(got[k], want[k], 0.0 if k in EXACT_KEYS else RTOL) for k in want))
    return same(got, want, RTOL)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_diagnostics_match_reference(golden_dir, dtype):
    mod = _Device(dtype)
    n = 0
    for name, (u, v, z, dx, calls) in diag_states(golden_dir).items():
        if dtype == torch.float32:
            u = u.astype(np.float32).astype(np.float64)
            v = v.astype(np.float32).astype(np.float64)
        for c in calls:
            with warnings.catch_warnings():
                warnings.simplefilter("ignore", RuntimeWarning)
                want = c["out"] if dtype == torch.float64 else replay(c, VD, u, v, z, dx)
            got = replay(c, mod, u, v, z, dx)
            assert _check(got, want, c["fn"]), (name, c["fn"], c["kw"], got, want)
            n += 1
    assert n == 78


def test_diagnostics_at_size_against_oracle():
    """A 256 x 192 x 48 state with several vortices and noise (seeded): the
    vorticity centre and the speed maxima equal the oracle's; every sum is
    within 1e-12."""
    rng = np.random.default_rng(91)
    nx, ny, nz, dx = 256, 192, 48, 5e3
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(x, y, indexing="ij")
    u = np.zeros((nx, ny, nz))
    v = np.zeros((nx, ny, nz))
    for (xc, yc, s) in ((0.4, 0.55, 30.0), (0.75, 0.3, -18.0), (0.2, 0.2, 12.0)):
        dxv, dyv = X - xc * nx * dx, Y - yc * ny * dx
        r2 = dxv ** 2 + dyv ** 2
        vt = s * np.exp(-r2 / (2 * (40e3) ** 2))
        r = np.sqrt(r2) + 1.0
        u += (-vt * dyv / r)[:, :, None] * np.linspace(1.0, 0.3, nz)[None, None, :]
        v += (vt * dxv / r)[:, :, None] * np.linspace(1.0, 0.3, nz)[None, None, :]
    u += 0.3 * rng.standard_normal(u.shape)
    v += 0.3 * rng.standard_normal(v.shape)
    z = (np.arange(nz) + 0.5) * (15e3 / nz)
    mod = _Device(torch.float64)
    cx, cy = 0.41 * nx * dx, 0.54 * ny * dx
    want = VD.compute_diagnostics(u, v, z, cx, cy, dx, dx, 1.0, -0.5, theta_xy_m=(cx, cy))
    got = mod.compute_diagnostics(u, v, z, cx, cy, dx, dx, 1.0, -0.5, theta_xy_m=(cx, cy))
    assert _check(got, want, "compute_diagnostics"), (got, want)
    assert same(mod.subcell_refine(u, v, got["xv_m"], got["yv_m"], dx),
                VD.subcell_refine(u, v, got["xv_m"], got["yv_m"], dx), RTOL)

