"""Kernel variants and the autotuner.

Each kernel class of the projection has several forms (register-resident
pencils for 512- and 1024-point lines, compile-time-chunk Stockham pencils,
runtime-chunk Stockham pencils) at several z-chunks.  The autotuner times the
forms the grid allows on the plan's own buffers and keeps the fastest, once
per grid, precision, component set and device.

* every form of every class gives the projection (and the FP64-residual
  correction) within the FP32 parity bound of the FP64 projection;
* tuning picks allowed values and a second plan of the same key reuses them;
* values a grid does not allow are refused;
* the choice persists in ORACLE_B200_TUNE_CACHE across processes.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import lh82 as O
from tests.gpu_helpers import dev, host

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _plan(nx, ny, nz, prec, autotune=True, **kw):
    from oraclev8_b200._plan import Plan, PlanSpec
    Lx, Ly, Lz = nx * 5e3, ny * 5e3, 16e3
    z, rho0, th0 = O.build_base_state(nz, Lz)
    return Plan(PlanSpec(nx, ny, nz, Lx, Ly, Lz, rho0, th0, precision=prec, projection=True,
                         autotune=autotune, **kw))


def _smooth(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(nx)[:, None, None]
    ky = np.fft.fftfreq(ny)[None, :, None]
    filt = np.exp(-(kx ** 2 + ky ** 2) / 0.02)

    def field(shape, amp):
        f = np.fft.fft2(rng.standard_normal(shape), axes=(0, 1)) * filt
        return amp * np.real(np.fft.ifft2(f, axes=(0, 1)))
    u, v = field((nx, ny, nz), 30.0), field((nx, ny, nz), 30.0)
    w = field((nx, ny, nz + 1), 0.5)
    w[:, :, 0] = w[:, :, -1] = 0.0
    return [np.asarray(a, dtype=np.float32).astype(np.float64) for a in (u, v, w)]


def _project(plan, fields, dtype, refine=False):
    u, v, w = (dev(a, dtype) for a in fields)
    phi = torch.empty_like(u)
    plan.project(u, v, w, phi)
    if refine:
        plan.refine(u, v, w, phi)
    return [host(a).astype(np.float64) for a in (u, v, w, phi)]


# per class: the variants that select its form
CLASSES = {
    "fx": ("zc4_fx", "zc3_fx", "zc2_fx"),
    "ix": ("zc4_ix", "zc3_ix", "zc2_ix"),
    "fy": ("zc4_fy", "zc3_fy", "zc2_fy"),
    "iy": ("zc4_iy", "zc3_fy", "zc2_iy"),
    "rfx": ("zc4_fxd", "zc3_fxd", "rzc2_fx"),
    "rfy": ("zc3_fyd", "rzc2_fy"),
    "thomas": ("thomas_fast",),
}


@pytest.mark.parametrize("nx, ny, nz", [(512, 512, 16), (1024, 1024, 8), (192, 384, 13)])
def test_every_form_stays_within_the_parity_bound(nx, ny, nz):
    """Each class's forms in turn (the others at the plan's choice): the FP32
    projection (and, for the residual transforms, its correction) against the
    FP64 projection of the same input: u and v within a few FP32 ulp of the
    wind, w and phi within 1e-3 of their own scale."""
    p64 = _plan(nx, ny, nz, "fp64")
    p32 = _plan(nx, ny, nz, "fp32")
    p32.set_refinement(0)
    fields = _smooth(nx, ny, nz, seed=nx + nz)
    r64 = _project(p64, fields, torch.float64)
    wind = max(np.abs(r64[0]).max(), np.abs(r64[1]).max())
    base = p32.variants()
    tried = 0
    for cls, names in CLASSES.items():
        for name in names:
            allowed = _allowed(p32, name)
            for val in allowed:
                if val == 0:
                    continue
                kw = {n: 0 for n in names}
                kw[name] = val
                p32.set_variants(**kw)
                out = _project(p32, fields, torch.float32, refine=cls.startswith("r"))
                for i, f in enumerate(("u", "v", "w", "phi")):
                    scale = np.abs(r64[i]).max()
                    err = np.abs(out[i] - r64[i]).max() / scale
                    assert err <= (1e-5 if f in ("u", "v") else 1e-3), (cls, name, val, f, err)
                for i in (0, 1):
                    assert np.abs(out[i] - r64[i]).max() <= 1e-6 * wind, (cls, name, val)
                tried += 1
                p32.set_variants(**{n: base[n] for n in names})
    assert tried >= 6


def _allowed(plan, name):
    """The values the library accepts for one variant (probed: set, read back)."""
    cur = plan.variants()
    ok = []
    for v in (0, 1, 2, 4, 8):
        try:
            plan.set_variants(**{name: v})
            ok.append(v)
        except ValueError:
            pass
    plan.set_variants(**{name: cur[name]})
    return ok


def test_tuning_reuses_its_choice_and_refuses_bad_values():
    p1 = _plan(256, 192, 24, "fp32", buoyancy=True)
    v1 = p1.tune(force=True)
    p2 = _plan(256, 192, 24, "fp32", buoyancy=True)
    assert p2.variants() == v1
    # forms the grid does not have
    with pytest.raises(ValueError):
        p1.set_variants(zc4_fx=4)   # nx != 1024
    with pytest.raises(ValueError):
        p1.set_variants(zc3_fy=4)   # ny != 512
    with pytest.raises(ValueError):
        p1.set_variants(zc2_fx=3)
    p64 = _plan(96, 64, 16, "fp64")
    with pytest.raises(ValueError):
        p64.set_variants(zc3_fx=4)  # register forms are single precision


_TUNE = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
from oracle import lh82 as O
from oraclev8_b200._plan import Plan, PlanSpec
nx, ny, nz = 160, 128, 20
z, rho0, th0 = O.build_base_state(nz, 16e3)
p = Plan(PlanSpec(nx, ny, nz, nx * 5e3, ny * 5e3, 16e3, rho0, th0, precision="fp32",
                  projection=True))
print(json.dumps(p.variants()))
"""


def test_tune_cache_file_persists_across_processes(tmp_path):
    cache = tmp_path / "tune.txt"
    env = dict(os.environ, ORACLE_B200_TUNE_CACHE=str(cache), PYTHONDONTWRITEBYTECODE="1")
    outs = []
    for _ in range(2):
        r = subprocess.run([sys.executable, "-c", _TUNE, str(ROOT)], capture_output=True,
                           text=True, timeout=600, env=env, cwd=str(ROOT))
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(json.loads(r.stdout.strip().splitlines()[-1]))
    lines = [ln for ln in cache.read_text().splitlines() if ln.strip()]
    assert len(lines) == 1 and "160x128x20" in lines[0]  # the second process read it
    assert outs[0] == outs[1]
