"""Single-precision step and its FP64-residual defect correction, measured
against the plain FP64 GPU step (itself held to the reference at 1e-12 by
test_gpu_parity.py).

The FP32 state cannot be more accurate than its own rounding, so the
correction is measured against that floor: the non-Nyquist anelastic
divergence (evaluated in FP64) of the FP64 projection rounded to FP32.
"""
import math

import numpy as np
import pytest
import torch

from oracle import lh82 as O
from tests.gpu_helpers import Base, b200_config, dev, host, rel

pytestmark = pytest.mark.gpu


def _non_nyquist(a):
    nx, ny = a.shape[:2]
    ah = np.fft.fft2(a, axes=(0, 1))
    ah[nx // 2, :, :] = 0
    ah[:, ny // 2, :] = 0
    return np.real(np.fft.ifft2(ah, axes=(0, 1)))


def _plans(nx, ny, nz, Lx, Ly, Lz):
    from oraclev8_b200._plan import Plan, PlanSpec
    z, rho0, th0 = O.build_base_state(nz, Lz)
    mk = lambda prec: Plan(PlanSpec(nx, ny, nz, Lx, Ly, Lz, rho0, th0, precision=prec,
                                    projection=True))
    return mk("fp64"), mk("fp32")


def _div64(p64, u, v, w):
    """max |non-Nyquist anelastic divergence| of FP32 fields, in FP64."""
    d = p64.divergence(u.double(), v.double(), w.double())
    return float(np.max(np.abs(_non_nyquist(host(d)))))


def _smooth_state(nx, ny, nz, seed):
    """Band-limited random flow (Gaussian horizontal spectrum) with w = 0 at
    the surface and the lid."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(nx)[:, None, None]
    ky = np.fft.fftfreq(ny)[None, :, None]
    filt = np.exp(-(kx ** 2 + ky ** 2) / 0.02)

    def field(shape, amp):
        f = np.fft.fft2(rng.standard_normal(shape), axes=(0, 1)) * filt
        return amp * np.real(np.fft.ifft2(f, axes=(0, 1)))
    u = field((nx, ny, nz), 30.0)
    v = field((nx, ny, nz), 30.0)
    w = field((nx, ny, nz + 1), 0.5)
    w[:, :, 0] = 0.0
    w[:, :, -1] = 0.0
    return u, v, w


# nz = 48 and 64 run the single-precision sweep with a compile-time level
# count (k_thomas_f32), nz = 16 and 24 the generic one; nx = 512 runs the
# register-resident x pencils (xreg.cuh)
@pytest.mark.parametrize("shape", [(128, 96, 16), (192, 160, 24), (96, 64, 48), (128, 96, 64),
                                   (512, 48, 16)])
def test_refinement_reaches_fp32_storage_floor(shape):
    nx, ny, nz = shape
    Lx, Ly, Lz = nx * 5e3, ny * 5e3, 16e3
    p64, p32 = _plans(nx, ny, nz, Lx, Ly, Lz)
    u, v, w = _smooth_state(nx, ny, nz, seed=nx + ny + nz)
    # FP64 projection of the same (FP32-representable) input
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    u64, v64, w64 = dev(f32(u)), dev(f32(v)), dev(f32(w))
    phi64 = torch.empty_like(u64)
    d_in = _div64(p64, u64, v64, w64)
    p64.project(u64, v64, w64, phi64)
    floor = _div64(p64, u64.float(), v64.float(), w64.float())
    # plain FP32 projection, then one and two correction passes
    mk32 = lambda a: dev(a, torch.float32)
    u32, v32, w32 = mk32(u), mk32(v), mk32(w)
    phi32 = torch.empty_like(u32)
    p32.project(u32, v32, w32, phi32)
    d_plain = _div64(p64, u32, v32, w32)
    e_phi_plain = rel(phi32, host(phi64))
    w_nyq = host(w32).astype(np.float64) - _non_nyquist(host(w32).astype(np.float64))
    p32.refine(u32, v32, w32, phi32)
    # the correction leaves the Nyquist rows (which no projection controls) alone
    w_nyq1 = host(w32).astype(np.float64) - _non_nyquist(host(w32).astype(np.float64))
    d_r1 = _div64(p64, u32, v32, w32)
    e_phi_r1 = rel(phi32, host(phi64))
    p32.refine(u32, v32, w32, phi32)
    d_r2 = _div64(p64, u32, v32, w32)
    print(f"{shape}: div in {d_in:.3e} plain {d_plain:.3e} refined {d_r1:.3e} / {d_r2:.3e} "
          f"floor {floor:.3e}; phi rel err plain {e_phi_plain:.3e} refined {e_phi_r1:.3e}")
    assert d_r1 <= 2.0 * floor and d_r2 <= 2.0 * floor
    assert d_r1 < d_plain
    assert e_phi_r1 <= e_phi_plain
    # the corrected velocity is the FP64 projection to FP32 storage accuracy:
    # the rounding of the stored horizontal wind (a few ulp of max |u, v|)
    # reaches every component through the projection, w included
    scale = max(float(u64.abs().max()), float(v64.abs().max()))
    assert float(np.max(np.abs(w_nyq1 - w_nyq))) <= 1e-7 * scale
    for a, r in ((u32, u64), (v32, v64), (w32, w64)):
        assert float((a.double() - r).abs().max()) <= 4e-7 * scale


def _vortex_case(nx, ny, nz):
    return dict(nx=nx, ny=ny, nz=nz, Lx=nx * 10e3, Ly=ny * 10e3, Lz=16e3, dt=30.0,
                vortex=dict(Vmax=50.0, Rmax=40e3, B=1.6, f=5.0e-5),
                coriolis=dict(f=5.0e-5, mode="beta_plane", beta=2.0e-11, periodic_taper=True),
                advection="upwind5h", buoyancy=True,
                heating=dict(Q_max=3.0 / 3600.0, r_eyewall=40e3, width_r=math.sqrt(2.0) * 15e3,
                             z_peak=6e3, width_z=math.sqrt(2.0) * 2e3), noise_seed=3)


@pytest.mark.parametrize("shape", [(96, 72, 16), (512, 40, 16), (48, 512, 16), (1024, 32, 16),
                                   (32, 1024, 16)])
def test_fp32_steps_track_fp64(shape):
    """Ten full steps of the vortex configuration in FP32, FP32 with one
    correction per step, and FP64: per-field error of the single-precision
    runs, relative to each field's max |.|, and the post-step divergence."""
    from oraclev8_b200.solver import RK3Integrator, State
    from tests.test_oracle_golden import oracle_initial_state
    c = _vortex_case(*shape)
    s0, _ = oracle_initial_state(c)
    base = Base(c["nz"], c["Lz"])
    cfg = b200_config(c)
    p64, _ = _plans(c["nx"], c["ny"], c["nz"], c["Lx"], c["Ly"], c["Lz"])
    runs = {}
    for prec in ("fp64", "fp32", "fp32r"):
        dt = torch.float64 if prec == "fp64" else torch.float32
        integ = RK3Integrator(cfg, base, precision=prec)
        s = State(dev(s0.u, dt), dev(s0.v, dt), dev(s0.w, dt), dev(s0.theta_prime, dt),
                  dev(s0.projection_potential, dt), 0.0)
        for n in range(10):
            s, _ = integ.step(s, c["dt"], n)
        runs[prec] = s
    ref = runs["fp64"]
    fields = ("u", "v", "w", "theta_prime", "projection_potential")
    err = {p: {f: rel(getattr(runs[p], f), host(getattr(ref, f))) for f in fields}
           for p in ("fp32", "fp32r")}
    div = {p: _div64(p64, runs[p].u.float(), runs[p].v.float(), runs[p].w.float())
           for p in ("fp32", "fp32r")}
    print("errors vs fp64:", err, "non-Nyquist divergence:", div)
    # after ten steps (50 projections) the FP32 runs carry a few 1e-6 of the
    # wind scale; w, whose own scale is ~1/100 of the wind's, is held to the
    # same absolute level through a looser relative bound
    bound = dict(u=2e-5, v=2e-5, w=1e-3, theta_prime=2e-5, projection_potential=1e-3)
    for p in ("fp32", "fp32r"):
        for f in fields:
            assert err[p][f] <= bound[f], (p, f, err[p][f])
    assert div["fp32r"] <= div["fp32"]


@pytest.mark.parametrize("zc", [2, 4, 8])
def test_shared_stage_transforms_match_per_stage_transforms(zc):
    """On 1024 x 1024 grids the FP32 plans can take the three fast stages'
    forward x transforms from one launch over the anchor state (variant
    zc4_fxsh): a stage's divergence is linear in its sdt, so its X0 spectrum
    is X0 + sdt X2 with X2 the transform of the buoyancy's flux divergence,
    and the stage's y pencils form it.  Every stage is still projected in full.
    Three FP32-refined steps with the form on and off (every other form the
    same) agree to FP32 rounding, and both track the FP64 step within the
    bounds of the FP32 forms."""
    from oraclev8_b200.solver import RK3Integrator, State
    from tests.test_oracle_golden import oracle_initial_state
    c = _vortex_case(1024, 1024, 8)
    s0, _ = oracle_initial_state(c)
    base = Base(c["nz"], c["Lz"])
    cfg = b200_config(c)
    runs = {}
    for mode in ("fp64", "per_stage", "shared"):
        prec = "fp64" if mode == "fp64" else "fp32r"
        dt = torch.float64 if mode == "fp64" else torch.float32
        integ = RK3Integrator(cfg, base, precision=prec, autotune=False)
        if mode != "fp64":
            # the 1024-point forms on (the defaults of this grid), the shared
            # transforms on or off
            integ.plan.set_variants(zc4_fx=4, zc4_fxs=4, zc4_ix=4, zc4_fy=4, zc4_iy=4,
                                    zc4_fxsh=zc if mode == "shared" else 0)
            assert integ.plan.variants()["zc4_fxsh"] == (zc if mode == "shared" else 0)
        s = State(dev(s0.u, dt), dev(s0.v, dt), dev(s0.w, dt), dev(s0.theta_prime, dt),
                  dev(s0.projection_potential, dt), 0.0)
        for n in range(3):
            s, _ = integ.step(s, c["dt"], n)
        runs[mode] = s
    fields = ("u", "v", "w", "theta_prime", "projection_potential")
    ref = runs["fp64"]
    wind = max(float(ref.u.abs().max()), float(ref.v.abs().max()))
    for f in ("u", "v"):
        d = float((getattr(runs["shared"], f).double() - getattr(runs["per_stage"], f).double())
                  .abs().max())
        assert d <= 1e-6 * wind, (f, d)
    bound = dict(u=2e-5, v=2e-5, w=1e-3, theta_prime=2e-5, projection_potential=1e-3)
    for mode in ("per_stage", "shared"):
        for f in fields:
            err = rel(getattr(runs[mode], f), host(getattr(ref, f)))
            print(mode, f, f"{err:.3e}")
            assert err <= bound[f], (mode, f, err)
    for f in ("w", "theta_prime", "projection_potential"):
        e_sh = rel(getattr(runs["shared"], f), host(getattr(ref, f)))
        e_ps = rel(getattr(runs["per_stage"], f), host(getattr(ref, f)))
        assert e_sh <= 2.0 * e_ps + 1e-6, (f, e_sh, e_ps)


def test_refinement_controls():
    from oraclev8_b200._plan import Plan, PlanSpec
    p64, p32 = _plans(16, 12, 8, 16e4, 12e4, 16e3)
    with pytest.raises(ValueError):
        p64.set_refinement(1)
    with pytest.raises(ValueError):
        p32.set_refinement(5)
    with pytest.raises(ValueError):
        p32.set_refinement(1, every=0)
    p32.set_refinement(2, every=3)
    p32.set_refinement(0)
    u = torch.zeros((16, 12, 8), dtype=torch.float64, device="cuda")
    w = torch.zeros((16, 12, 9), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        p64.refine(u, u.clone(), w, u.clone())


def _register_forms(plan, nx, ny):
    """Turn the register-resident pencil forms of the plan's grid on."""
    kw = {}
    if nx == 512:
        kw.update(zc3_fx=4, zc3_fxs=4, zc3_ix=4, zc3_fxd=4)
    if nx == 1024:
        kw.update(zc4_fx=4, zc4_fxs=4, zc4_ix=4, zc4_fxd=2)
    if ny == 512:
        kw.update(zc3_fy=4, zc3_fyd=2)
    if ny == 1024:
        kw.update(zc4_fy=4, zc4_iy=4)
    plan.set_variants(**kw)


@pytest.mark.parametrize("nx, ny, nz", [(512, 40, 16), (512, 40, 13), (64, 512, 16),
                                        (48, 512, 13), (1024, 40, 16), (1024, 24, 13),
                                        (64, 1024, 16), (48, 1024, 13), (1024, 1024, 8)])
def test_register_pencils_match_stockham(nx, ny, nz, monkeypatch):
    """At nx = 512 or 1024 the FP32 x pencils run the register-resident FFT
    (xreg.cuh, xreg4.cuh), the defect correction's FP64 residual transform
    included, and at ny = 512 or 1024 the y pencils (forced on here, whatever
    the autotuner picks); with those forms off the plan keeps the
    shared-memory Stockham kernels.  Against the FP64
    projection of the same input, the register path is as accurate as the
    Stockham path, field by field, before and after one correction pass; u
    and v of the two agree to a few FP32 ulp of the wind.  nz = 13 leaves a
    partial z-chunk.  (The staged form runs in test_fp32_steps_track_fp64 at
    nx = 512.)"""
    from oraclev8_b200._plan import Plan, PlanSpec
    Lx, Ly, Lz = nx * 5e3, ny * 5e3, 16e3
    z, rho0, th0 = O.build_base_state(nz, Lz)
    mk = lambda prec: Plan(PlanSpec(nx, ny, nz, Lx, Ly, Lz, rho0, th0, precision=prec,
                                    projection=True))
    p_ref = mk("fp32")
    p_ref.shared_memory_forms()
    p_new = mk("fp32")
    _register_forms(p_new, nx, ny)
    p64 = mk("fp64")
    u, v, w = _smooth_state(nx, ny, nz, seed=7 + nz)
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    outs, refined = [], []
    for p, dt in ((p64, torch.float64), (p_ref, torch.float32), (p_new, torch.float32)):
        uu, vv, ww = (dev(f32(a), dt) for a in (u, v, w))
        phi = torch.empty_like(uu)
        p.project(uu, vv, ww, phi)
        outs.append([host(a).astype(np.float64) for a in (uu, vv, ww, phi)])
        if dt == torch.float32:
            p.refine(uu, vv, ww, phi)
            refined.append([host(a).astype(np.float64) for a in (uu, vv, ww, phi)])
    wind = max(float(np.max(np.abs(outs[0][0]))), float(np.max(np.abs(outs[0][1]))))
    for stage, (ref_f, new_f) in (("plain", (outs[1], outs[2])), ("refined", refined)):
        for i, name in enumerate(("u", "v", "w", "phi")):
            r64, ref, new = outs[0][i], ref_f[i], new_f[i]
            scale = float(np.max(np.abs(r64)))
            e_ref = float(np.max(np.abs(ref - r64))) / scale
            e_new = float(np.max(np.abs(new - r64))) / scale
            d = float(np.max(np.abs(new - ref)))
            print(f"nz {nz} {stage} {name}: error vs FP64 stockham {e_ref:.3e} "
                  f"register {e_new:.3e}; max |register - stockham| {d:.3e}")
            assert e_new <= 1.5 * e_ref + 1e-7, (stage, name, e_new, e_ref)
            if name in ("u", "v"):
                assert d <= 1e-6 * wind, (stage, name, d)


@pytest.mark.parametrize("shape", [(32, 16, 16), (48, 24, 40), (48, 24, 80), (64, 40, 32),
                                   (96, 16, 64), (40, 12, 48)])
def test_slow_tendency_forms_agree(shape, monkeypatch):
    """For FP32 state the slow tendency has three forms: a gather (k_slow_f32,
    the plan's slow_xw variant at 0), marching along x with the neighbour rows
    loaded per step (k_slow_xw, variant 1; nx % 16 == 0, ny % 8 == 0), and
    marching along x over planes of 4 or 8 rows staged by bulk copies
    (k_slow_xt, variants 4 and 8, and 24 and 28 with two cells per thread;
    nz in {32, 48, 64, 80}).  The first two share
    the gather's operation order and agree with it to FP32 rounding; the
    plane-staged form forms the WS5 derivative as a centred part less the
    upwind sign times a dissipative part, so two full steps of the vortex
    configuration are held against the FP64 step instead, to the accuracy
    class of every FP32 form after two steps (a few 1e-7 of the wind scale
    for u, v, theta'; w and phi, whose scales are ~1/100 of the wind's,
    through looser relative bounds).  The shapes
    cover the periodic halo rows and columns (several tiles and x-segments, a
    last segment shorter than the others, row blocks whose halo wraps at both
    ends) and, at nz = 40, two z-chunks of k_slow_xw with the lid in the
    second."""
    from oraclev8_b200.solver import RK3Integrator, State
    from tests.test_oracle_golden import oracle_initial_state
    c = _vortex_case(*shape)
    s0, _ = oracle_initial_state(c)
    base = Base(c["nz"], c["Lz"])
    cfg = b200_config(c)
    fields = ("u", "v", "w", "theta_prime", "projection_potential")

    def run(prec, xw=None):
        dt = torch.float64 if prec == "fp64" else torch.float32
        integ = RK3Integrator(cfg, base, precision=prec)
        if xw is not None:
            integ.plan.set_variants(slow_xw=xw)
        d = lambda a: dev(a, dt)
        s = State(d(s0.u), d(s0.v), d(s0.w), d(s0.theta_prime), d(s0.projection_potential), 0.0)
        for n in range(2):
            s, _ = integ.step(s, c["dt"], n)
        return {f: host(getattr(s, f)).astype(np.float64) for f in fields}

    ref = run("fp64")
    outs = {}
    for xw in (0, 1, 4, 8, 24, 28):
        try:
            outs[xw] = run("fp32", xw)
        except ValueError:  # the form does not exist for this grid
            continue
    assert 0 in outs and len(outs) >= 2, sorted(outs)
    if shape[2] in (32, 48, 64, 80):
        assert 4 in outs, sorted(outs)
    err = {xw: {f: float(np.max(np.abs(o[f] - ref[f]))) / float(np.max(np.abs(ref[f])))
                for f in fields} for xw, o in outs.items()}
    for xw in outs:
        print(shape, "form", xw, " ".join(f"{f}:{e:.2e}" for f, e in err[xw].items()))
    if 1 in outs:  # same operation order as the gather
        for f in fields:
            d = float(np.max(np.abs(outs[1][f] - outs[0][f]))) / float(np.max(np.abs(ref[f])))
            assert d <= 1e-5, (f, d)
    bound = dict(u=2e-6, v=2e-6, w=3e-4, theta_prime=2e-6, projection_potential=2e-4)
    for xw in outs:
        for f in fields:
            assert err[xw][f] <= bound[f], (xw, f, err[xw][f])


@pytest.mark.parametrize("shape", [(48, 24, 80), (64, 40, 32), (96, 16, 64), (40, 12, 48)])
def test_slow_tendency_forms_against_fp64(shape):
    """The slow tendency alone (oracle_b200_tendency: advection, beta-plane
    Coriolis and heating) of a band-limited random state with w != 0, in
    each FP32 form against the FP64 tendency of the same (FP32-representable)
    input: every form within 1e-5 of each field's max |tendency|, the
    plane-staged form (k_slow_xt) within twice the gather form's own error,
    and within 1e-6 of the row-loading x-march (k_slow_xw) where both exist."""
    from oraclev8_b200 import _lib as L
    from oraclev8_b200.solver import RK3Integrator
    c = _vortex_case(*shape)
    nx, ny, nz = shape
    base = Base(nz, c["Lz"])
    cfg = b200_config(c)
    u, v, w = _smooth_state(nx, ny, nz, seed=nx + nz)
    th = 0.5 * _smooth_state(nx, ny, nz, seed=nx + nz + 1)[0] / 30.0
    fields = [np.asarray(a, dtype=np.float32).astype(np.float64) for a in (u, v, w, th)]
    mask = L.OB_TEND_ADVECTION | L.OB_TEND_CORIOLIS | L.OB_TEND_HEATING
    p64 = RK3Integrator(cfg, base, precision="fp64").plan
    ref = [host(t) for t in p64.tendency(mask, *(dev(a, torch.float64) for a in fields), c["dt"])]
    scale = [np.abs(r).max() for r in ref]
    errs, outs = {}, {}
    for xw in (0, 1, 4, 8, 24, 28):
        p = RK3Integrator(cfg, base, precision="fp32").plan
        try:
            p.set_variants(slow_xw=xw)
        except ValueError:
            continue
        outs[xw] = [host(t).astype(np.float64)
                    for t in p.tendency(mask, *(dev(a, torch.float32) for a in fields), c["dt"])]
        errs[xw] = [np.abs(a - r).max() / sc for a, r, sc in zip(outs[xw], ref, scale)]
        print(shape, "form", xw, " ".join(f"{n}:{e:.2e}" for n, e in
                                          zip(("du", "dv", "dw", "dth"), errs[xw])))
    assert 0 in errs and 4 in errs, sorted(errs)
    for xw, e in errs.items():
        assert max(e) <= 1e-5, (xw, e)
    for xw in (4, 8, 24, 28):
        if xw not in errs:
            continue
        for n in range(4):
            assert errs[xw][n] <= 2 * errs[0][n] + 1e-7, (xw, n, errs[xw][n], errs[0][n])
            if 1 in outs:
                d = np.abs(outs[xw][n] - outs[1][n]).max() / scale[n]
                assert d <= 1e-6, (xw, n, d)


@pytest.mark.parametrize("nx, ny, nz", [(64, 512, 16), (48, 512, 13), (512, 40, 16),
                                        (512, 48, 13), (512, 512, 8)])
def test_register_damper_matches_stockham(nx, ny, nz, monkeypatch):
    """An FP32 plan runs the Helmholtz damper in the register-resident
    kernels where the grid allows: the x transforms at nx = 512 (the field
    forms of the forward and inverse x pencils) and the y stage at ny = 512
    (forward y transforms, the divergent-part multipliers and inverse y
    transforms in one pass).  With the register forms off it keeps the
    shared-memory kernels.  Against the FP64 damper tendency of the same
    input, the register forms are as accurate as the shared-memory ones, and
    the two FP32 forms agree to FP32 rounding.  nz = 13 leaves a partial
    z-chunk."""
    from oraclev8_b200 import _lib as L
    from oraclev8_b200._plan import Plan, PlanSpec
    Lx, Ly, Lz = nx * 5e3, ny * 5e3, 16e3
    z, rho0, th0 = O.build_base_state(nz, Lz)
    mk = lambda prec: Plan(PlanSpec(nx, ny, nz, Lx, Ly, Lz, rho0, th0, precision=prec,
                                    projection=True, damping=True, epsilon=0.5))
    p_ref = mk("fp32")
    p_ref.shared_memory_forms()
    p_new = mk("fp32")
    _register_forms(p_new, nx, ny)
    p64 = mk("fp64")
    u, v, w = _smooth_state(nx, ny, nz, seed=31 + nz)
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    th = np.zeros((nx, ny, nz))
    outs = []
    for p, dt in ((p64, torch.float64), (p_ref, torch.float32), (p_new, torch.float32)):
        du, dv, _, _ = p.tendency(L.OB_TEND_DAMPING, dev(f32(u), dt), dev(f32(v), dt),
                                  dev(f32(w), dt), dev(th, dt), 30.0)
        outs.append([host(du).astype(np.float64), host(dv).astype(np.float64)])
    for i, name in enumerate(("du", "dv")):
        r64, ref, new = outs[0][i], outs[1][i], outs[2][i]
        scale = float(np.max(np.abs(r64)))
        assert scale > 0.0
        e_ref = float(np.max(np.abs(ref - r64))) / scale
        e_new = float(np.max(np.abs(new - r64))) / scale
        e_two = float(np.max(np.abs(new - ref))) / scale
        print(name, f"shared-memory {e_ref:.2e} register {e_new:.2e} between {e_two:.2e}")
        assert e_new <= 1.5 * e_ref + 1e-7, (name, e_new, e_ref)
        assert e_two <= 2e-6, (name, e_two)
