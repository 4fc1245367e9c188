"""Production slow components on the GPU (tendency.py:1259-1668).

* Surface drag, the sponge, Laplacian and biharmonic diffusion, Newtonian
  cooling and the intensity cap: each component's tendency against the
  reference's own output (production.npz), FP64 within 1e-12 of the field's
  max |.|, FP32 within its rounding.
* Full RK3 steps of two production configurations (beta-plane with WS5,
  heating, drag, sponge, biharmonic diffusion and cooling; f-plane with
  centred advection, the divergence damper, drag, sponge, Laplacian diffusion
  and cooling) against the reference's states, every field, every step.
* The FP32 and FP32-refined steps of a production configuration track FP64.
* The reference's production run loop (vortex, pre-balance, production
  steps with the intensity cap after each) through the public API.
"""
import numpy as np
import pytest
import torch

from tests.gpu_helpers import TOL64, Base, b200_config, dev, host, load_case, rel

pytestmark = pytest.mark.gpu

PROD_CASES = ["prod_beta", "prod_lap_fplane"]


@pytest.fixture(scope="module")
def prod(golden_dir):
    return np.load(golden_dir / "production.npz")


def _state(g, dtype):
    from oraclev8_b200.solver import State
    return State(dev(g["in_u"], dtype), dev(g["in_v"], dtype), dev(g["in_w"], dtype),
                 dev(g["in_th"], dtype), dev(g["in_phi"], dtype), 0.0)


def _components(g):
    from oraclev8_b200.solver import (HorizontalDiffusionComponent, HyperDiffusionComponent,
                                      IntensityCapComponent, NewtonianCoolingComponent,
                                      SpongeDampingComponent, SurfaceDragComponent)
    nx, ny, Lx, Ly, Lz = int(g["nx"]), int(g["ny"]), float(g["Lx"]), float(g["Ly"]), \
        float(g["Lz"])
    return {
        "drag": SurfaceDragComponent(Cd=1.5e-3, H_bl=1500.0, u_env=2.0, v_env=-1.0),
        "drag0": SurfaceDragComponent(),
        "sponge": SpongeDampingComponent(Lz=Lz, alpha_max=0.01, sponge_fraction=0.4,
                                         u_env=-1.5, v_env=0.5),
        "lap": HorizontalDiffusionComponent(nu_H=2.0e5, Lx=Lx, Ly=Ly, nx=nx, ny=ny),
        "hyper": HyperDiffusionComponent(nu4=3.0e12, Lx=Lx, Ly=Ly, nx=nx, ny=ny),
        "cool": NewtonianCoolingComponent(tau=1800.0),
        "cap": IntensityCapComponent(v_cap=15.0, tau=300.0, u_env=1.0, v_env=-2.0),
    }


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_production_component_tendencies(prod, dtype):
    g = prod
    base = Base(int(g["nz"]), float(g["Lz"]))
    s = _state(g, dtype)
    # FP32: single-precision arithmetic on FP32 inputs; the biharmonic's two
    # Laplacians cancel about two digits of the inputs' scale
    tol = TOL64 if dtype == torch.float64 else 2e-5
    seen = set()
    for name, comp in _components(g).items():
        t = comp.compute_tendency(s, None, None, base, 30.0)
        for f in ("du_dt", "dv_dt", "dw_dt", "dtheta_prime_dt"):
            key = f"{name}_{f}"
            val = getattr(t, f)
            if key not in g.files:
                assert val is None, key
                continue
            assert val is not None and val.dtype == dtype, key
            e = rel(val, g[key])
            assert e <= tol, (key, e)
            seen.add(key)
    assert seen == {k for k in g.files if not (k.startswith("in_") or len(g[k].shape) == 0)}


def test_intensity_cap_env_and_inactive_cells(prod):
    """Below the cap the tendency is exactly zero; set_env moves the
    perturbation origin (tendency.py:1396-1408)."""
    from oraclev8_b200.solver import IntensityCapComponent
    g = prod
    base = Base(int(g["nz"]), float(g["Lz"]))
    s = _state(g, torch.float64)
    cap = IntensityCapComponent(v_cap=15.0, tau=300.0)
    cap.set_env(1.0, -2.0)
    t = cap.compute_tendency(s, None, None, base, 30.0)
    assert rel(t.du_dt, g["cap_du_dt"]) <= TOL64 and rel(t.dv_dt, g["cap_dv_dt"]) <= TOL64
    sp = np.hypot(g["in_u"] - 1.0, g["in_v"] + 2.0)
    below = sp <= 15.0
    assert below.any() and (~below).any()
    assert np.all(host(t.du_dt)[below] == 0.0) and np.all(host(t.dv_dt)[below] == 0.0)
    big = IntensityCapComponent(v_cap=1e6).compute_tendency(s, None, None, base, 30.0)
    assert not host(big.du_dt).any() and not host(big.dv_dt).any()


@pytest.mark.parametrize("case", PROD_CASES)
def test_production_steps_match_reference(golden_dir, case):
    from oraclev8_b200.solver import RK3Integrator, State
    g, c = load_case(golden_dir, case)
    base = Base(c["nz"], c["Lz"])
    integ = RK3Integrator(b200_config(c), base, precision="fp64")
    s = State(dev(g["s0_u"]), dev(g["s0_v"]), dev(g["s0_w"]), dev(g["s0_th"]),
              dev(g["s0_phi"]), float(g["s0_t"]))
    for n in range(c["nsteps"]):
        s, dg = integ.step(s, dt=c["dt"], step_number=n)
        for f, k in (("u", "u"), ("v", "v"), ("w", "w"), ("theta_prime", "th"),
                     ("projection_potential", "phi")):
            key = f"s{n + 1}_{k}"
            if key not in g.files:
                continue
            e = rel(getattr(s, f), g[key])
            assert e <= TOL64, (case, n, f, e)
        if f"d{n + 1}" in g.files:
            d = np.array([dg.max_u, dg.max_v, dg.max_w, dg.max_theta_prime,
                          dg.surface_phi_min, dg.surface_phi_max])
            ref = g[f"d{n + 1}"]
            assert np.all(np.abs(d - ref) <= 1e-11 * np.maximum(np.abs(ref), 1e-30)), (d, ref)


@pytest.mark.parametrize("case", PROD_CASES)
def test_production_steps_fp32_track_fp64(golden_dir, case):
    """The single-precision steps of the production configurations against
    the reference's FP64 states: within the rounding of the FP32 state."""
    from oraclev8_b200.solver import RK3Integrator, State
    g, c = load_case(golden_dir, case)
    base = Base(c["nz"], c["Lz"])
    for prec in ("fp32", "fp32r"):
        integ = RK3Integrator(b200_config(c), base, precision=prec)
        f32 = torch.float32
        s = State(dev(g["s0_u"], f32), dev(g["s0_v"], f32), dev(g["s0_w"], f32),
                  dev(g["s0_th"], f32), dev(g["s0_phi"], f32), float(g["s0_t"]))
        for n in range(c["nsteps"]):
            s, _ = integ.step(s, dt=c["dt"], step_number=n)
        last = c["nsteps"]
        bound = dict(u=2e-5, v=2e-5, w=1e-3, th=2e-5, phi=1e-3)
        for f, k in (("u", "u"), ("v", "v"), ("w", "w"), ("theta_prime", "th"),
                     ("projection_potential", "phi")):
            key = f"s{last}_{k}"
            if key in g.files:
                e = rel(getattr(s, f), g[key])
                assert e <= bound[k], (case, prec, f, e)


def test_production_fp32_slow_forms_at_marching_size():
    """At a size where the plain configuration takes the x-marching slow
    kernel (nx % 16 == 0, ny % 8 == 0), the production terms route the step
    through the gather kernel; its FP32 tendencies match FP64 to rounding."""
    from oraclev8_b200 import _lib as L
    from oraclev8_b200._plan import Plan, PlanSpec
    from oraclev8_b200.solver.tendency import drag_fields, sponge_fields
    from oraclev8_b200.solver import SpongeDampingComponent, SurfaceDragComponent
    nx, ny, nz, Lx, Ly, Lz = 64, 48, 16, 1280e3, 960e3, 16e3
    base = Base(nz, Lz)
    z = np.asarray(base.z)
    extra = dict(advection=L.OB_ADV_UPWIND5H, coriolis=L.OB_COR_FPLANE, f0=5e-5,
                 diffusion=L.OB_DIFF_BIHARMONIC, diff_nu=1e13, diff_dx2=(Lx / nx) ** 2,
                 diff_dy2=(Ly / ny) ** 2, cooling=True, cool_alpha=1.0 / 3600.0,
                 **drag_fields(SurfaceDragComponent(2e-3, 2000.0, -3.0, 1.0), z),
                 **sponge_fields(SpongeDampingComponent(Lz, 0.02, 0.3, -3.0, 1.0), z))
    rng = np.random.default_rng(77)
    fields = [10.0 * rng.standard_normal((nx, ny, nz)), 10.0 * rng.standard_normal((nx, ny, nz)),
              0.3 * rng.standard_normal((nx, ny, nz + 1)), rng.standard_normal((nx, ny, nz))]
    out = {}
    for prec, dt in (("fp64", torch.float64), ("fp32", torch.float32)):
        p = Plan(PlanSpec(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz, rho0=base.rho0,
                          theta0=base.theta0, precision=prec, **extra))
        mask = (L.OB_TEND_ADVECTION | L.OB_TEND_CORIOLIS | L.OB_TEND_DRAG | L.OB_TEND_SPONGE
                | L.OB_TEND_DIFFUSION | L.OB_TEND_COOLING)
        out[prec] = [host(t) for t in p.tendency(mask, *(dev(a, dt) for a in fields), 30.0)]
    for a, r, name in zip(out["fp32"], out["fp64"], ("du", "dv", "dw", "dth")):
        e = rel(a, r)
        assert e <= 2e-5, (name, e)


@pytest.mark.parametrize("shape, adv, diff", [
    ((64, 40, 32), "upwind5h", "biharmonic"), ((48, 24, 80), "centered2", "biharmonic"),
    ((96, 16, 64), "centered2", "laplacian"), ((40, 12, 48), "upwind5h", "laplacian")])
def test_production_slow_forms_against_fp64(shape, adv, diff):
    """The production slow tendency (advection, f-plane Coriolis, surface
    drag, sponge, Laplacian or biharmonic diffusion, Newtonian cooling) of a
    random state in every FP32 slow form the grid allows -- the gather
    (variant 0) and the plane-staged x-march's production form (4, 8; its
    planes carry the inner Laplacians) -- against the FP64 tendency of the
    same input: within 2e-5 of each field's max |tendency|.  The shapes cover
    y-halos that wrap at both ends, several x-segments and a short last one,
    and the lid (w's sponge on every half level)."""
    from oraclev8_b200 import _lib as L
    from oraclev8_b200._plan import Plan, PlanSpec
    from oraclev8_b200.solver.tendency import drag_fields, sponge_fields
    from oraclev8_b200.solver import SpongeDampingComponent, SurfaceDragComponent
    nx, ny, nz = shape
    Lx, Ly, Lz = nx * 20e3, ny * 20e3, 16e3
    base = Base(nz, Lz)
    z = np.asarray(base.z)
    extra = dict(advection=L.OB_ADV_UPWIND5H if adv == "upwind5h" else L.OB_ADV_CENTERED2,
                 coriolis=L.OB_COR_FPLANE, f0=5e-5,
                 diffusion=L.OB_DIFF_BIHARMONIC if diff == "biharmonic" else L.OB_DIFF_LAPLACIAN,
                 diff_nu=1e13 if diff == "biharmonic" else 2e4,
                 diff_dx2=(Lx / nx) ** 2, diff_dy2=(Ly / ny) ** 2, cooling=True,
                 cool_alpha=1.0 / 3600.0,
                 **drag_fields(SurfaceDragComponent(2e-3, 2000.0, -3.0, 1.0), z),
                 **sponge_fields(SpongeDampingComponent(Lz, 0.02, 0.3, -3.0, 1.0), z))
    rng = np.random.default_rng(nx + nz)
    fields = [np.asarray(a, np.float32).astype(np.float64) for a in (
        10.0 * rng.standard_normal((nx, ny, nz)), 10.0 * rng.standard_normal((nx, ny, nz)),
        0.3 * rng.standard_normal((nx, ny, nz + 1)), rng.standard_normal((nx, ny, nz)))]
    mask = (L.OB_TEND_ADVECTION | L.OB_TEND_CORIOLIS | L.OB_TEND_DRAG | L.OB_TEND_SPONGE
            | L.OB_TEND_DIFFUSION | L.OB_TEND_COOLING)

    def plan(prec):
        return Plan(PlanSpec(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz, rho0=base.rho0,
                             theta0=base.theta0, precision=prec, autotune=False, **extra))
    ref = [host(t) for t in plan("fp64").tendency(mask, *(dev(a, torch.float64) for a in fields),
                                                  30.0)]
    forms = []
    for xw in (0, 4, 8):
        p = plan("fp32")
        try:
            p.set_variants(slow_xw=xw)
        except ValueError:
            continue
        forms.append(xw)
        out = [host(t) for t in p.tendency(mask, *(dev(a, torch.float32) for a in fields), 30.0)]
        errs = [rel(a, r) for a, r in zip(out, ref)]
        print(shape, adv, diff, "form", xw, " ".join(f"{e:.2e}" for e in errs))
        for name, e in zip(("du", "dv", "dw", "dth"), errs):
            assert e <= 2e-5, (xw, name, e)
    assert forms[0] == 0 and 4 in forms, forms


@pytest.mark.parametrize("precision", ["fp64", "fp32r"])
def test_production_run_loop_matches_reference(golden_dir, precision):
    """The production run loop of the reference (run_storm.py:120-172) through
    the public API: device vortex fill with the wind taper, theta' zeroed,
    build_prebal_config pre-balance, build_production_config steps with the
    intensity cap added after each step.  FP64 within 1e-12 of the reference
    at every stage; FP32-refined within the FP32 bounds of the step tests."""
    import json
    from dataclasses import replace as dc_replace
    from oraclev8_b200.production_config import (BaseState, build_prebal_config,
                                                 build_production_config)
    from oraclev8_b200.solver import IntensityCapComponent, RK3Integrator
    from oraclev8_b200.vortex_init import HollandVortexInit
    g = np.load(golden_dir / "production_storm.npz")
    c = json.loads(str(g["config_json"]))
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    Lx, Ly, Lz = nx * c["dx"], ny * c["dx"], c["Lz"]
    base = BaseState(nz, Lz)
    dtype = torch.float64 if precision == "fp64" else torch.float32
    fp64 = precision == "fp64"
    # FP32-refined: theta' starts at zero and grows from small increments, so
    # its error relative to its own max carries the rounding of those
    # increments, which varies (1.9e-5 to 2.1e-5 after the first step) with
    # the kernel forms the timing-based autotuner keeps; 5e-5 bounds it
    bound = (dict(u=TOL64, v=TOL64, w=TOL64, th=TOL64, phi=TOL64) if fp64 else
             dict(u=2e-5, v=2e-5, w=1e-3, th=5e-5, phi=1e-3))
    fields = (("u", "u"), ("v", "v"), ("w", "w"), ("theta_prime", "th"),
              ("projection_potential", "phi"))

    def check(s, prefix, what, phi_bound=None):
        for f, k in fields:
            e = rel(getattr(s, f), g[prefix + k])
            b = phi_bound if (k == "phi" and phi_bound is not None) else bound[k]
            assert e <= b, (what, f, e)
        # without fast components the step leaves t where it was
        # (integrator.py:241-258, 489)
        assert s.t == float(g[prefix + "t"]), what

    s = HollandVortexInit(f=c["f"], u_env=c["u_env"], v_env=c["v_env"], **c["vortex"]
                          ).build_state(nx, ny, nz, Lx, Ly, base, dtype=dtype)
    s = dc_replace(s, theta_prime=torch.zeros_like(s.theta_prime))
    check(s, "s0_", "init")
    pre = RK3Integrator(build_prebal_config(nx, ny, nz, Lx, Ly, Lz), base, precision=precision)
    for i in range(c["n_prebal"]):
        s, _ = pre.step(s, dt=1.0, step_number=i)
    # phi of the last pre-balance projection is the potential of what the
    # four before it left behind (max |phi| falls from 948 to 92 Pa): moving
    # u, v of the initial state by one ulp moves the reference's own value by
    # 1.5e-12 to 1.8e-12 of its max, so FP64 is held to 5e-12 there; every
    # other field, and phi after each production step, keeps the 1e-12 bar
    check(s, "pb_", "prebal", phi_bound=5e-12 if fp64 else None)
    integ = RK3Integrator(build_production_config(nx, ny, nz, Lx, Ly, Lz, c["f"], c["u_env"],
                                                  c["v_env"]), base, precision=precision)
    cap = IntensityCapComponent(v_cap=c["v_cap"], tau=c["tau_cap"], u_env=c["u_env"],
                                v_env=c["v_env"])
    for n in range(c["nsteps"]):
        s, dg = integ.step(s, dt=c["dt"], step_number=n)
        ct = cap.compute_tendency(s, None, None, base, c["dt"])
        if fp64:
            assert int(torch.count_nonzero(ct.du_dt)) == int(g["capped_cells"][n])
        s = dc_replace(s, u=s.u + c["dt"] * ct.du_dt, v=s.v + c["dt"] * ct.dv_dt)
        check(s, f"s{n + 1}_", f"step {n}")
        if fp64:
            d = np.array([dg.max_u, dg.max_v, dg.max_w, dg.max_theta_prime,
                          dg.surface_phi_min, dg.surface_phi_max])
            ref = g[f"d{n + 1}"]
            assert np.all(np.abs(d - ref) <= 1e-11 * np.maximum(np.abs(ref), 1e-30)), (d, ref)
