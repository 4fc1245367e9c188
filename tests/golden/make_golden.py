"""Generate golden fixtures by running the UNMODIFIED reference (Oracle V8).

Give the root of the reference tree (the directory holding ``oracle_v8``) with
``--reference PATH`` or the ``ORACLE_V8_REF`` environment variable:

    python tests/golden/make_golden.py --reference PATH          # small fixtures (seconds)
    python tests/golden/make_golden.py --reference PATH --long   # + config-0 6 h run (~8 min)

It imports ``oracle_v8`` from the reference with ``ORACLE_GPU=0`` (NumPy path),
builds seeded inputs with the reference's own public constructors, and stores
the reference's outputs as ``.npz`` / ``.json`` files beside this script.  The
tests never import the reference: they read these files only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
from pathlib import Path

os.environ["ORACLE_GPU"] = "0"
os.environ.setdefault("ORACLE_DIAG_EVERY", "1")
sys.dont_write_bytecode = True


def _reference_root() -> str:
    """The reference tree's root: ``--reference PATH`` or ``ORACLE_V8_REF``."""
    argv = sys.argv[1:]
    for i, a in enumerate(argv):
        if a == "--reference" and i + 1 < len(argv):
            return argv[i + 1]
        if a.startswith("--reference="):
            return a.split("=", 1)[1]
    ref = os.environ.get("ORACLE_V8_REF")
    if not ref:
        sys.exit("make_golden.py: give the reference tree with --reference PATH or ORACLE_V8_REF")
    return ref


REF = _reference_root()
sys.path.insert(0, REF)

import numpy as np  # noqa: E402

from oracle_v8.solver import (  # noqa: E402
    LH82AnelasticEquationSet, BuoyancyComponent, AnelasticProjection,
    AdvectionComponent, CoriolisComponent, DiabaticHeatingComponent,
    HelmholtzDivergenceDampingComponent, OperatorConfig, RK3Integrator, State,
)
from oracle_v8.solver.tendency import (  # noqa: E402
    SurfaceDragComponent, SpongeDampingComponent, HorizontalDiffusionComponent,
    HyperDiffusionComponent, NewtonianCoolingComponent, IntensityCapComponent,
)
from oracle_v8.grid.staggering import LorenzStaggering  # noqa: E402
from oracle_v8.solver.tendency import anelastic_divergence, _phi_gradient  # noqa: E402
from oracle_v8.solver.poisson import VariableCoefficientPoissonSolver  # noqa: E402
from oracle_v8.production_config import build_base_state  # noqa: E402
from oracle_v8 import production_config as PC  # noqa: E402
from oracle_v8.vortex_init import HollandVortexInit  # noqa: E402
from oracle_v8.storm_tracker import find_storm_centre  # noqa: E402
from oracle_v8.validation import analytical_solutions as ana  # noqa: E402

OUT = Path(__file__).resolve().parent


class Base:
    def __init__(self, nz, Lz):
        self.z, self.rho0, self.theta0 = build_base_state(nz=nz, Lz=Lz)


class LinearDecayHolland(HollandVortexInit):
    """Holland vortex whose wind decays linearly to zero at ``top`` metres."""

    def __init__(self, *a, top=12_000.0, **k):
        super().__init__(*a, **k)
        self._top = float(top)

    def wind_vertical_structure(self, z):
        return np.maximum(0.0, 1.0 - z / self._top)


def random_state(rng, nx, ny, nz):
    u = 10.0 * rng.standard_normal((nx, ny, nz))
    v = 10.0 * rng.standard_normal((nx, ny, nz))
    w = 0.5 * rng.standard_normal((nx, ny, nz + 1))
    w[:, :, 0] = 0.0
    w[:, :, -1] = 0.0
    th = 2.0 * rng.standard_normal((nx, ny, nz))
    phi = 50.0 * rng.standard_normal((nx, ny, nz))
    return State(u=u, v=v, w=w, theta_prime=th, projection_potential=phi, t=0.0)


def st_dict(prefix, s):
    return {f"{prefix}u": s.u, f"{prefix}v": s.v, f"{prefix}w": s.w,
            f"{prefix}th": s.theta_prime, f"{prefix}phi": s.projection_potential,
            f"{prefix}t": np.float64(s.t)}


# ---------------------------------------------------------------------------
# Component-level fixtures
# ---------------------------------------------------------------------------

def gen_components():
    nx, ny, nz = 16, 12, 8
    Lx, Ly, Lz = 320e3, 300e3, 4000.0
    rng = np.random.default_rng(1234)
    base = Base(nz, Lz)
    s = random_state(rng, nx, ny, nz)
    eq, stg = LH82AnelasticEquationSet(), LorenzStaggering()
    out = dict(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz)
    out.update(st_dict("in_", s))
    out["z"], out["rho0"], out["theta0"] = base.z, base.rho0, base.theta0
    # a tie case for the upwind selector (a == 0 exactly)
    s.u[3, 4, :] = 0.0
    s.v[5, 2, :] = 0.0
    out["in_u"], out["in_v"] = s.u.copy(), s.v.copy()

    out["buoy_dw"] = BuoyancyComponent().compute_tendency(s, eq, stg, base, 1.0).dw_dt
    for scheme in ("upwind5h", "centered2"):
        t = AdvectionComponent(nx, ny, nz, Lx, Ly, Lz, scheme=scheme).compute_tendency(
            s, eq, stg, base, 30.0)
        out[f"adv_{scheme}_du"] = t.du_dt
        out[f"adv_{scheme}_dv"] = t.dv_dt
        out[f"adv_{scheme}_dw"] = t.dw_dt
        out[f"adv_{scheme}_dth"] = t.dtheta_prime_dt
    cor = {
        "fplane": CoriolisComponent(f=5e-5, mode="f_plane", u_env=1.5, v_env=-0.5),
        "beta_taper": CoriolisComponent(f=4.99e-5, mode="beta_plane", beta=2.15e-11,
                                        Ly=Ly, ny=ny, periodic_taper=True),
        "beta_derived": CoriolisComponent(f=6.164e-5, mode="beta_plane", Ly=Ly, ny=ny,
                                          u_env=-3.0, periodic_taper=False),
    }
    for k, c in cor.items():
        t = c.compute_tendency(s, eq, stg, base, 30.0)
        out[f"cor_{k}_du"] = t.du_dt
        out[f"cor_{k}_dv"] = t.dv_dt
    heat = DiabaticHeatingComponent(Q_max=3.0 / 3600.0, r_eyewall=40e3,
                                    width_r=math.sqrt(2.0) * 15e3, z_peak=2e3,
                                    width_z=math.sqrt(2.0) * 1e3, nx=nx, ny=ny, nz=nz,
                                    Lx=Lx, Ly=Ly, Lz=Lz)
    out["heat_dth"] = heat.compute_tendency(s, eq, stg, base, 30.0).dtheta_prime_dt
    hd = HelmholtzDivergenceDampingComponent(epsilon=0.5, Lx=Lx, Ly=Ly, nx=nx, ny=ny)
    t = hd.compute_tendency(s, eq, stg, base, 30.0)
    out["helm_du"], out["helm_dv"] = t.du_dt, t.dv_dt

    proj = AnelasticProjection(nx, ny, nz, Lx, Ly, Lz)
    solver = proj._solver
    rf = base.rho0
    rh = np.zeros(nz + 1)
    rh[1:-1] = 0.5 * (rf[:-1] + rf[1:])
    rh[0], rh[-1] = rf[0], rf[-1]
    d = anelastic_divergence(s.u, s.v, s.w, rf, rh, solver.kx, solver.ky, Lz / nz)
    out["div"] = d
    gx, gy, gz = _phi_gradient(s.projection_potential, solver.kx, solver.ky, Lz / nz)
    out["grad_x"], out["grad_y"], out["grad_z"] = gx, gy, gz
    res = solver.solve(d, rf, rh, log_diagnostics=True)
    out["solve_phi"] = res.phi
    out["solve_compat"] = np.float64(res.compatibility_residual)
    out["solve_disc"] = np.float64(res.discrete_operator_residual)
    out["apply_op"] = solver.apply_operator(s.projection_potential, rf, rh)
    s2 = State(u=s.u.copy(), v=s.v.copy(), w=s.w.copy(), theta_prime=s.theta_prime.copy(),
               projection_potential=s.projection_potential.copy(), t=0.0)
    proj.apply_projection(s2, eq, stg, base, 1.0)
    out.update(st_dict("proj_", s2))
    out["proj_div_after"] = anelastic_divergence(s2.u, s2.v, s2.w, rf, rh, solver.kx,
                                                 solver.ky, Lz / nz)
    np.savez_compressed(OUT / "components.npz", **out)


def gen_production():
    """Production slow components (tendency.py:1259-1668) and the intensity
    cap, on the components fixture's random state."""
    nx, ny, nz = 16, 12, 8
    Lx, Ly, Lz = 320e3, 300e3, 4000.0
    rng = np.random.default_rng(1234)
    base = Base(nz, Lz)
    s = random_state(rng, nx, ny, nz)
    eq, stg = LH82AnelasticEquationSet(), LorenzStaggering()
    out = dict(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz)
    out.update(st_dict("in_", s))
    comps = {
        "drag": SurfaceDragComponent(Cd=1.5e-3, H_bl=1500.0, u_env=2.0, v_env=-1.0),
        "drag0": SurfaceDragComponent(),
        "sponge": SpongeDampingComponent(Lz=Lz, alpha_max=0.01, sponge_fraction=0.4,
                                         u_env=-1.5, v_env=0.5),
        "lap": HorizontalDiffusionComponent(nu_H=2.0e5, Lx=Lx, Ly=Ly, nx=nx, ny=ny),
        "hyper": HyperDiffusionComponent(nu4=3.0e12, Lx=Lx, Ly=Ly, nx=nx, ny=ny),
        "cool": NewtonianCoolingComponent(tau=1800.0),
        "cap": IntensityCapComponent(v_cap=15.0, tau=300.0, u_env=1.0, v_env=-2.0),
    }
    for k, c in comps.items():
        t = c.compute_tendency(s, eq, stg, base, 30.0)
        for f in ("du_dt", "dv_dt", "dw_dt", "dtheta_prime_dt"):
            val = getattr(t, f)
            if val is not None:
                out[f"{k}_{f}"] = val
    np.savez_compressed(OUT / "production.npz", **out)


# ---------------------------------------------------------------------------
# Integrator fixtures (a few full RK3 steps per component set)
# ---------------------------------------------------------------------------

STEP_CASES = {
    # config-0 physics: β-plane (taper), WS5, buoyancy, no heating, no damper
    "beta_ws5": dict(nx=32, ny=32, nz=8, Lx=640e3, Ly=640e3, Lz=16e3, dt=60.0, nsteps=3,
                     vortex=dict(Vmax=40.0, Rmax=50e3, B=1.5, f=4.99e-5),
                     coriolis=dict(f=4.99e-5, mode="beta_plane", beta=2.15e-11,
                                   periodic_taper=True),
                     advection="upwind5h", buoyancy=True),
    # config-1 physics: + eyewall heating + seeded theta' noise, non-square grid
    "beta_ws5_heat": dict(nx=32, ny=24, nz=10, Lx=640e3, Ly=480e3, Lz=16e3, dt=20.0,
                          nsteps=3, vortex=dict(Vmax=50.0, Rmax=40e3, B=1.6, f=4.99e-5),
                          coriolis=dict(f=4.99e-5, mode="beta_plane", beta=2.15e-11,
                                        periodic_taper=True),
                          advection="upwind5h", buoyancy=True,
                          heating=dict(Q_max=3.0 / 3600.0, r_eyewall=40e3,
                                       width_r=math.sqrt(2.0) * 15e3, z_peak=6e3,
                                       width_z=math.sqrt(2.0) * 2e3),
                          noise_seed=20261203),
    # config-2 physics: derived β at 25N, easterly background flow
    "beta_env": dict(nx=24, ny=24, nz=8, Lx=480e3, Ly=480e3, Lz=20e3, dt=15.0, nsteps=2,
                     vortex=dict(Vmax=55.0, Rmax=30e3, B=1.8,
                                 f=2 * 7.2921e-5 * math.sin(math.radians(25.0)),
                                 u_env=-3.0),
                     coriolis=dict(f=2 * 7.2921e-5 * math.sin(math.radians(25.0)),
                                   mode="beta_plane", periodic_taper=True, u_env=-3.0),
                     advection="upwind5h", buoyancy=True),
    # divergence damper + centred advection + f-plane with background flow
    "damper_fplane": dict(nx=16, ny=16, nz=8, Lx=320e3, Ly=320e3, Lz=10e3, dt=30.0,
                          nsteps=2, vortex=dict(Vmax=30.0, Rmax=40e3, B=1.5, f=5e-5,
                                                u_env=2.0, v_env=-1.0),
                          coriolis=dict(f=5e-5, mode="f_plane", u_env=2.0, v_env=-1.0),
                          advection="centered2", buoyancy=True, damping=0.5),
    # production slow components: drag, sponge, biharmonic diffusion, Newtonian
    # cooling (production_config.py:128-150) on the beta plane, with heating
    "prod_beta": dict(nx=32, ny=24, nz=10, Lx=640e3, Ly=480e3, Lz=16e3, dt=30.0, nsteps=3,
                      vortex=dict(Vmax=45.0, Rmax=40e3, B=1.6, f=4.99e-5, u_env=-2.0,
                                  v_env=1.0),
                      coriolis=dict(f=4.99e-5, mode="beta_plane", beta=2.15e-11,
                                    periodic_taper=True, u_env=-2.0, v_env=1.0),
                      advection="upwind5h", buoyancy=True,
                      heating=dict(Q_max=3.0 / 3600.0, r_eyewall=40e3,
                                   width_r=math.sqrt(2.0) * 15e3, z_peak=6e3,
                                   width_z=math.sqrt(2.0) * 2e3),
                      drag=dict(Cd=1.5e-3, H_bl=1000.0, u_env=-2.0, v_env=1.0),
                      sponge=dict(alpha_max=0.01, sponge_fraction=0.3, u_env=-2.0, v_env=1.0),
                      hyper=3.0e12, cooling=3600.0),
    # Laplacian diffusion, drag and sponge with a background flow, f plane,
    # centred advection and the divergence damper
    "prod_lap_fplane": dict(nx=16, ny=16, nz=8, Lx=320e3, Ly=320e3, Lz=10e3, dt=30.0,
                            nsteps=2, vortex=dict(Vmax=35.0, Rmax=40e3, B=1.5, f=5e-5,
                                                  u_env=2.0, v_env=-1.0),
                            coriolis=dict(f=5e-5, mode="f_plane", u_env=2.0, v_env=-1.0),
                            advection="centered2", buoyancy=True, damping=0.5,
                            drag=dict(Cd=2.0e-3, H_bl=1500.0, u_env=2.0, v_env=-1.0),
                            sponge=dict(alpha_max=0.02, sponge_fraction=0.4, u_env=2.0,
                                        v_env=-1.0),
                            laplacian=2.0e5, cooling=1800.0),
    # projection only (the pre-balance else-branch)
    "projection_only": dict(nx=16, ny=16, nz=8, Lx=320e3, Ly=320e3, Lz=10e3, dt=1.0,
                            nsteps=2, vortex=dict(Vmax=30.0, Rmax=40e3, B=1.5, f=5e-5),
                            buoyancy=False),
}


def build_ref_config(c):
    nx, ny, nz, Lx, Ly, Lz = c["nx"], c["ny"], c["nz"], c["Lx"], c["Ly"], c["Lz"]
    kw = dict(equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
              projection=AnelasticProjection(nx, ny, nz, Lx, Ly, Lz))
    if c.get("buoyancy"):
        kw["buoyancy"] = BuoyancyComponent()
    if c.get("advection"):
        kw["advection"] = AdvectionComponent(nx, ny, nz, Lx, Ly, Lz, scheme=c["advection"])
    if c.get("coriolis"):
        ck = dict(c["coriolis"])
        if ck.get("mode") == "beta_plane":
            ck.update(Ly=Ly, ny=ny)
        kw["coriolis"] = CoriolisComponent(**ck)
    if c.get("damping") is not None:
        kw["divergence_damping"] = HelmholtzDivergenceDampingComponent(
            epsilon=c["damping"], Lx=Lx, Ly=Ly, nx=nx, ny=ny)
    if c.get("heating"):
        kw["diabatic_heating"] = DiabaticHeatingComponent(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly,
                                                          Lz=Lz, **c["heating"])
    if c.get("drag"):
        kw["surface_drag"] = SurfaceDragComponent(**c["drag"])
    if c.get("sponge"):
        kw["sponge_damping"] = SpongeDampingComponent(Lz=Lz, **c["sponge"])
    if c.get("laplacian") is not None:
        kw["horiz_diffusion"] = HorizontalDiffusionComponent(nu_H=c["laplacian"], Lx=Lx, Ly=Ly,
                                                             nx=nx, ny=ny)
    if c.get("hyper") is not None:
        kw["horiz_diffusion"] = HyperDiffusionComponent(nu4=c["hyper"], Lx=Lx, Ly=Ly,
                                                        nx=nx, ny=ny)
    if c.get("cooling") is not None:
        kw["newtonian_cooling"] = NewtonianCoolingComponent(tau=c["cooling"])
    return OperatorConfig(**kw)


def initial_state(c, base):
    v = dict(c["vortex"])
    init = LinearDecayHolland(**v, top=12_000.0)
    s = init.build_state(c["nx"], c["ny"], c["nz"], c["Lx"], c["Ly"], base)
    if c.get("noise_seed") is not None:
        rng = np.random.default_rng(c["noise_seed"])
        s.theta_prime = s.theta_prime + rng.uniform(-0.05, 0.05, (c["nx"], c["ny"], c["nz"]))
    return s


def gen_steps():
    for name, c in STEP_CASES.items():
        base = Base(c["nz"], c["Lz"])
        s = initial_state(c, base)
        out = {"config_json": np.array(json.dumps(c))}
        out.update(st_dict("s0_", s))
        integ = RK3Integrator(config=build_ref_config(c), base=base)
        for n in range(c["nsteps"]):
            s, dg = integ.step(s, dt=c["dt"], step_number=n)
            out.update(st_dict(f"s{n + 1}_", s))
            out[f"d{n + 1}"] = np.array([dg.max_u, dg.max_v, dg.max_w, dg.max_theta_prime,
                                         dg.surface_phi_min, dg.surface_phi_max])
            out[f"d{n + 1}_compat"] = np.array(dg.stage_compat_residuals, dtype=float)
            out[f"d{n + 1}_disc"] = np.array(dg.stage_disc_op_residuals, dtype=float)
        np.savez_compressed(OUT / f"steps_{name}.npz", **out)


# ---------------------------------------------------------------------------
# The production run loop (run_storm.py:120-172) on a small grid: the vortex
# with wind taper, theta' zeroed, the projection-only pre-balance, then the
# reference's build_production_config steps with the intensity cap added after
# each step.  Vmax is above the cap so the cap acts.
# ---------------------------------------------------------------------------

STORM = dict(nx=32, ny=32, nz=8, dx=PC.DX, Lz=PC.LZ, f=6.0e-5, u_env=-4.0, v_env=1.5,
             vortex=dict(Vmax=78.0, Rmax=60e3, B=1.6, R_env=220e3, wind_taper=True,
                         taper_start_frac=0.4),
             n_prebal=PC.N_PREBAL, nsteps=4, dt=PC.DT, v_cap=PC.VMAX_CAP_MS,
             tau_cap=PC.TAU_CAP)


def gen_production_storm():
    from dataclasses import replace as dc_replace
    c = STORM
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    Lx, Ly, Lz = nx * c["dx"], ny * c["dx"], c["Lz"]
    base = Base(nz, Lz)
    init = HollandVortexInit(f=c["f"], u_env=c["u_env"], v_env=c["v_env"], **c["vortex"])
    s = init.build_state(nx, ny, nz, Lx, Ly, base)
    s = dc_replace(s, theta_prime=np.zeros_like(s.theta_prime))
    out = {"config_json": np.array(json.dumps(c))}
    out.update(st_dict("s0_", s))
    pre = RK3Integrator(config=PC.build_prebal_config(nx, ny, nz, Lx, Ly, Lz), base=base)
    for i in range(c["n_prebal"]):
        s, _ = pre.step(s, dt=1.0, step_number=i)
    out.update(st_dict("pb_", s))
    integ = RK3Integrator(config=PC.build_production_config(nx, ny, nz, Lx, Ly, Lz, c["f"],
                                                            c["u_env"], c["v_env"]),
                          base=base)
    cap = IntensityCapComponent(v_cap=c["v_cap"], tau=c["tau_cap"], u_env=c["u_env"],
                                v_env=c["v_env"])
    capped = []
    for n in range(c["nsteps"]):
        s, dg = integ.step(s, dt=c["dt"], step_number=n)
        ct = cap.compute_tendency(s, None, None, base, c["dt"])
        capped.append(int(np.count_nonzero(ct.du_dt)))
        s = dc_replace(s, u=s.u + c["dt"] * ct.du_dt, v=s.v + c["dt"] * ct.dv_dt)
        out.update(st_dict(f"s{n + 1}_", s))
        out[f"d{n + 1}"] = np.array([dg.max_u, dg.max_v, dg.max_w, dg.max_theta_prime,
                                     dg.surface_phi_min, dg.surface_phi_max])
    out["capped_cells"] = np.array(capped)
    np.savez_compressed(OUT / "production_storm.npz", **out)


# ---------------------------------------------------------------------------
# Vortex diagnostics read-outs (diagnostics.py) and the sub-cell centre
# refinement of run_translation_test.py.  That module exits on import without
# CuPy, so its _subcell_refine is taken from the file with ast and run as is,
# with NumPy as its array module.
# ---------------------------------------------------------------------------

def _reference_subcell_refine():
    import ast
    path = Path(REF) / "oracle_v8" / "run_translation_test.py"
    tree = ast.parse(path.read_text())
    fn = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "_subcell_refine"]
    ns = {"xp": np, "np": np}
    exec(compile(ast.Module(body=fn, type_ignores=[]), str(path), "exec"), ns)
    return ns["_subcell_refine"]


def gen_diagnostics():
    import types
    import warnings
    from oracle_v8 import diagnostics as dg
    refine = _reference_subcell_refine()
    ps = np.load(OUT / "production_storm.npz")
    vt = np.load(OUT / "vortex_tracker.npz")
    # a deeper state: 40 levels, off-centre vortex in a background flow, noise
    nx, ny, nz, Lx, Ly, Lz = 24, 20, 40, 480e3, 400e3, 10e3
    base_c = Base(nz, Lz)
    sc = HollandVortexInit(Vmax=60.0, Rmax=30e3, B=1.7, f=5.5e-5, u_env=2.0, v_env=-1.5
                           ).build_state(nx, ny, nz, Lx, Ly, base_c, x_c=210e3, y_c=230e3)
    rng = np.random.default_rng(4242)
    cu = sc.u + 0.5 * rng.standard_normal(sc.u.shape)
    cv = sc.v + 0.5 * rng.standard_normal(sc.v.shape)
    out = {"c_u": cu, "c_v": cv}
    cases = {
        "storm": (ps["s4_u"], ps["s4_v"], 32, 32, 8, 15_625.0, 20e3, -4.0, 1.5),
        "tracker": (vt["exp_u"], vt["exp_v"], 32, 24, 8, 20e3, 16e3, -3.0, 1.0),
        "deep": (cu, cv, nx, ny, nz, 20e3, Lz, 2.0, -1.5),
    }
    res = {}
    for name, (u, v, nx_, ny_, nz_, dx, Lz_, ue, ve) in cases.items():
        st = types.SimpleNamespace(u=u, v=v, theta_prime=np.zeros_like(u))
        base = Base(nz_, Lz_)
        Lx_, Ly_ = nx_ * dx, ny_ * dx
        cx, cy = 0.47 * Lx_, 0.52 * Ly_
        calls = []

        def rec(fn, kw, val):
            calls.append(dict(fn=fn, kw=kw, out=val))

        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            kw = dict(cx_m=cx, cy_m=cy, u_env=ue, v_env=ve, theta_xy_m=[cx + 7e3, cy - 4e3],
                      r_vent_m=120e3)
            d = dg.compute_diagnostics(st, base, kw["cx_m"], kw["cy_m"], dx, dx, ue, ve,
                                       theta_xy_m=tuple(kw["theta_xy_m"]), r_vent_m=120e3)
            rec("compute_diagnostics", kw, d)
            rec("format_diag_line", kw, dg.format_diag_line(d))
            for w, zt in ((200e3, 3000.0), (100e3, 1500.0), (250e3, 6000.0), (1.0, 3000.0)):
                rec("vorticity_center", dict(cx_m=cx, cy_m=cy, window_m=w, z_top_m=zt),
                    dg.vorticity_center(st, cx, cy, dx, dx, base=base, window_m=w,
                                        z_top_m=zt))
            rec("vorticity_center", dict(cx_m=cx, cy_m=cy, window_m=200e3, z_top_m=3000.0,
                                         no_base=True),
                dg.vorticity_center(st, cx, cy, dx, dx, base=None))
            for zt in (3000.0, 500.0, 1e5):
                rec("low_level_vmax", dict(cx_m=cx, cy_m=cy, u_env=ue, v_env=ve, z_top_m=zt),
                    dg.low_level_vmax(st, base, cx, cy, dx, dx, u_env=ue, v_env=ve,
                                      z_top_m=zt))
            rec("vmax_3d", dict(u_env=ue, v_env=ve), dg.vmax_3d(st, base, u_env=ue, v_env=ve))
            for r_v, nb, c in ((150e3, 12, (cx, cy)), (80e3, 5, (cx, cy)),
                               (120e3, 12, (-1e7, -1e7)), (90e3, 7, (0.1 * Lx_, 0.9 * Ly_))):
                rec("ventilation_flow", dict(cx_m=c[0], cy_m=c[1], r_vent_m=r_v, n_bins=nb,
                                             u_env=ue, v_env=ve),
                    dg.ventilation_flow(st, c[0], c[1], dx, dx, base=base, r_vent_m=r_v,
                                        n_bins=nb, u_env=ue, v_env=ve))
            rec("ventilation_flow", dict(cx_m=cx, cy_m=cy, r_vent_m=150e3, n_bins=12,
                                         no_base=True, z_lo_m=0.0, z_hi_m=12000.0),
                dg.ventilation_flow(st, cx, cy, dx, dx, base=None))
            rec("ventilation_flow", dict(cx_m=cx, cy_m=cy, r_vent_m=150e3, n_bins=12,
                                         z_lo_m=2000.0, z_hi_m=5000.0),
                dg.ventilation_flow(st, cx, cy, dx, dx, base=base, z_lo_m=2000.0,
                                    z_hi_m=5000.0))
            rec("perturbation_ke", dict(u_env=ue, v_env=ve),
                dg.perturbation_ke(st, u_env=ue, v_env=ve))
            for zt in (3000.0, 8000.0):
                rec("enstrophy", dict(z_top_m=zt), dg.enstrophy(st, dx, dx, base=base,
                                                               z_top_m=zt))
            for (x0, y0, patch) in ((cx, cy, 9), (0.3 * dx, 0.2 * dx, 9), (cx, cy, 3),
                                    (Lx_ - 0.4 * dx, 0.5 * Ly_, 5), (float("nan"), cy, 9),
                                    (-60 * dx, cy, 9)):
                xr, yr = refine(st, x0, y0, dx, patch=patch)
                rec("subcell_refine", dict(x_m=x0, y_m=y0, patch=patch), [xr, yr])
        res[name] = dict(dx=dx, Lz=Lz_, nz=nz_, calls=calls)
    out["results_json"] = np.array(json.dumps(res))
    np.savez_compressed(OUT / "diagnostics.npz", **out)


# ---------------------------------------------------------------------------
# Vortex init and tracker fixtures
# ---------------------------------------------------------------------------

def gen_vortex_tracker():
    out = {}
    nx, ny, nz, Lx, Ly, Lz = 32, 24, 8, 640e3, 480e3, 16e3
    base = Base(nz, Lz)
    s = LinearDecayHolland(Vmax=40.0, Rmax=50e3, B=1.5, f=4.99e-5, top=12e3).build_state(
        nx, ny, nz, Lx, Ly, base)
    out.update(st_dict("lin_", s))
    s2 = HollandVortexInit(Vmax=55.0, Rmax=30e3, B=1.8, f=6.1e-5, u_env=-3.0,
                           v_env=1.0, wind_taper=True).build_state(nx, ny, nz, Lx, Ly, base,
                                                                   x_c=300e3, y_c=250e3)
    out.update(st_dict("exp_", s2))
    # tracker calls: chained first fix, a windowed fix, re-acquisition, vorticity
    # fallback and dead-reckoning
    dx = Lx / nx
    calls = [
        dict(last_pos=None, last_raw_pos=None),
        dict(last_pos=(330e3, 250e3), last_raw_pos=None),
        dict(last_pos=(500e3, 400e3), last_raw_pos=(330e3, 250e3)),
        dict(last_pos=(500e3, 400e3), last_raw_pos=None),
        dict(last_pos=(600e3, 60e3), last_raw_pos=None, u_env_ms=-3.0, v_env_ms=1.0),
        dict(last_pos=(600e3, 60e3), last_raw_pos=None),
        dict(last_pos=(460e3, 240e3), last_raw_pos=None),
        dict(last_pos=(320e3, 400e3), last_raw_pos=None),
        dict(last_pos=(200e3, 120e3), last_raw_pos=(60e3, 60e3)),
    ]
    res = []
    for kw in calls:
        (x, y), m, dg = find_storm_centre(s, base, nx, ny, dx, return_diag=True, **kw)
        res.append(dict(kw=kw, x=x, y=y, method=m, raw=list(dg["theta_raw_m"])))
    out["tracker_json"] = np.array(json.dumps(res))
    np.savez_compressed(OUT / "vortex_tracker.npz", **out)


def gen_vortex_helpers():
    """The vortex initialiser's host helpers (vortex_init.py:191-411): the
    warm-core profile, the central surface pressure deficit, the peak-wind
    check and the one-line summary, for two vortices."""
    out = []
    z = np.linspace(0.0, 20e3, 9)
    for kw in (dict(Vmax=60.0, Rmax=40e3, B=1.6, f=5e-5),
               dict(Vmax=78.0, Rmax=75e3, B=1.4, f=6e-5, R_env=500e3, wind_taper=True,
                    taper_start_frac=0.4, u_env=-3.0, v_env=1.5)):
        v = HollandVortexInit(**kw)
        out.append(dict(kw=kw, summary=v.summary(), peak=list(v.peak_wind_check()),
                        p_sfc=v.surface_pressure_deficit(1.15),
                        s_z=[float(x) for x in v.vertical_structure(z)]))
    (OUT / "vortex_helpers.json").write_text(json.dumps(out, indent=1))


# ---------------------------------------------------------------------------
# Scalar known answers of the reference's own tests
# ---------------------------------------------------------------------------

def gen_pins():
    pins = {}
    Lx, Ly, Lz = 2_000_000.0, 2_000_000.0, 20_000.0
    mms = []
    for n in (16, 32, 64):
        x = np.linspace(0, Lx, n, endpoint=False)
        y = np.linspace(0, Ly, n, endpoint=False)
        dz = Lz / n
        z = (np.arange(n) + 0.5) * dz
        X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
        phi_true, f = ana.neumann_poisson_solution(X, Y, Z, Lx, Ly, Lz, epsilon=0.1)
        rf = ana.base_state_density_periodic(z, epsilon=0.1, Lz=Lz)
        rh = np.zeros(n + 1)
        rh[1:-1] = 0.5 * (rf[:-1] + rf[1:])
        rh[0], rh[-1] = rf[0], rf[-1]
        r = VariableCoefficientPoissonSolver(n, n, n, Lx, Ly, Lz).solve(f, rf, rh)
        pc = r.phi - np.mean(r.phi)
        tc = phi_true - np.mean(phi_true)
        l2 = float(np.sqrt(np.mean((pc - tc) ** 2)) / np.sqrt(np.mean(tc ** 2)))
        mms.append(dict(n=n, l2=l2, compat=r.compatibility_residual,
                        disc=r.discrete_operator_residual))
    pins["poisson_mms"] = mms

    # warm bubble first step (test_rk3_hydrostatic_adjustment.py section A)
    from oracle_v8.validation.tests.test_hydrostatic_adjustment import (
        WarmBubbleParams, warm_bubble_theta_perturbation)
    nx = ny = 64
    nz = 32
    Lx = Ly = 100_000.0
    Lz = 10_000.0
    dz = Lz / nz
    zc = (np.arange(nz) + 0.5) * dz

    class CB:
        pass
    cb = CB()
    cb.z, cb.rho0, cb.theta0 = build_base_state(nz=nz, Lz=Lz)
    x = np.linspace(0, Lx, nx, endpoint=False)
    y = np.linspace(0, Ly, ny, endpoint=False)
    X, Y, Z = np.meshgrid(x, y, zc, indexing="ij")
    th = warm_bubble_theta_perturbation(X, Y, Z, Lx, Ly, WarmBubbleParams())
    cfg = OperatorConfig(equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
                         buoyancy=BuoyancyComponent(),
                         projection=AnelasticProjection(nx, ny, nz, Lx, Ly, Lz))
    st = State(u=np.zeros((nx, ny, nz)), v=np.zeros((nx, ny, nz)), w=np.zeros((nx, ny, nz + 1)),
               theta_prime=th, projection_potential=np.zeros((nx, ny, nz)), t=0.0)
    wb = {}
    for dt in (1.0, 5.0):
        s1, dg = RK3Integrator(config=cfg, base=cb).step(st, dt=dt, step_number=0)
        phi_c = s1.projection_potential - np.mean(s1.projection_potential)
        wb[str(dt)] = dict(phi_min=float(np.min(phi_c[:, :, 0])), max_u=dg.max_u,
                           max_w=dg.max_w, surface_phi_min=dg.surface_phi_min)
    pins["warm_bubble"] = wb
    (OUT / "pins.json").write_text(json.dumps(pins, indent=1))


# ---------------------------------------------------------------------------
# Config 0 full run (6 h, hourly tracker) — long
# ---------------------------------------------------------------------------

def gen_config0_long():
    nx = ny = 128
    nz = 32
    Lx = Ly = 2_560e3
    Lz = 16e3
    dt = 60.0
    base = Base(nz, Lz)
    c = dict(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz,
             vortex=dict(Vmax=40.0, Rmax=50e3, B=1.5, f=4.99e-5),
             coriolis=dict(f=4.99e-5, mode="beta_plane", beta=2.15e-11, periodic_taper=True),
             advection="upwind5h", buoyancy=True)
    s = initial_state(c, base)
    integ = RK3Integrator(config=build_ref_config(c), base=base)
    dx = Lx / nx
    hours = []
    last, last_raw = None, None
    out = {}
    for n in range(361):
        if n > 0:
            s, dg = integ.step(s, dt=dt, step_number=n - 1)
        if n % 60 == 0:
            (x, y), m, d = find_storm_centre(s, base, nx, ny, dx, last_pos=last,
                                             last_raw_pos=last_raw, return_diag=True)
            last, last_raw = (x, y), d["theta_raw_m"]
            hours.append(dict(h=n // 60, x=x, y=y, method=m,
                              max_u=float(np.max(np.abs(s.u))),
                              max_w=float(np.max(np.abs(s.w))),
                              max_th=float(np.max(np.abs(s.theta_prime)))))
            print("hour", n // 60, x, y, m, hours[-1]["max_w"], flush=True)
        if n == 1:
            for f, a in (("u", s.u), ("v", s.v), ("th", s.theta_prime),
                         ("phi", s.projection_potential)):
                out[f"s1_{f}_k0"] = a[:, :, 0]
                out[f"s1_{f}_k16"] = a[:, :, 16]
            out["s1_w_k1"] = s.w[:, :, 1]
            out["s1_w_k16"] = s.w[:, :, 16]
            out["s1_t"] = np.float64(s.t)
    out["final_u_k0"] = s.u[:, :, 0]
    out["final_v_k8"] = s.v[:, :, 8]
    out["final_w_k8"] = s.w[:, :, 8]
    out["final_th_k4"] = s.theta_prime[:, :, 4]
    out["final_phi_k0"] = s.projection_potential[:, :, 0]
    out["final_stats"] = np.array([[f.mean(), np.sqrt(np.mean(f ** 2)), np.abs(f).max()]
                                   for f in (s.u, s.v, s.w, s.theta_prime,
                                             s.projection_potential)])
    out["hours_json"] = np.array(json.dumps(hours))
    np.savez_compressed(OUT / "config0_6h.npz", **out)


# ---------------------------------------------------------------------------
# Blow-up of the LH82 physics: config-1 parameters (dx 5 km, dz 250 m,
# beta-plane at 20N, Holland 50 m/s / 40 km / 1.6 with the 12-km linear wind
# decay, eyewall heating, seeded theta' noise, dt 20 s) on a 96 x 96 x 64
# grid, stepped by the reference until max|u| exceeds 400 m/s or is not
# finite (the test of measure_lh82_phase3.py:129-130).  Every step's max|u|
# and max|w| are kept.  About 12 minutes on one core (--blowup).
# ---------------------------------------------------------------------------

BLOWUP = dict(nx=96, ny=96, nz=64, Lx=96 * 5e3, Ly=96 * 5e3, Lz=16e3, dt=20.0,
              vortex=dict(Vmax=50.0, Rmax=40e3, B=1.6, f=4.99e-5),
              coriolis=dict(f=4.99e-5, mode="beta_plane", beta=2.15e-11, periodic_taper=True),
              advection="upwind5h", buoyancy=True,
              heating=dict(Q_max=3.0 / 3600.0, r_eyewall=40e3, width_r=math.sqrt(2.0) * 15e3,
                           z_peak=6e3, width_z=math.sqrt(2.0) * 2e3),
              noise_seed=20261203, max_steps=800)


def gen_blowup():
    c = BLOWUP
    base = Base(c["nz"], c["Lz"])
    s = initial_state(c, base)
    integ = RK3Integrator(config=build_ref_config(c), base=base)
    mu, mw = [], []
    blew = -1
    for n in range(c["max_steps"]):
        s, dg = integ.step(s, dt=c["dt"], step_number=n)
        mu.append(float(dg.max_u))
        mw.append(float(dg.max_w))
        if n % 50 == 0:
            print("step", n, mu[-1], mw[-1], flush=True)
        if not math.isfinite(mu[-1]) or mu[-1] > 400.0:
            blew = n
            break
    np.savez_compressed(OUT / "blowup_lh82.npz", config_json=np.array(json.dumps(c)),
                        max_u=np.array(mu), max_w=np.array(mw), blew_step=np.int64(blew))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--long", action="store_true")
    ap.add_argument("--reference", default=None, help="root of the reference tree (read above)")
    ap.add_argument("--only", default=None)
    ap.add_argument("--blowup", action="store_true")
    a = ap.parse_args()
    jobs = dict(components=gen_components, production=gen_production, steps=gen_steps,
                production_storm=gen_production_storm, diagnostics=gen_diagnostics,
                vortex_helpers=gen_vortex_helpers,
                vortex_tracker=gen_vortex_tracker, pins=gen_pins)
    for k, f in jobs.items():
        if a.only and k != a.only:
            continue
        f()
        print("wrote", k, flush=True)
    if a.long:
        gen_config0_long()
        print("wrote config0_6h", flush=True)
    if a.blowup:
        gen_blowup()
        print("wrote blowup_lh82", flush=True)
