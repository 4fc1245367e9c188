"""FP64 parity of the sm_100a kernels with the reference (golden fixtures made by
the unmodified reference) and with the oracle on fresh seeded inputs.

Bar: each tendency, the projected velocity and every state field within
1e-12 of the reference, relative to the field's max |.|.
"""
import json
import math

import numpy as np
import pytest
import torch

from oracle import lh82 as O
from tests.gpu_helpers import TOL64, Base, b200_config, dev, host, load_case, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def comp(golden_dir):
    return np.load(golden_dir / "components.npz")


@pytest.fixture(scope="module")
def cstate(comp):
    from oraclev8_b200.solver import State
    g = comp
    return State(dev(g["in_u"]), dev(g["in_v"]), dev(g["in_w"]), dev(g["in_th"]),
                 dev(g["in_phi"]), 0.0)


def _grid(g):
    return (int(g["nx"]), int(g["ny"]), int(g["nz"]), float(g["Lx"]), float(g["Ly"]),
            float(g["Lz"]))


def test_buoyancy_component(comp, cstate):
    from oraclev8_b200.solver import BuoyancyComponent, LH82AnelasticEquationSet
    from oraclev8_b200.grid import LorenzStaggering
    base = Base(int(comp["nz"]), float(comp["Lz"]))
    t = BuoyancyComponent().compute_tendency(cstate, LH82AnelasticEquationSet(),
                                             LorenzStaggering(), base, 1.0)
    assert rel(t.dw_dt, comp["buoy_dw"]) <= 1e-15
    assert float(host(t.dw_dt)[..., 0].max()) == 0.0 and float(host(t.dw_dt)[..., -1].max()) == 0.0


@pytest.mark.parametrize("scheme", ["upwind5h", "centered2"])
def test_advection_component(comp, cstate, scheme):
    from oraclev8_b200.solver import AdvectionComponent
    nx, ny, nz, Lx, Ly, Lz = _grid(comp)
    base = Base(nz, Lz)
    t = AdvectionComponent(nx, ny, nz, Lx, Ly, Lz, scheme=scheme).compute_tendency(
        cstate, None, None, base, 30.0)
    for name, got in (("du", t.du_dt), ("dv", t.dv_dt), ("dw", t.dw_dt), ("dth", t.dtheta_prime_dt)):
        assert rel(got, comp[f"adv_{scheme}_{name}"]) <= TOL64, name


def test_coriolis_components(comp, cstate):
    from oraclev8_b200.solver import CoriolisComponent
    nx, ny, nz, Lx, Ly, Lz = _grid(comp)
    base = Base(nz, Lz)
    cases = {
        "fplane": CoriolisComponent(f=5e-5, mode="f_plane", u_env=1.5, v_env=-0.5),
        "beta_taper": CoriolisComponent(f=4.99e-5, mode="beta_plane", beta=2.15e-11, Ly=Ly,
                                        ny=ny, periodic_taper=True),
        "beta_derived": CoriolisComponent(f=6.164e-5, mode="beta_plane", Ly=Ly, ny=ny,
                                          u_env=-3.0),
    }
    for k, c in cases.items():
        t = c.compute_tendency(cstate, None, None, base, 30.0)
        assert rel(t.du_dt, comp[f"cor_{k}_du"]) <= 1e-15, k
        assert rel(t.dv_dt, comp[f"cor_{k}_dv"]) <= 1e-15, k


def test_heating_and_damper(comp, cstate):
    from oraclev8_b200.solver import (DiabaticHeatingComponent,
                                      HelmholtzDivergenceDampingComponent)
    nx, ny, nz, Lx, Ly, Lz = _grid(comp)
    base = Base(nz, Lz)
    h = DiabaticHeatingComponent(Q_max=3.0 / 3600.0, r_eyewall=40e3,
                                 width_r=math.sqrt(2.0) * 15e3, z_peak=2e3,
                                 width_z=math.sqrt(2.0) * 1e3, nx=nx, ny=ny, nz=nz, Lx=Lx,
                                 Ly=Ly, Lz=Lz)
    t = h.compute_tendency(cstate, None, None, base, 30.0)
    assert np.array_equal(host(t.dtheta_prime_dt), comp["heat_dth"])
    d = HelmholtzDivergenceDampingComponent(epsilon=0.5, Lx=Lx, Ly=Ly, nx=nx, ny=ny)
    t = d.compute_tendency(cstate, None, None, base, 30.0)
    assert rel(t.du_dt, comp["helm_du"]) <= TOL64
    assert rel(t.dv_dt, comp["helm_dv"]) <= TOL64


def test_operators_divergence_gradient(comp, cstate):
    from oraclev8_b200.solver.tendency import _phi_gradient, anelastic_divergence
    nx, ny, nz, Lx, Ly, Lz = _grid(comp)
    rf = comp["rho0"]
    rh = O.rho_half_levels(rf)
    kx, ky = O.wavenumbers(nx, ny, Lx, Ly)
    d = anelastic_divergence(cstate.u, cstate.v, cstate.w, rf, rh, kx, ky, Lz / nz)
    assert rel(d, comp["div"]) <= TOL64
    gx, gy, gz = _phi_gradient(cstate.projection_potential, kx, ky, Lz / nz)
    assert rel(gx, comp["grad_x"]) <= TOL64
    assert rel(gy, comp["grad_y"]) <= TOL64
    assert rel(gz, comp["grad_z"]) <= TOL64


def test_poisson_solve_and_operator(comp):
    from oraclev8_b200.solver import VariableCoefficientPoissonSolver
    nx, ny, nz, Lx, Ly, Lz = _grid(comp)
    rf = comp["rho0"]
    rh = O.rho_half_levels(rf)
    s = VariableCoefficientPoissonSolver(nx, ny, nz, Lx, Ly, Lz)
    r = s.solve(dev(comp["div"]), rf, rh, log_diagnostics=True)
    assert rel(r.phi, comp["solve_phi"]) <= TOL64
    assert r.compatibility_residual < 1e-8 and r.discrete_operator_residual < 1e-6
    op = s.apply_operator(dev(comp["in_phi"]), rf, rh)
    assert rel(op, comp["apply_op"]) <= TOL64


def test_projection(comp, cstate):
    from oraclev8_b200.solver import AnelasticProjection, State
    nx, ny, nz, Lx, Ly, Lz = _grid(comp)
    base = Base(nz, Lz)
    st = State(cstate.u.clone(), cstate.v.clone(), cstate.w.clone(),
               cstate.theta_prime.clone(), cstate.projection_potential.clone(), 0.0)
    AnelasticProjection(nx, ny, nz, Lx, Ly, Lz).apply_projection(st, None, None, base, 1.0)
    for f, k in (("u", "u"), ("v", "v"), ("w", "w"), ("projection_potential", "phi")):
        assert rel(getattr(st, f), comp["proj_" + k]) <= TOL64, f


STEP_CASES = ["beta_ws5", "beta_ws5_heat", "beta_env", "damper_fplane", "projection_only"]


@pytest.mark.parametrize("case", STEP_CASES)
def test_rk3_steps_match_reference(golden_dir, case):
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
            e = rel(getattr(s, f), g[f"s{n + 1}_{k}"])
            assert e <= TOL64, (case, n, f, e)
        assert s.t == float(g[f"s{n + 1}_t"])
        d = np.array([dg.max_u, dg.max_v, dg.max_w, dg.max_theta_prime, dg.surface_phi_min,
                      dg.surface_phi_max])
        ref = g[f"d{n + 1}"]
        assert np.all(np.abs(d - ref) <= 1e-11 * np.maximum(np.abs(ref), 1e-30)), (d, ref)


def _seeded_state(rng, nx, ny, nz, zero_w_ends=True):
    u = 10.0 * rng.standard_normal((nx, ny, nz))
    v = 10.0 * rng.standard_normal((nx, ny, nz))
    w = 0.3 * rng.standard_normal((nx, ny, nz + 1))
    if zero_w_ends:
        w[:, :, 0] = 0.0
        w[:, :, -1] = 0.0
    th = 1.5 * rng.standard_normal((nx, ny, nz))
    return O.State(u, v, w, th, np.zeros((nx, ny, nz)), 0.0)


@pytest.mark.parametrize("shape", [(24, 20, 6), (96, 64, 7), (40, 30, 5), (8, 12, 3)])
def test_projection_vs_oracle_mixed_radix(shape):
    """Odd nz, radix 3 and 5 lengths, odd-chunked z: GPU projection == oracle."""
    from oraclev8_b200.solver import AnelasticProjection, State
    nx, ny, nz = shape
    Lx, Ly, Lz = nx * 15e3, ny * 12e3, 9e3
    rng = np.random.default_rng(nx * 1000 + ny * 10 + nz)
    s = _seeded_state(rng, nx, ny, nz, zero_w_ends=False)
    z, rho0, th0 = O.build_base_state(nz, Lz)
    ref = O.Projection(nx, ny, nz, Lx, Ly, Lz).apply(s.copy(), rho0)
    base = Base(nz, Lz)
    st = State(dev(s.u), dev(s.v), dev(s.w), dev(s.theta_prime), dev(s.projection_potential), 0.0)
    AnelasticProjection(nx, ny, nz, Lx, Ly, Lz).apply_projection(st, None, None, base, 1.0)
    for f in ("u", "v", "w", "projection_potential"):
        assert rel(getattr(st, f), getattr(ref, f)) <= TOL64, (shape, f)


def test_step_vs_oracle_fresh_inputs():
    """A different grid from the fixtures (non-square, radix 3), two steps,
    full config-1 component set."""
    from oraclev8_b200.solver import RK3Integrator, State
    c = dict(nx=48, ny=36, nz=12, Lx=48 * 10e3, Ly=36 * 10e3, Lz=16e3, dt=30.0,
             vortex=dict(Vmax=45.0, Rmax=40e3, B=1.4, f=5.5e-5),
             coriolis=dict(f=5.5e-5, mode="beta_plane", beta=2.1e-11, periodic_taper=True),
             advection="upwind5h", buoyancy=True,
             heating=dict(Q_max=3.0 / 3600.0, r_eyewall=40e3, width_r=math.sqrt(2.0) * 15e3,
                          z_peak=6e3, width_z=math.sqrt(2.0) * 2e3), noise_seed=7)
    from tests.test_oracle_golden import oracle_config, oracle_initial_state
    s, (z, rho0, th0) = oracle_initial_state(c)
    integ_o = O.Integrator(oracle_config(c), z, rho0, th0)
    base = Base(c["nz"], c["Lz"])
    integ = RK3Integrator(b200_config(c), base, precision="fp64")
    sg = State(dev(s.u), dev(s.v), dev(s.w), dev(s.theta_prime), dev(s.projection_potential), 0.0)
    for n in range(2):
        s, _ = integ_o.step(s, c["dt"], n)
        sg, _ = integ.step(sg, c["dt"], n)
        for f in ("u", "v", "w", "theta_prime", "projection_potential"):
            assert rel(getattr(sg, f), getattr(s, f)) <= TOL64, (n, f)


def test_reference_known_answers_on_gpu(golden_dir):
    """Warm-bubble first step (test_rk3_hydrostatic_adjustment.py:178): phi_min
    = -64.843 Pa per second of dt; Poisson MMS second-order convergence."""
    from oraclev8_b200.solver import (AnelasticProjection, BuoyancyComponent,
                                      LH82AnelasticEquationSet, OperatorConfig, RK3Integrator,
                                      State, VariableCoefficientPoissonSolver)
    from oraclev8_b200.grid import LorenzStaggering
    pins = json.loads((golden_dir / "pins.json").read_text())
    nx = ny = 64
    nz = 32
    Lx = Ly = 100_000.0
    Lz = 10_000.0
    base = Base(nz, Lz)
    x = np.linspace(0, Lx, nx, endpoint=False)
    y = np.linspace(0, Ly, ny, endpoint=False)
    X, Y, Z = np.meshgrid(x, y, base.z, indexing="ij")
    L_ = np.sqrt(((X - Lx / 2) / 10e3) ** 2 + ((Y - Ly / 2) / 10e3) ** 2 + ((Z - 2e3) / 2e3) ** 2)
    th = np.where(L_ <= 1.0, 2.0 * np.cos(np.pi * L_ / 2.0) ** 2, 0.0)
    cfg = OperatorConfig(equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
                         buoyancy=BuoyancyComponent(),
                         projection=AnelasticProjection(nx, ny, nz, Lx, Ly, Lz))
    for dt in (1.0, 5.0):
        st = State(dev(np.zeros((nx, ny, nz))), dev(np.zeros((nx, ny, nz))),
                   dev(np.zeros((nx, ny, nz + 1))), dev(th), dev(np.zeros((nx, ny, nz))), 0.0)
        s1, dg = RK3Integrator(cfg, base, precision="fp64").step(st, dt, 0)
        ref = pins["warm_bubble"][str(dt)]
        assert dg.surface_phi_min == pytest.approx(ref["surface_phi_min"], rel=1e-11)
        assert dg.max_w == pytest.approx(ref["max_w"], rel=1e-11)
    assert pins["warm_bubble"]["1.0"]["phi_min"] == pytest.approx(-64.843, abs=0.01)
    # MMS convergence (test_poisson_solver.py:52-113)
    Lx = Ly = 2_000_000.0
    Lz = 20_000.0
    l2 = []
    for row in pins["poisson_mms"]:
        n = row["n"]
        x = np.linspace(0, Lx, n, endpoint=False)
        zc = (np.arange(n) + 0.5) * (Lz / n)
        X, Y, Z = np.meshgrid(x, x, zc, indexing="ij")
        kx, kz = 2 * np.pi / Lx, np.pi / Lz
        phi_t = np.sin(2 * np.pi * X / Lx) * np.sin(2 * np.pi * Y / Ly) * np.cos(np.pi * Z / Lz)
        rho = 1.225 * (1.0 + 0.1 * np.cos(2.0 * np.pi * Z / Lz))
        f = rho * (-(2 * kx ** 2 + kz ** 2) * phi_t) + (
            -1.225 * 0.1 * (2.0 * np.pi / Lz) * np.sin(2.0 * np.pi * Z / Lz)) * (
            -kz * np.sin(kx * X) * np.sin(kx * Y) * np.sin(kz * Z))
        rf = 1.225 * (1.0 + 0.1 * np.cos(2.0 * np.pi * zc / Lz))
        r = VariableCoefficientPoissonSolver(n, n, n, Lx, Ly, Lz).solve(
            dev(f), rf, O.rho_half_levels(rf), log_diagnostics=True)
        phi = host(r.phi)
        pc, tc = phi - phi.mean(), phi_t - phi_t.mean()
        e = float(np.sqrt(np.mean((pc - tc) ** 2)) / np.sqrt(np.mean(tc ** 2)))
        assert e == pytest.approx(row["l2"], rel=1e-9)
        assert r.compatibility_residual < 1e-8 and r.discrete_operator_residual < 1e-6
        l2.append(e)
    assert l2[0] / l2[1] > 3.0 and l2[1] / l2[2] > 3.0


def test_zero_source_gives_zero_phi():
    """test_poisson_solver.py:116-148: d = 0 -> phi = 0 exactly."""
    from oraclev8_b200.solver import VariableCoefficientPoissonSolver
    n = 16
    rf = 1.225 * (1.0 + 0.1 * np.cos(2 * np.pi * (np.arange(n) + 0.5) / n))
    r = VariableCoefficientPoissonSolver(n, n, n, 2e6, 2e6, 2e4).solve(
        dev(np.zeros((n, n, n))), rf, O.rho_half_levels(rf))
    assert float(host(r.phi).__abs__().max()) < 1e-12


def test_projection_properties_large():
    """Size-independent properties at a production-like size: after the
    projection the divergence is at round-off outside the Nyquist rows (the
    reference's spectral gradient drops the Nyquist derivative), the
    projection is idempotent, and the dead fast stages leave stage 3 equal to
    P(u_n, v_n, w_n + dt b(theta'_n))."""
    from oraclev8_b200._plan import Plan, PlanSpec
    nx, ny, nz = 256, 192, 32
    Lx, Ly, Lz = nx * 5e3, ny * 5e3, 16e3
    z, rho0, th0 = O.build_base_state(nz, Lz)
    p = Plan(PlanSpec(nx, ny, nz, Lx, Ly, Lz, rho0, th0, projection=True))
    rng = np.random.default_rng(5)
    s = _seeded_state(rng, nx, ny, nz)
    u, v, w, phi = dev(s.u), dev(s.v), dev(s.w), dev(np.zeros((nx, ny, nz)))
    d0 = host(p.divergence(u, v, w))
    p.project(u, v, w, phi)
    d1 = p.divergence(u, v, w)
    dh = np.fft.fft2(host(d1), axes=(0, 1))
    dh[nx // 2, :, :] = 0
    dh[:, ny // 2, :] = 0
    assert np.max(np.abs(np.real(np.fft.ifft2(dh, axes=(0, 1))))) <= 1e-12 * np.max(np.abs(d0))
    # idempotence outside the Nyquist rows: a second projection only moves the
    # Nyquist modes, which no projection can make divergence-free
    u2, v2, w2, phi2 = u.clone(), v.clone(), w.clone(), torch.empty_like(phi)
    p.project(u2, v2, w2, phi2)

    def non_nyquist(a):
        ah = np.fft.fft2(a, axes=(0, 1))
        ah[nx // 2, :, :] = 0
        ah[:, ny // 2, :] = 0
        return np.real(np.fft.ifft2(ah, axes=(0, 1)))

    du = non_nyquist(host(u2) - host(u))
    assert np.max(np.abs(du)) <= 1e-12 * float(torch.max(torch.abs(u)))


def test_dead_fast_stages():
    """With buoyancy the only fast component, stages 1 and 2 do not reach the
    result: the step equals P(u_n, v_n, w_n + dt b(theta'_n)) (integrator.py:461-500)."""
    from oraclev8_b200._plan import Plan, PlanSpec
    from oraclev8_b200.solver import (AnelasticProjection, BuoyancyComponent,
                                      LH82AnelasticEquationSet, OperatorConfig, RK3Integrator,
                                      State)
    from oraclev8_b200.grid import LorenzStaggering
    nx, ny, nz = 64, 48, 16
    Lx, Ly, Lz = nx * 10e3, ny * 10e3, 16e3
    base = Base(nz, Lz)
    rng = np.random.default_rng(11)
    s = _seeded_state(rng, nx, ny, nz)
    cfg = OperatorConfig(equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
                         buoyancy=BuoyancyComponent(),
                         projection=AnelasticProjection(nx, ny, nz, Lx, Ly, Lz))
    st = State(dev(s.u), dev(s.v), dev(s.w), dev(s.theta_prime), dev(s.projection_potential), 0.0)
    out, _ = RK3Integrator(cfg, base, precision="fp64").step(st, 45.0, 0)
    p = Plan(PlanSpec(nx, ny, nz, Lx, Ly, Lz, base.rho0, base.theta0, projection=True))
    b = p.buoyancy(dev(s.theta_prime))
    u, v, w = dev(s.u), dev(s.v), dev(s.w) + 45.0 * b
    phi = torch.empty_like(u)
    p.project(u, v, w, phi)
    for a, r in ((out.u, u), (out.v, v), (out.w, w), (out.projection_potential, phi)):
        assert rel(a, host(r)) <= 1e-13
