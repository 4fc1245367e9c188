"""Pin the NumPy oracle against fixtures produced by the unmodified reference.

The oracle restates the reference op for op, so every comparison here is
exact (bit-for-bit) or within a few ulps where NumPy's pairwise sums meet a
different array shape.  Scalar known answers come from the reference's own
tests (validation/tests/test_poisson_solver.py:52-221 and
test_rk3_hydrostatic_adjustment.py:178,277,343).
"""
import json
import math

import numpy as np
import pytest

from oracle import lh82 as O

TIGHT = 1e-14  # relative to the field's max magnitude


def rel(a, b):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) / scale


@pytest.fixture(scope="module")
def comp(golden_dir):
    return np.load(golden_dir / "components.npz")


def _state(g, p):
    return O.State(g[p + "u"].copy(), g[p + "v"].copy(), g[p + "w"].copy(),
                   g[p + "th"].copy(), g[p + "phi"].copy(), float(g[p + "t"]))


def test_base_state_matches(comp):
    z, r, t = O.build_base_state(int(comp["nz"]), float(comp["Lz"]))
    assert np.array_equal(z, comp["z"])
    assert np.array_equal(r, comp["rho0"])
    assert np.array_equal(t, comp["theta0"])


def test_component_tendencies(comp):
    g = comp
    s = _state(g, "in_")
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    Lx, Ly, Lz = float(g["Lx"]), float(g["Ly"]), float(g["Lz"])
    th0 = g["theta0"]
    assert np.array_equal(O.buoyancy_half(s.theta_prime, th0), g["buoy_dw"])
    for scheme in ("upwind5h", "centered2"):
        out = O.advection_tendency(s.u, s.v, s.w, s.theta_prime, th0, Lx / nx, Ly / ny,
                                   Lz / nz, scheme)
        for name, a in zip(("du", "dv", "dw", "dth"), out):
            assert np.array_equal(a, g[f"adv_{scheme}_{name}"]), (scheme, name)
    fy = O.coriolis_profile(5e-5, "f_plane")
    du, dv = O.coriolis_tendency(s.u, s.v, 5e-5, fy, 1.5, -0.5)
    assert np.array_equal(du, g["cor_fplane_du"]) and np.array_equal(dv, g["cor_fplane_dv"])
    fy = O.coriolis_profile(4.99e-5, "beta_plane", 2.15e-11, Ly, ny, None, True)
    du, dv = O.coriolis_tendency(s.u, s.v, 4.99e-5, fy)
    assert np.array_equal(du, g["cor_beta_taper_du"]) and np.array_equal(dv, g["cor_beta_taper_dv"])
    fy = O.coriolis_profile(6.164e-5, "beta_plane", None, Ly, ny, None, False)
    du, dv = O.coriolis_tendency(s.u, s.v, 6.164e-5, fy, -3.0, 0.0)
    assert np.array_equal(du, g["cor_beta_derived_du"])
    assert np.array_equal(dv, g["cor_beta_derived_dv"])
    q = O.heating_field(3.0 / 3600.0, 40e3, math.sqrt(2.0) * 15e3, 2e3, math.sqrt(2.0) * 1e3,
                        nx, ny, nz, Lx, Ly, Lz)
    assert np.array_equal(q, g["heat_dth"])
    hu, hv = O.helmholtz_tendency(s.u, s.v, 0.5, 30.0, Lx, Ly)
    assert np.array_equal(hu, g["helm_du"]) and np.array_equal(hv, g["helm_dv"])


def test_operators_and_solve(comp):
    g = comp
    s = _state(g, "in_")
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    Lx, Ly, Lz = float(g["Lx"]), float(g["Ly"]), float(g["Lz"])
    rf = g["rho0"]
    rh = O.rho_half_levels(rf)
    kx, ky = O.wavenumbers(nx, ny, Lx, Ly)
    d = O.anelastic_divergence(s.u, s.v, s.w, rf, rh, kx, ky, Lz / nz)
    assert np.array_equal(d, g["div"])
    gx, gy, gz = O.phi_gradient(s.projection_potential, kx, ky, Lz / nz)
    assert np.array_equal(gx, g["grad_x"]) and np.array_equal(gy, g["grad_y"])
    assert np.array_equal(gz, g["grad_z"])
    P = O.Poisson(nx, ny, nz, Lx, Ly, Lz)
    phi, compat, disc = P.solve(d, rf, rh, log_diagnostics=True)
    assert np.array_equal(phi, g["solve_phi"])
    assert compat == float(g["solve_compat"]) and disc == float(g["solve_disc"])
    assert np.array_equal(P.apply_operator(s.projection_potential, rf, rh), g["apply_op"])
    pr = O.Projection(nx, ny, nz, Lx, Ly, Lz)
    s2 = pr.apply(s.copy(), rf)
    for f, k in (("u", "u"), ("v", "v"), ("w", "w"), ("projection_potential", "phi")):
        assert np.array_equal(getattr(s2, f), g["proj_" + k]), f


STEP_CASES = ["beta_ws5", "beta_ws5_heat", "beta_env", "damper_fplane", "projection_only",
              "prod_beta", "prod_lap_fplane"]


def oracle_config(c):
    cor = None
    if c.get("coriolis"):
        cor = dict(c["coriolis"])
        if cor.get("mode") == "beta_plane":
            cor.update(Ly=c["Ly"], ny=c["ny"])
    return O.StepConfig(nx=c["nx"], ny=c["ny"], nz=c["nz"], Lx=c["Lx"], Ly=c["Ly"],
                        Lz=c["Lz"], buoyancy=bool(c.get("buoyancy")),
                        advection=c.get("advection"), coriolis=cor,
                        damping_epsilon=c.get("damping"), heating=c.get("heating"),
                        drag=c.get("drag"), sponge=c.get("sponge"),
                        laplacian=c.get("laplacian"), hyper=c.get("hyper"),
                        cooling=c.get("cooling"))


def oracle_initial_state(c):
    z, rho0, th0 = O.build_base_state(c["nz"], c["Lz"])
    v = dict(c["vortex"])
    s = O.Holland(**v, wind_decay_top=12_000.0).build_state(
        c["nx"], c["ny"], c["nz"], c["Lx"], c["Ly"], z, rho0, th0)
    if c.get("noise_seed") is not None:
        rng = np.random.default_rng(c["noise_seed"])
        s.theta_prime = s.theta_prime + rng.uniform(-0.05, 0.05, (c["nx"], c["ny"], c["nz"]))
    return s, (z, rho0, th0)


@pytest.mark.parametrize("case", STEP_CASES)
def test_rk3_steps_match_reference(golden_dir, case):
    g = np.load(golden_dir / f"steps_{case}.npz")
    c = json.loads(str(g["config_json"]))
    s, (z, rho0, th0) = oracle_initial_state(c)
    s0 = _state(g, "s0_")
    for f in ("u", "v", "w", "theta_prime"):
        assert np.array_equal(getattr(s, f), getattr(s0, f)), f
    integ = O.Integrator(oracle_config(c), z, rho0, th0)
    for n in range(c["nsteps"]):
        s, dg = integ.step(s, c["dt"], step_number=n)
        ref = _state(g, f"s{n + 1}_")
        for f in ("u", "v", "w", "theta_prime", "projection_potential"):
            assert rel(getattr(s, f), getattr(ref, f)) <= TIGHT, (case, n, f)
        assert s.t == ref.t
        d = np.array([dg.max_u, dg.max_v, dg.max_w, dg.max_theta_prime,
                      dg.surface_phi_min, dg.surface_phi_max])
        np.testing.assert_allclose(d, g[f"d{n + 1}"], rtol=1e-13, atol=0)


def test_production_run_loop(golden_dir):
    """The reference's production run loop (run_storm.py:120-172): tapered
    vortex with theta' zeroed, projection-only pre-balance, then
    build_production_config steps (production_config.py:128-150) with the
    intensity cap added after each step."""
    g = np.load(golden_dir / "production_storm.npz")
    c = json.loads(str(g["config_json"]))
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    Lx, Ly, Lz = nx * c["dx"], ny * c["dx"], c["Lz"]
    z, rho0, th0 = O.build_base_state(nz, Lz)
    s = O.Holland(f=c["f"], u_env=c["u_env"], v_env=c["v_env"], **c["vortex"]).build_state(
        nx, ny, nz, Lx, Ly, z, rho0, th0)
    s.theta_prime = np.zeros_like(s.theta_prime)
    ref = _state(g, "s0_")
    for f in ("u", "v", "w", "theta_prime"):
        assert rel(getattr(s, f), getattr(ref, f)) <= TIGHT, f
    pre = O.Integrator(O.StepConfig(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz, buoyancy=False,
                                    advection=None), z, rho0, th0)
    for i in range(c["n_prebal"]):
        s, _ = pre.step(s, 1.0, step_number=i)
    ref = _state(g, "pb_")
    for f in ("u", "v", "w", "theta_prime", "projection_potential"):
        assert rel(getattr(s, f), getattr(ref, f)) <= TIGHT, ("prebal", f)
    cfg = O.StepConfig(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz, buoyancy=False,
                       advection="centered2",
                       coriolis=dict(f=c["f"], mode="beta_plane", Ly=Ly, ny=ny,
                                     u_env=c["u_env"], v_env=c["v_env"], periodic_taper=True),
                       damping_epsilon=0.5, hyper=3.0e11, cooling=1800.0,
                       drag=dict(Cd=1.5e-3, H_bl=1000.0, u_env=c["u_env"], v_env=c["v_env"]))
    integ = O.Integrator(cfg, z, rho0, th0)
    for n in range(c["nsteps"]):
        s, dg = integ.step(s, c["dt"], step_number=n)
        du, dv = O.intensity_cap_tendency(s.u, s.v, c["v_cap"], c["tau_cap"], c["u_env"],
                                          c["v_env"])
        assert np.count_nonzero(du) == g["capped_cells"][n]
        s.u = s.u + c["dt"] * du
        s.v = s.v + c["dt"] * dv
        ref = _state(g, f"s{n + 1}_")
        for f in ("u", "v", "w", "theta_prime", "projection_potential"):
            assert rel(getattr(s, f), getattr(ref, f)) <= TIGHT, (n, f)
        d = np.array([dg.max_u, dg.max_v, dg.max_w, dg.max_theta_prime,
                      dg.surface_phi_min, dg.surface_phi_max])
        np.testing.assert_allclose(d, g[f"d{n + 1}"], rtol=1e-13, atol=0)


def test_vortex_init_and_tracker(golden_dir):
    g = np.load(golden_dir / "vortex_tracker.npz")
    nx, ny, nz, Lx, Ly, Lz = 32, 24, 8, 640e3, 480e3, 16e3
    z, rho0, th0 = O.build_base_state(nz, Lz)
    s = O.Holland(40.0, 50e3, 1.5, 4.99e-5, wind_decay_top=12e3).build_state(
        nx, ny, nz, Lx, Ly, z, rho0, th0)
    for f, k in (("u", "u"), ("v", "v"), ("w", "w"), ("theta_prime", "th")):
        assert np.array_equal(getattr(s, f), g["lin_" + k]), f
    s2 = O.Holland(55.0, 30e3, 1.8, 6.1e-5, u_env=-3.0, v_env=1.0, wind_taper=True).build_state(
        nx, ny, nz, Lx, Ly, z, rho0, th0, x_c=300e3, y_c=250e3)
    for f, k in (("u", "u"), ("v", "v"), ("theta_prime", "th")):
        assert np.array_equal(getattr(s2, f), g["exp_" + k]), f
    dx = Lx / nx
    for r in json.loads(str(g["tracker_json"])):
        kw = dict(r["kw"])
        for k in ("last_pos", "last_raw_pos"):
            if kw.get(k) is not None:
                kw[k] = tuple(kw[k])
        (x, y), m, raw = O.find_storm_centre(s, z, rho0, th0, nx, ny, dx, **kw)
        assert m == r["method"]
        assert (x, y) == (r["x"], r["y"])
        assert list(raw) == r["raw"]


def test_reference_known_answers(golden_dir):
    """Scalar pins of the reference's own tests, reproduced by the oracle."""
    pins = json.loads((golden_dir / "pins.json").read_text())
    # Poisson MMS second-order convergence (test_poisson_solver.py:52-113)
    Lx = Ly = 2_000_000.0
    Lz = 20_000.0
    l2s = []
    for row in pins["poisson_mms"][:2]:
        n = row["n"]
        x = np.linspace(0, Lx, n, endpoint=False)
        y = np.linspace(0, Ly, n, endpoint=False)
        zc = (np.arange(n) + 0.5) * (Lz / n)
        X, Y, Z = np.meshgrid(x, y, zc, indexing="ij")
        kx, ky, kz = 2 * np.pi / Lx, 2 * np.pi / Ly, np.pi / Lz
        phi_t = np.sin(2.0 * np.pi * X / Lx) * np.sin(2.0 * np.pi * Y / Ly) * np.cos(np.pi * Z / Lz)
        rho = 1.225 * (1.0 + 0.1 * np.cos(2.0 * np.pi * Z / Lz))
        lap = -(kx ** 2 + ky ** 2 + kz ** 2) * phi_t
        dphi = -kz * np.sin(kx * X) * np.sin(ky * Y) * np.sin(kz * Z)
        drho = -1.225 * 0.1 * (2.0 * np.pi / Lz) * np.sin(2.0 * np.pi * Z / Lz)
        f = rho * lap + drho * dphi
        rf = 1.225 * (1.0 + 0.1 * np.cos(2.0 * np.pi * zc / Lz))
        rh = O.rho_half_levels(rf)
        phi, compat, disc = O.Poisson(n, n, n, Lx, Ly, Lz).solve(f, rf, rh, True)
        pc, tc = phi - phi.mean(), phi_t - phi_t.mean()
        l2 = float(np.sqrt(np.mean((pc - tc) ** 2)) / np.sqrt(np.mean(tc ** 2)))
        assert l2 == pytest.approx(row["l2"], rel=1e-12)
        assert compat < 1e-8 and disc < 1e-6
        l2s.append(l2)
    assert l2s[0] / l2s[1] > 3.0
    assert pins["poisson_mms"][0]["l2"] == pytest.approx(2.191e-3, abs=1e-6)
    assert pins["warm_bubble"]["1.0"]["phi_min"] == pytest.approx(-64.843, abs=0.01)
    assert pins["warm_bubble"]["5.0"]["phi_min"] == pytest.approx(-324.217, abs=0.01)


def test_warm_bubble_first_step(golden_dir):
    """test_rk3_hydrostatic_adjustment.py section A: phi_min = -64.843 Pa/s."""
    pins = json.loads((golden_dir / "pins.json").read_text())["warm_bubble"]
    nx = ny = 64
    nz = 32
    Lx = Ly = 100_000.0
    Lz = 10_000.0
    z, rho0, th0 = O.build_base_state(nz, Lz)
    x = np.linspace(0, Lx, nx, endpoint=False)
    y = np.linspace(0, Ly, ny, endpoint=False)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    L = np.sqrt(((X - Lx / 2) / 10e3) ** 2 + ((Y - Ly / 2) / 10e3) ** 2 + ((Z - 2e3) / 2e3) ** 2)
    th = np.where(L <= 1.0, 2.0 * np.cos(np.pi * L / 2.0) ** 2, 0.0)
    cfg = O.StepConfig(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz, buoyancy=True, advection=None)
    s = O.State(np.zeros((nx, ny, nz)), np.zeros((nx, ny, nz)), np.zeros((nx, ny, nz + 1)),
                th, np.zeros((nx, ny, nz)), 0.0)
    s1, dg = O.Integrator(cfg, z, rho0, th0).step(s, 1.0)
    assert dg.surface_phi_min == pytest.approx(pins["1.0"]["surface_phi_min"], rel=1e-12)
    assert dg.max_w == pytest.approx(pins["1.0"]["max_w"], rel=1e-12)


def test_production_component_tendencies(golden_dir):
    """Surface drag, sponge, Laplacian and biharmonic diffusion, Newtonian
    cooling and the intensity cap (tendency.py:1259-1668) against the
    reference's own outputs on a random state, bit for bit."""
    g = np.load(golden_dir / "production.npz")
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    Lx, Ly, Lz = float(g["Lx"]), float(g["Ly"]), float(g["Lz"])
    z, _, _ = O.build_base_state(nz, Lz)
    u, v, w, th = g["in_u"], g["in_v"], g["in_w"], g["in_th"]
    got = {
        "drag": O.surface_drag_tendency(u, v, z, Cd=1.5e-3, H_bl=1500.0, u_env=2.0, v_env=-1.0),
        "drag0": O.surface_drag_tendency(u, v, z),
        "sponge": O.sponge_tendency(u, v, w, th, z, Lz=Lz, alpha_max=0.01,
                                    sponge_fraction=0.4, u_env=-1.5, v_env=0.5),
        "lap": O.horizontal_diffusion_tendency(u, v, 2.0e5, Lx, Ly, nx, ny),
        "hyper": O.hyper_diffusion_tendency(u, v, 3.0e12, Lx, Ly, nx, ny),
        "cool": (O.newtonian_cooling_tendency(th, 1800.0),),
        "cap": O.intensity_cap_tendency(u, v, v_cap=15.0, tau=300.0, u_env=1.0, v_env=-2.0),
    }
    fields = {"drag": ("du_dt", "dv_dt"), "drag0": ("du_dt", "dv_dt"),
              "sponge": ("du_dt", "dv_dt", "dw_dt", "dtheta_prime_dt"),
              "lap": ("du_dt", "dv_dt"), "hyper": ("du_dt", "dv_dt"),
              "cool": ("dtheta_prime_dt",), "cap": ("du_dt", "dv_dt")}
    for k, names in fields.items():
        for a, f in zip(got[k], names):
            assert np.array_equal(a, g[f"{k}_{f}"]), (k, f)
    # the cap acts only above v_cap
    assert 0 < np.count_nonzero(g["cap_du_dt"]) < g["cap_du_dt"].size


def test_vortex_diagnostics_match_reference(golden_dir):
    """Every recorded call of diagnostics.py (vorticity centre with and without
    a base state and with an empty window, low-level Vmax with an empty band,
    ventilation flow with an off-grid centre, budgets, the one-call wrapper and
    its log line) and run_translation_test._subcell_refine (clipped and empty
    patches, a NaN seed), bit for bit."""
    import warnings
    from oracle import vortex_diag as VD
    from tests.diag_cases import diag_states, replay, same
    n = 0
    for name, (u, v, z, dx, calls) in diag_states(golden_dir).items():
        for c in calls:
            with warnings.catch_warnings():
                warnings.simplefilter("ignore", RuntimeWarning)
                got = replay(c, VD, u, v, z, dx)
            assert same(got, c["out"]), (name, c["fn"], c["kw"], got, c["out"])
            n += 1
    assert n == 78


def test_blowup_run_first_steps(golden_dir):
    """The first steps of the reference's LH82 blow-up run (blowup_lh82.npz:
    the reference stepped until max|u| > 400 m/s, make_golden.py --blowup):
    the oracle's max|u| and max|w| follow the recorded ones."""
    g = np.load(golden_dir / "blowup_lh82.npz")
    c = json.loads(str(g["config_json"]))
    assert int(g["blew_step"]) > 0 and len(g["max_u"]) == int(g["blew_step"]) + 1
    assert not math.isfinite(g["max_u"][-1]) or g["max_u"][-1] > 400.0
    s, (z, rho0, th0) = oracle_initial_state(c)
    integ = O.Integrator(oracle_config(c), z, rho0, th0)
    for n in range(3):
        s, dg = integ.step(s, c["dt"], step_number=n)
        np.testing.assert_allclose([dg.max_u, dg.max_w], [g["max_u"][n], g["max_w"][n]],
                                   rtol=1e-12, atol=0)
