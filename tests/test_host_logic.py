"""Host-side logic of the B200 package that needs no GPU: configuration
compilation, reference-identical host tables, guards and error types."""
import math

import numpy as np
import pytest

from oracle import lh82 as O


def test_base_state_and_constants_identical():
    from oraclev8_b200.production_config import build_base_state
    for nz, Lz in ((32, 16e3), (64, 16e3), (80, 20e3), (7, 3e3)):
        a = build_base_state(nz, Lz)
        b = O.build_base_state(nz, Lz)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_coriolis_profile_identical():
    from oraclev8_b200.solver import CoriolisComponent
    for kw in (dict(f=4.99e-5, beta=2.15e-11, periodic_taper=True),
               dict(f=6.164e-5, periodic_taper=False),
               dict(f=3.7e-5, periodic_taper=True, y0=1e5)):
        c = CoriolisComponent(mode="beta_plane", Ly=2.56e6, ny=128, **kw)
        ref = O.coriolis_profile(kw["f"], "beta_plane", kw.get("beta"), 2.56e6, 128,
                                 kw.get("y0"), kw["periodic_taper"])
        assert np.array_equal(c.f_y, ref)
    with pytest.raises(ValueError):
        CoriolisComponent(mode="beta_plane")


def test_heating_factors_reproduce_reference_field():
    from oraclev8_b200.solver import DiabaticHeatingComponent
    kw = dict(Q_max=3.0 / 3600.0, r_eyewall=40e3, width_r=math.sqrt(2.0) * 15e3, z_peak=6e3,
              width_z=math.sqrt(2.0) * 2e3, nx=24, ny=20, nz=9, Lx=240e3, Ly=200e3, Lz=16e3)
    h = DiabaticHeatingComponent(**kw)
    r, z = h.heat_factors
    assert np.array_equal(r[:, :, None] * z[None, None, :], O.heating_field(**kw))


def _cfg(**extra):
    from oraclev8_b200.solver import (AdvectionComponent, AnelasticProjection,
                                      BuoyancyComponent, CoriolisComponent,
                                      LH82AnelasticEquationSet, OperatorConfig)
    from oraclev8_b200.grid import LorenzStaggering
    kw = dict(equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
              buoyancy=BuoyancyComponent(),
              projection=AnelasticProjection(32, 24, 8, 640e3, 480e3, 16e3),
              advection=AdvectionComponent(32, 24, 8, 640e3, 480e3, 16e3, scheme="upwind5h"),
              coriolis=CoriolisComponent(f=4.99e-5, mode="beta_plane", beta=2.15e-11,
                                         Ly=480e3, ny=24, periodic_taper=True))
    kw.update(extra)
    return OperatorConfig(**kw)


def test_compile_config_maps_every_slot():
    from oraclev8_b200 import _lib as L
    from oraclev8_b200.solver.integrator import compile_config
    from oraclev8_b200.solver import HelmholtzDivergenceDampingComponent, DiabaticHeatingComponent
    from oraclev8_b200.production_config import BaseState
    cfg = _cfg(divergence_damping=HelmholtzDivergenceDampingComponent(0.5, 640e3, 480e3, 32, 24),
               diabatic_heating=DiabaticHeatingComponent(1e-3, 40e3, 20e3, 6e3, 3e3, 32, 24, 8,
                                                         640e3, 480e3, 16e3))
    spec = compile_config(cfg, BaseState(8, 16e3), "fp32")
    assert (spec.nx, spec.ny, spec.nz) == (32, 24, 8)
    assert spec.buoyancy and spec.projection and spec.damping and spec.heating
    assert spec.advection == L.OB_ADV_UPWIND5H and spec.coriolis == L.OB_COR_BETA
    assert spec.epsilon == 0.5 and spec.f_y.shape == (24,) and spec.precision == "fp32"
    assert not (spec.drag or spec.sponge or spec.cooling) and spec.diffusion == L.OB_DIFF_NONE


@pytest.mark.parametrize("hyper", [False, True])
def test_compile_config_maps_production_slots(hyper):
    """The drag weight and level spacing, the sponge's full and half level
    rates, the diffusion kind and 1/tau reach the plan as the reference forms
    them (tendency.py:1318-1338, 1478-1498, 1544-1546, 1604-1606, 1659)."""
    from oraclev8_b200 import _lib as L
    from oraclev8_b200.solver.integrator import compile_config
    from oraclev8_b200.solver import (SurfaceDragComponent, SpongeDampingComponent,
                                      HorizontalDiffusionComponent, HyperDiffusionComponent,
                                      NewtonianCoolingComponent)
    from oraclev8_b200.production_config import BaseState
    base = BaseState(8, 16e3)
    diff = (HyperDiffusionComponent(1e12, 640e3, 480e3, 32, 24) if hyper
            else HorizontalDiffusionComponent(500.0, 640e3, 480e3, 32, 24))
    cfg = _cfg(surface_drag=SurfaceDragComponent(2e-3, 3000.0, -4.0, 1.5),
               sponge_damping=SpongeDampingComponent(16e3, 0.02, 0.25, -4.0, 1.5),
               horiz_diffusion=diff, newtonian_cooling=NewtonianCoolingComponent(1800.0))
    spec = compile_config(cfg, base, "fp64")
    z = np.asarray(base.z, dtype=np.float64)
    assert spec.drag and spec.drag_cd == 2e-3 and spec.drag_dz == z[1] - z[0]
    assert np.array_equal(spec.drag_weight, np.maximum(0.0, 1.0 - z / 3000.0))
    assert (spec.drag_u_env, spec.drag_v_env) == (-4.0, 1.5)
    zs = 16e3 * 0.75
    a = np.where(z > zs, 0.02 * ((z - zs) / (16e3 - zs)) ** 2, 0.0)
    assert spec.sponge and np.array_equal(spec.sponge_alpha, a)
    assert np.array_equal(spec.sponge_alpha_h, np.r_[a[0], 0.5 * (a[:-1] + a[1:]), a[-1]])
    assert (spec.sponge_u_env, spec.sponge_v_env) == (-4.0, 1.5)
    assert spec.diffusion == (L.OB_DIFF_BIHARMONIC if hyper else L.OB_DIFF_LAPLACIAN)
    assert spec.diff_nu == (1e12 if hyper else 500.0)
    assert (spec.diff_dx2, spec.diff_dy2) == ((640e3 / 32) ** 2, (480e3 / 24) ** 2)
    assert spec.cooling and spec.cool_alpha == 1.0 / 1800.0


def test_unsupported_components_raise_and_guards():
    from oraclev8_b200.solver import PressureGradientComponent, AdvectionComponent
    from oraclev8_b200.solver.integrator import compile_config
    from oraclev8_b200.production_config import BaseState
    with pytest.raises(ValueError):
        _cfg(pressure_gradient=PressureGradientComponent(32, 24, 8, 1, 1, 1))
    cfg = _cfg(pressure_gradient=PressureGradientComponent(32, 24, 8, 1, 1, 1),
               _unsafe_pgc_override=True)
    with pytest.raises(NotImplementedError):
        compile_config(cfg, BaseState(8, 16e3), "fp64")
    with pytest.raises(ValueError):
        AdvectionComponent(scheme="weno")


def test_operator_config_slot_order_and_stages():
    cfg = _cfg()
    names = [c.name for c in cfg.active_components()]
    assert names == ["buoyancy", "anelastic_projection", "advection", "coriolis"]
    assert [c.name for c in cfg.fast_components()] == ["buoyancy"]
    assert [c.name for c in cfg.slow_components()] == ["advection", "coriolis"]
    d = cfg.to_log_dict()
    assert d["n_pre_projection"] == 1 and d["n_slow"] == 2 and d["n_projection"] == 1


def test_product_path_has_no_cpu_fallback():
    """Without a CUDA device the backend refuses to run (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from oraclev8_b200.solver import RK3Integrator
    from oraclev8_b200.production_config import BaseState
    with pytest.raises(RuntimeError):
        RK3Integrator(_cfg(), BaseState(8, 16e3))


def test_product_package_never_imports_oracle():
    import pathlib
    import re
    pkg = pathlib.Path(__file__).resolve().parents[1] / "oraclev8_b200"
    for f in pkg.rglob("*.py"):
        assert not re.search(r"^\s*(from|import)\s+oracle\b", f.read_text(), re.M), f


def test_vortex_init_identical_to_reference_restatement():
    from oraclev8_b200.vortex_init import HollandVortexInit
    from oraclev8_b200.production_config import BaseState
    base = BaseState(8, 16e3)
    for kw in (dict(Vmax=40.0, Rmax=50e3, B=1.5, f=4.99e-5, wind_decay_top=12e3),
               dict(Vmax=55.0, Rmax=30e3, B=1.8, f=6.1e-5, u_env=-3.0, v_env=1.0,
                    wind_taper=True)):
        a = HollandVortexInit(**kw).build_state(32, 24, 8, 640e3, 480e3, base, device=False)
        b = O.Holland(**kw).build_state(32, 24, 8, 640e3, 480e3, base.z, base.rho0, base.theta0)
        for f in ("u", "v", "w", "theta_prime"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_tracker_host_logic_matches_oracle():
    """The host half of the B200 tracker (sub-cell refine from the device's
    5-point neighbourhood, vorticity fall-back on the device's column means)
    gives the oracle's answers on the same fields."""
    from oraclev8_b200 import storm_tracker as T
    rng = np.random.default_rng(4)
    nx, ny, nz, dx = 20, 16, 6, 10e3
    p = rng.standard_normal((nx, ny))
    for ix, iy in ((5, 7), (0, 3), (nx - 1, ny - 1), (10, 0)):
        nb = [p[ix, iy]] + [p[x, y] if 0 <= x < nx and 0 <= y < ny else 0.0
                            for x, y in ((ix - 1, iy), (ix + 1, iy), (ix, iy - 1), (ix, iy + 1))]
        assert T._refine(nb, ix, iy, nx, ny) == O.parabolic_refine(p, ix, iy)
    u = 5 * rng.standard_normal((nx, ny, nz))
    v = 5 * rng.standard_normal((nx, ny, nz))
    h = nz // 2
    dvdx = (np.roll(v[:, :, :h], -1, 0) - np.roll(v[:, :, :h], 1, 0)) / (2.0 * dx)
    dudy = (np.roll(u[:, :, :h], -1, 1) - np.roll(u[:, :, :h], 1, 1)) / (2.0 * dx)
    zcol = np.mean(np.maximum(dvdx - dudy, 0.0), axis=2)
    for last in (None, (80e3, 70e3), (150e3, 20e3)):
        assert T._vorticity_centre(zcol, nx, ny, dx, last) == \
            O.vorticity_centre(u, v, nx, ny, dx, last_pos=last)


def test_diagnostics_refuse_host_fields():
    """The diagnostics read device fields only (no CPU fallback)."""
    import types
    from oraclev8_b200 import diagnostics as D
    st = types.SimpleNamespace(u=np.zeros((4, 4, 4)), v=np.zeros((4, 4, 4)))
    with pytest.raises(TypeError):
        D.vmax_3d(st, None)
    with pytest.raises(TypeError):
        D.subcell_refine(st, 1.0, 1.0, 1.0)


def test_snapshot_file_round_trip(tmp_path):
    """The snapshot record of run_translation_test.py:291-295 through .npz and
    back, keys and values unchanged; a file without the fields is refused."""
    from oraclev8_b200 import snapshot as S
    rng = np.random.default_rng(5)
    snap = {f: rng.standard_normal((6, 5, 4 + (f == "w"))) for f in S.FIELDS}
    snap.update(t=1234.5, cx=3.5e5, cy=None, step=17)
    back = S.load_snapshot(S.save_snapshot(tmp_path / "s", snap))
    assert set(back) == set(snap)
    for k, val in snap.items():
        if isinstance(val, np.ndarray):
            assert np.array_equal(back[k], val) and back[k].dtype == val.dtype
        else:
            assert back[k] == val
    np.savez(tmp_path / "bad.npz", u=snap["u"])
    with pytest.raises(ValueError):
        S.load_snapshot(tmp_path / "bad.npz")


def test_gyre_snapshot_record(tmp_path):
    """run_translation_test.py:2104-2125: column means, centred vorticity with
    dx on both axes, centre and dx."""
    from oraclev8_b200 import snapshot as S
    rng = np.random.default_rng(6)
    u, v = rng.standard_normal((8, 6, 5)), rng.standard_normal((8, 6, 5))
    p = S.save_gyre_snapshot(tmp_path / "g", dict(u=u, v=v, cx=1.0, cy=2.0), 5e3)
    d = np.load(p)
    u2, v2 = u.mean(axis=2), v.mean(axis=2)
    zeta = ((np.roll(v2, -1, 0) - np.roll(v2, 1, 0)) / (2 * 5e3)
            - (np.roll(u2, -1, 1) - np.roll(u2, 1, 1)) / (2 * 5e3))
    assert np.array_equal(d["zeta"], zeta) and np.array_equal(d["u"], u2)
    assert float(d["cx"]) == 1.0 and float(d["cy"]) == 2.0 and float(d["dx"]) == 5e3


def test_vortex_init_host_helpers(golden_dir):
    """vertical_structure, surface_pressure_deficit, peak_wind_check and the
    summary line equal the reference's (vortex_init.py:191-411)."""
    import json
    from oraclev8_b200.vortex_init import HollandVortexInit
    z = np.linspace(0.0, 20e3, 9)
    for rec in json.loads((golden_dir / "vortex_helpers.json").read_text()):
        v = HollandVortexInit(**rec["kw"])
        assert v.summary() == rec["summary"]
        assert list(v.peak_wind_check()) == rec["peak"]
        assert v.surface_pressure_deficit(1.15) == rec["p_sfc"]
        assert [float(x) for x in v.vertical_structure(z)] == rec["s_z"]


def test_backend_xp_takes_the_harness_spellings():
    """The drivers and harnesses call the backend's ``xp`` with NumPy
    spellings (run_storm.py:128-137, run_translation_test.py:132-160):
    roll with axis=, maximum with a Python scalar, mean with axis=, arange
    with dtype, sum.  On torch tensors they give NumPy's values."""
    import torch
    from oraclev8_b200.backend import xp
    rng = np.random.default_rng(12)
    a = rng.standard_normal((6, 5, 4))
    t = torch.as_tensor(a)
    dx = 5e3
    got = xp.mean(xp.maximum((xp.roll(t, -1, axis=0) - xp.roll(t, 1, axis=0)) / (2.0 * dx)
                             - (xp.roll(t, -1, axis=1) - xp.roll(t, 1, axis=1)) / (2.0 * dx),
                             0.0), axis=2)
    want = np.mean(np.maximum((np.roll(a, -1, axis=0) - np.roll(a, 1, axis=0)) / (2.0 * dx)
                              - (np.roll(a, -1, axis=1) - np.roll(a, 1, axis=1)) / (2.0 * dx),
                              0.0), axis=2)
    assert np.allclose(got.numpy(), want, rtol=1e-15, atol=0.0)
    w = got ** 2
    ix = xp.arange(1, 5, dtype=xp.float64)[:, None]
    assert float(xp.sum(ix * w[1:5])) == pytest.approx(float(np.sum(np.arange(1, 5.0)[:, None]
                                                                     * (want ** 2)[1:5])),
                                                       rel=1e-14)
    assert np.array_equal(xp.minimum(t, 0.5).numpy(), np.minimum(a, 0.5))
    assert np.array_equal(xp.clip(t, -0.5, 0.5).numpy(), np.clip(a, -0.5, 0.5))
    assert float(xp.sqrt(xp.mean(t ** 2))) == pytest.approx(float(np.sqrt(np.mean(a ** 2))),
                                                            rel=1e-14)
    assert xp.zeros_like(t).shape == t.shape and isinstance(t, xp.Tensor)


def test_bench_byte_model_of_the_shared_stage_transforms():
    """bench.py's per-launch algorithmic bytes: with the fast stages' forward x
    transforms shared, a step's forward x and y launches move the bytes of two
    stage x launches less, plus one more spectrum written by the shared launch
    and one more read by each stage's y launch; every other class is as it
    was.  The inverse x class counts the potential only where the step keeps
    it (two of five launches)."""
    import bench
    w = bench.WORKLOADS["config2"]
    S = 4
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    n, nw, ns = nx * ny * nz, nx * ny * (nz + 1), (nx // 2 + 1) * ny * nz
    per = bench.kernel_bytes(w, S)
    sh = bench.kernel_bytes(w, S, shared_stages=True)
    step = lambda kb, nfx: kb["fx"] * nfx + kb["fy"] * 5
    stage_fx = (2 * n + 2 * nw) * S + 2 * ns * 2 * S
    spectrum = ns * 2 * S
    assert math.isclose(step(per, 5) - step(sh, 3), 2 * stage_fx - 4 * spectrum, rel_tol=1e-12)
    for c in ("thomas", "iy", "ix", "slow", "diag"):
        assert sh[c] == per[c]
    ix_all = 2 * spectrum * 5 + 2 * 2 * (2 * n + nw) * S + 3 * ((2 * n + 2 * nw) + (2 * n + nw)) * S
    assert math.isclose(per["ix"] * 5, ix_all + 2 * n * S, rel_tol=1e-12)


def test_serving_footprint_counts_every_plan_buffer():
    """The serving loop admits a run by footprint_bytes: its state plus the
    buffers its plan allocates.  A single-precision 1024 x 1024 run with the
    fast stages also holds the three spectra of the shared stage transforms;
    other sizes, FP64 runs and the production physics (no fast stages) do
    not."""
    from oraclev8_b200.serving import RunRequest, footprint_bytes

    def req(n, nz, precision, physics):
        return RunRequest(rid=0, n=n, nz=nz, vmax=50.0, rmax=40e3, b=1.6, lat_deg=20.0,
                          hours=1.0, precision=precision, physics=physics)

    def base(n, nz, precision, physics):
        S = 8 if precision == "fp64" else 4
        cells, ns = n * n * nz, (n // 2 + 1) * n * nz
        b = S * 17 * cells + 3 * ns * 2 * S
        if physics == "production":
            b += 4 * cells * S
        if precision != "fp64":
            b += 2 * ns * 16
        return b

    for n, nz in ((96, 32), (384, 64), (1024, 80)):
        for precision in ("fp64", "fp32r"):
            for physics in ("lh82", "production"):
                b = base(n, nz, precision, physics)
                if n == 1024 and precision == "fp32r" and physics == "lh82":
                    b += 3 * (n // 2 + 1) * n * nz * 8
                assert footprint_bytes(req(n, nz, precision, physics)) == int(b * 1.05) + (8 << 20)
    # the shared transforms are 1.0 GB of the 1024 x 1024 x 80 FP32 run's footprint
    extra = (footprint_bytes(req(1024, 80, "fp32r", "lh82"))
             - int(base(1024, 80, "fp32r", "lh82") * 1.05) - (8 << 20))
    assert 1.05e9 < extra < 1.07e9


def test_serving_admission_is_fifo_with_backfill_under_the_budget():
    """admit_from_queue (the serving loop's admission): queue order, a request
    that does not fit is skipped and a later smaller one takes the room, an
    oversized request runs alone, and the resident / set-up caps hold."""
    from types import SimpleNamespace as R
    from oraclev8_b200.serving import admit_from_queue
    size = lambda r: r.b
    q = [R(rid=0, b=60), R(rid=1, b=50), R(rid=2, b=30), R(rid=3, b=10)]
    adm, used = admit_from_queue(q, 0, 100, 0, 0, 8, 8, size)
    assert [r.rid for r in adm] == [0, 2, 3] and used == 100 and [r.rid for r in q] == [1]
    # the skipped request is admitted once its room is free
    adm, used = admit_from_queue(q, used - 60, 100, 2, 0, 8, 8, size)
    assert [r.rid for r in adm] == [1] and used == 90 and not q
    # a request larger than the budget: alone, and only when nothing is resident
    q = [R(rid=4, b=500), R(rid=5, b=10)]
    adm, used = admit_from_queue(q, 10, 100, 1, 0, 8, 8, size)
    assert [r.rid for r in adm] == [5] and used == 20
    adm, used = admit_from_queue(q, 0, 100, 0, 0, 8, 8, size)
    assert [r.rid for r in adm] == [4] and used == 500 and not q
    # caps: runs resident or in set-up, runs in set-up
    q = [R(rid=i, b=1) for i in range(10)]
    adm, _ = admit_from_queue(q, 0, 100, 3, 1, 6, 8, size)
    assert [r.rid for r in adm] == [0, 1]
    adm, _ = admit_from_queue(q, 0, 100, 0, 2, 100, 4, size)
    assert [r.rid for r in adm] == [2, 3]


def test_serving_feeds_least_remaining_work_first_under_the_inflight_cap():
    """runs_to_feed: shortest remaining work first; runs already in flight keep
    their work; idle runs start only while the in-flight cells stay under the
    cap; finished runs get nothing."""
    from types import SimpleNamespace as R
    from oraclev8_b200.serving import runs_to_feed
    run = lambda rid, left, cells, busy=False: R(req=R(rid=rid, cells=cells), left=left,
                                                  events=[object()] if busy else [])
    a = run(0, 10, 100)            # 1000 cell-steps left
    b = run(1, 2, 100)             # 200
    c = run(2, 5, 100, busy=True)  # 500, in flight
    d = run(3, 0, 100)             # finished
    e = run(4, 2, 100)             # 200, ties with b: rid order
    assert [x.req.rid for x in runs_to_feed([a, b, c, d, e], 1e9)] == [1, 4, 2, 0]
    # cap of 250 cells, c's 100 in flight: b starts (100 < 250, then 200 in
    # flight), e starts (200 < 250, then 300), a does not (300 >= 250)
    fed = [x.req.rid for x in runs_to_feed([a, b, c, d, e], 250)]
    assert fed == [1, 4, 2]
    fed = [x.req.rid for x in runs_to_feed([a, b, c, d, e], 150)]
    assert fed == [1, 2]
    # nothing idle starts once the runs in flight fill the cap
    assert [x.req.rid for x in runs_to_feed([a, c], 100)] == [2]


def test_serving_loop_on_a_fake_device(monkeypatch):
    """The serving loop itself (ServingEngine.run) with the device replaced:
    runs are set up, fed in chunks, retired and backfilled; the resident bytes
    never exceed the budget; a run whose blow-up flag is raised gets no
    further chunks and retires with an error record; every request ends with a
    record."""
    import threading
    import torch
    from oraclev8_b200 import serving as S

    monkeypatch.setattr(torch.cuda, "current_device", lambda: 0)
    monkeypatch.setattr(torch.cuda, "set_device", lambda d: None)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a: None)

    class Event:
        def __init__(self):
            self.polls = 0

        def query(self):  # completes on its second poll
            self.polls += 1
            return self.polls > 1

    class Fake(S.ServingEngine):
        def __init__(self, blow, **kw):
            super().__init__(**kw)
            self.blow, self.lock = set(blow), threading.Lock()
            self.resident = self.peak = 0

        def _prepare(self, req):
            with self.lock:
                self.resident += S.footprint_bytes(req)
                self.peak = max(self.peak, self.resident)
            rec = S.RunRecord(req.rid, req.n, req.nz, req.precision, req.nsteps, req.cells,
                              req.arrival_s)
            return S._Active(req, rec, None, None, None, {}, req.nsteps,
                             bytes=S.footprint_bytes(req), flag=[0.0] * 16)

        def _launch(self, a):
            k = min(self.chunk, a.left)
            a.events.append(Event())
            a.left -= k
            a.launched += k
            if a.req.rid in self.blow:
                a.flag[14] = 1.0  # the diagnostics block's blow-up slot

        def _retire(self, a, now):
            with self.lock:
                self.resident -= a.bytes
            a.rec.done_s = now
            if a.blown:
                a.rec.error = "blown up"
            return a.rec

    reqs = [S.RunRequest(rid=i, n=n, nz=nz, vmax=40.0, rmax=40e3, b=1.5, lat_deg=20.0,
                         hours=1.0, precision="fp32r")
            for i, (n, nz) in enumerate([(96, 32), (384, 64), (128, 48), (256, 32),
                                         (192, 64), (96, 48), (384, 32), (128, 32)])]
    budget = 2.2 * max(S.footprint_bytes(r) for r in reqs)
    eng = Fake(blow={3}, hbm_budget=budget, chunk=8, depth=2, realtime=False,
               max_active=4, prepare_ahead=2, inflight_cells=2e6)
    recs = eng.run(reqs)
    assert sorted(r.rid for r in recs) == list(range(len(reqs)))
    assert all(r.done_s == r.done_s for r in recs)  # every run retired (not NaN)
    assert 0 < eng.peak <= budget and eng.resident == 0
    by = {r.rid: r for r in recs}
    assert by[3].error == "blown up" and all(by[i].error is None for i in by if i != 3)
