"""Device vortex initialisation, captured step graphs and the serving loop.

* The device fill of the Holland state gives the host path's fields bit for
  bit (FP64) and their FP32 rounding (FP32).
* A step graph replayed k times gives the same state as k calls of the step.
* Every run served in a mix of concurrent runs ends in exactly the state it
  reaches when served alone, and the FP64 runs equal the plain public
  ``RK3Integrator.step`` loop.
"""
import numpy as np
import pytest
import torch

from tests.gpu_helpers import Base, host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [
    dict(n=(32, 24, 8), kw=dict(Vmax=40.0, Rmax=50e3, B=1.5, f=4.99e-5, wind_decay_top=12e3)),
    dict(n=(96, 80, 16), kw=dict(Vmax=55.0, Rmax=30e3, B=1.8, f=6.1e-5, u_env=-3.0, v_env=1.0,
                                 wind_taper=True), xc=(300e3, 250e3)),
])
def test_device_vortex_fill_matches_host(case):
    from oraclev8_b200.vortex_init import HollandVortexInit
    nx, ny, nz = case["n"]
    Lx, Ly = nx * 20e3, ny * 20e3
    base = Base(nz, 16e3)
    init = HollandVortexInit(**case["kw"])
    xc = case.get("xc", (None, None))
    h = init.build_state(nx, ny, nz, Lx, Ly, base, x_c=xc[0], y_c=xc[1], device=False)
    for dtype in (torch.float64, torch.float32):
        d = init.build_state(nx, ny, nz, Lx, Ly, base, x_c=xc[0], y_c=xc[1], dtype=dtype)
        for f in ("u", "v", "w", "theta_prime", "projection_potential"):
            a, r = host(getattr(d, f)), getattr(h, f)
            if dtype == torch.float64:
                assert np.array_equal(a, r), f
            else:
                assert np.array_equal(a, r.astype(np.float32)), f


@pytest.mark.parametrize("precision", ["fp64", "fp32r"])
def test_step_graph_equals_step_calls(precision):
    from oraclev8_b200.serving import RunRequest, build_run
    req = RunRequest(0, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.5, precision)
    integ, s1, _ = build_run(req)
    _, s2, _ = build_run(req)
    g = integ.capture(s2, req.dt, 4)
    l0 = integ.plan.launches
    integ.step_(s1, req.dt)
    per_step = integ.plan.launches - l0
    for _ in range(7):
        integ.step_(s1, req.dt)
    for _ in range(2):
        g.launch()
    torch.cuda.synchronize()
    # the graph holds exactly the kernels of its four steps plus the two
    # diagnostics kernels of its last step (the blow-up check), and its
    # launches are counted like the direct ones
    assert g.kernels == 4 * per_step + 2
    assert integ.plan.launches - l0 == 8 * per_step + 2 * g.kernels
    for f in ("u", "v", "w", "theta_prime", "projection_potential"):
        assert torch.equal(getattr(s1, f), getattr(s2, f)), f


def test_runs_equal_alone_and_in_the_mix():
    from oraclev8_b200.serving import RunRequest, ServingEngine, build_run
    reqs = [RunRequest(0, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.4, "fp32r"),
            RunRequest(1, 128, 48, 30.0, 60e3, 1.2, 12.0, 0.3, "fp64", arrival_s=0.05),
            RunRequest(2, 96, 48, 60.0, 25e3, 1.9, 28.0, 0.5, "fp64"),
            RunRequest(3, 192, 32, 50.0, 35e3, 1.6, 15.0, 0.2, "fp32r", arrival_s=0.1),
            RunRequest(4, 128, 32, 38.0, 70e3, 1.1, 25.0, 0.35, "fp32r")]
    eng = ServingEngine(hbm_budget=40e9, chunk=5, keep_final=True)
    mix = {r.rid: r for r in eng.run(reqs)}
    assert sorted(mix) == [0, 1, 2, 3, 4]
    for req in reqs:
        alone = ServingEngine(chunk=7, keep_final=True, realtime=False).run([req])[0]
        for f, a in alone.final.items():
            assert np.array_equal(a, mix[req.rid].final[f]), (req.rid, f)
        assert mix[req.rid].steps == req.nsteps
        assert mix[req.rid].done_s >= mix[req.rid].admit_s >= 0.0
    # the served FP64 run is the plain public step loop
    req = reqs[2]
    integ, s, _ = build_run(req)
    for n in range(req.nsteps):
        s, _ = integ.step(s, req.dt, n)
    for f, a in mix[req.rid].final.items():
        assert np.array_equal(a, host(getattr(s, f))), f


def test_production_physics_runs_equal_alone_and_in_the_mix():
    """Runs with the reference's production physics (build_production_config:
    centred advection, biharmonic diffusion, divergence damping, cooling,
    drag) served together end in the state each reaches alone, and the FP64
    run equals the plain public step loop; all stay finite."""
    from oraclev8_b200.serving import RunRequest, ServingEngine, build_run
    reqs = [RunRequest(0, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.5, "fp32r", physics="production"),
            RunRequest(1, 128, 48, 30.0, 60e3, 1.2, 12.0, 0.4, "fp64", physics="production"),
            RunRequest(2, 96, 64, 60.0, 25e3, 1.9, 28.0, 0.6, "fp32r", physics="production",
                       arrival_s=0.05)]
    eng = ServingEngine(hbm_budget=40e9, chunk=6, keep_final=True)
    mix = {r.rid: r for r in eng.run(reqs)}
    assert sorted(mix) == [0, 1, 2]
    for req in reqs:
        rec = mix[req.rid]
        assert rec.error is None and rec.steps == req.nsteps
        alone = ServingEngine(chunk=5, keep_final=True, realtime=False).run([req])[0]
        for f, a in alone.final.items():
            assert np.isfinite(a).all(), (req.rid, f)
            assert np.array_equal(a, rec.final[f]), (req.rid, f)
    req = reqs[1]
    integ, s, _ = build_run(req)
    for n in range(req.nsteps):
        s, _ = integ.step(s, req.dt, n)
    for f, a in mix[req.rid].final.items():
        assert np.array_equal(a, host(getattr(s, f))), f
    with pytest.raises(ValueError):
        build_run(RunRequest(9, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.1, "fp64", physics="dry"))


def test_admission_respects_the_budget():
    """With room for one run at a time the runs are served one after the
    other, each admitted only once the previous one retired."""
    from oraclev8_b200.serving import RunRequest, ServingEngine, footprint_bytes
    reqs = [RunRequest(i, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.1, "fp64") for i in range(3)]
    budget = footprint_bytes(reqs[0]) * 1.5
    recs = sorted(ServingEngine(hbm_budget=budget, realtime=False).run(reqs),
                  key=lambda r: r.admit_s)
    for a, b in zip(recs, recs[1:]):
        assert b.admit_s >= a.done_s


@pytest.mark.parametrize("precision", ["fp64", "fp32r"])
def test_resume_from_snapshot_file_is_bit_exact(tmp_path, precision):
    """k1 steps, snapshot to .npz, a fresh integrator from the file, k2 more
    steps: the same state and time as k1 + k2 uninterrupted steps."""
    from oraclev8_b200.serving import RunRequest, build_run
    from oraclev8_b200 import snapshot as S
    req = RunRequest(0, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.5, precision)
    integ, s, _ = build_run(req)
    for n in range(7):
        s, _ = integ.step(s, req.dt, n)
        if n == 3:
            path = S.save_snapshot(tmp_path / "ck", S.take_snapshot(s, step=4))
    snap = S.load_snapshot(path)
    assert snap["step"] == 4
    integ2, _, _ = build_run(req)
    r = S.state_from_snapshot(snap)
    for n in range(4, 7):
        r, _ = integ2.step(r, req.dt, n)
    assert r.t == s.t
    for f in S.FIELDS:
        assert torch.equal(getattr(r, f), getattr(s, f)), f


def test_snapshot_copy_is_ordered_before_the_next_step():
    """A snapshot enqueued on the stepping stream holds the state of that
    moment although in-place steps follow it at once."""
    from oraclev8_b200.serving import RunRequest, build_run
    from oraclev8_b200 import snapshot as S
    req = RunRequest(0, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.5, "fp64")
    integ, s, _ = build_run(req)
    integ.step_(s, req.dt)
    ref = {f: getattr(s, f).clone() for f in S.FIELDS}
    cp = S.SnapshotCopy(s, step=1)
    for _ in range(3):
        integ.step_(s, req.dt)
    snap = cp.result()
    for f in S.FIELDS:
        assert np.array_equal(snap[f], host(ref[f])), f
    assert not np.array_equal(snap["u"], host(s.u))


def test_serving_snapshots_and_resume():
    """The engine hands snapshots every 10 steps to the sink; each equals the
    plain step loop at that step, and a request resumed from one ends in the
    state the uninterrupted run ends in."""
    from oraclev8_b200.serving import RunRequest, ServingEngine, build_run
    from oraclev8_b200 import snapshot as S
    req = RunRequest(7, 96, 32, 45.0, 40e3, 1.5, 20.0, 1.0, "fp64")
    got = []
    eng = ServingEngine(chunk=5, keep_final=True, realtime=False, snapshot_every=10,
                        snapshot_sink=lambda rid, snap: got.append((rid, snap)))
    rec = eng.run([req])[0]
    steps = [s["step"] for _, s in got]
    assert steps == list(range(10, req.nsteps + 1, 10)) and all(r == 7 for r, _ in got)
    integ, s, _ = build_run(req)
    by_step = {sn["step"]: sn for _, sn in got}
    for n in range(req.nsteps):
        s, _ = integ.step(s, req.dt, n)
        if n + 1 in by_step:
            for f in S.FIELDS:
                assert np.array_equal(by_step[n + 1][f], host(getattr(s, f))), (n + 1, f)
            assert by_step[n + 1]["t"] == s.t
    mid = by_step[10]
    req2 = RunRequest(8, 96, 32, 45.0, 40e3, 1.5, 20.0, 1.0, "fp64", resume=mid)
    rec2 = ServingEngine(chunk=7, keep_final=True, realtime=False).run([req2])[0]
    for f, a in rec.final.items():
        assert np.array_equal(a, rec2.final[f]), f
