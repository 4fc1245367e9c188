"""Blow-up detection on the device.

The reference's step does not raise on a blown-up state: its diagnostics carry
NumPy's NaN-propagating maxima (integrator.py:287-295), and its harnesses stop
a run when max|u| exceeds 400 m/s or is not finite
(measure_lh82_phase3.py:129-130).  The B200 step keeps both: the diagnostics
maxima propagate NaN, and the plan keeps a sticky blow-up flag that
``oracle_b200_read_diag`` reports as OB_ERR_NONFINITE.  The serving loop reads
that flag when it retires a run and records the blow-up.

Failures are made on the host (a NaN planted in an input state, a speed limit
below the vortex's wind), never by faulting the GPU.
"""
import ctypes
import math

import numpy as np
import pytest
import torch

from tests.gpu_helpers import Base, dev, TOL64

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 24, 8
LX, LY, LZ = NX * 20e3, NY * 20e3, 16e3
COR = dict(f=4.99e-5, mode="beta_plane", beta=2.15e-11, periodic_taper=True)


def _integ(precision, blowup_u_max=0.0):
    from oraclev8_b200.grid import LorenzStaggering
    from oraclev8_b200.solver import (AdvectionComponent, AnelasticProjection,
                                      BuoyancyComponent, CoriolisComponent,
                                      LH82AnelasticEquationSet, OperatorConfig, RK3Integrator)
    cfg = OperatorConfig(equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
                         buoyancy=BuoyancyComponent(),
                         projection=AnelasticProjection(NX, NY, NZ, LX, LY, LZ),
                         advection=AdvectionComponent(NX, NY, NZ, LX, LY, LZ, scheme="upwind5h"),
                         coriolis=CoriolisComponent(Ly=LY, ny=NY, **COR))
    base = Base(NZ, LZ)
    return RK3Integrator(cfg, base, precision=precision, blowup_u_max=blowup_u_max), base


def _host_state(base):
    from oracle import lh82 as O
    return O.Holland(40.0, 50e3, 1.5, 4.99e-5, wind_decay_top=12e3).build_state(
        NX, NY, NZ, LX, LY, base.z, base.rho0, base.theta0)


def _dev_state(s, dtype):
    from oraclev8_b200.solver import State
    return State(dev(s.u, dtype), dev(s.v, dtype), dev(s.w, dtype), dev(s.theta_prime, dtype),
                 dev(s.projection_potential, dtype), 0.0)


@pytest.mark.parametrize("precision", ["fp64", "fp32r"])
def test_nan_in_the_state_propagates_and_raises_the_flag(precision):
    from oracle import lh82 as O
    from oraclev8_b200 import _lib as L
    integ, base = _integ(precision)
    s = _host_state(base)
    s.u[5, 7, 3] = np.nan
    dtype = torch.float64 if precision == "fp64" else torch.float32
    out, dg = integ.step(_dev_state(s, dtype), 60.0, 0)
    # the reference's diagnostics are NumPy maxima, which propagate NaN
    ref = O.Integrator(O.StepConfig(nx=NX, ny=NY, nz=NZ, Lx=LX, Ly=LY, Lz=LZ, coriolis=dict(
        COR, Ly=LY, ny=NY)), base.z, base.rho0, base.theta0)
    _, rdg = ref.step(s, 60.0)
    assert math.isnan(rdg.max_u) and math.isnan(dg.max_u)
    assert dg.blowup == 1
    buf = (ctypes.c_double * L.DIAG_COUNT)()
    rc = L.load().oracle_b200_read_diag(integ.plan.handle, buf, L.DIAG_COUNT,
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == L.OB_ERR_NONFINITE
    assert b"non-finite" in L.load().oracle_b200_last_error()
    # sticky: a later diagnosed step still reports it
    _, dg2 = integ.step(out, 60.0, 1)
    assert dg2.blowup == 1


def test_speed_limit_raises_the_flag_and_maxima_match_the_oracle():
    from oracle import lh82 as O
    integ, base = _integ("fp64", blowup_u_max=10.0)
    s = _host_state(base)
    _, dg = integ.step(_dev_state(s, torch.float64), 60.0, 0)
    ref = O.Integrator(O.StepConfig(nx=NX, ny=NY, nz=NZ, Lx=LX, Ly=LY, Lz=LZ, coriolis=dict(
        COR, Ly=LY, ny=NY)), base.z, base.rho0, base.theta0)
    _, rdg = ref.step(s, 60.0)
    assert dg.max_u > 10.0
    assert abs(dg.max_u - rdg.max_u) <= TOL64 * rdg.max_u
    assert dg.blowup == 2


def test_clean_run_keeps_the_flag_down():
    integ, base = _integ("fp32r", blowup_u_max=400.0)
    st = _dev_state(_host_state(base), torch.float32)
    for n in range(3):
        st, dg = integ.step(st, 60.0, n)
        assert dg.blowup == 0 and math.isfinite(dg.max_u)


def test_serving_retires_a_blown_up_run_and_backfills():
    from oraclev8_b200.serving import RunRequest, ServingEngine, build_run
    from oraclev8_b200.snapshot import take_snapshot
    good = RunRequest(0, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.3, "fp32r")
    bad = RunRequest(1, 96, 32, 45.0, 40e3, 1.5, 20.0, 0.3, "fp32r")
    later = RunRequest(2, 96, 32, 50.0, 30e3, 1.7, 15.0, 0.2, "fp64")
    # the bad run resumes from a snapshot with one NaN planted in theta'
    _, s0, _ = build_run(bad)
    snap = take_snapshot(s0, step=0)
    snap["theta_prime"] = np.array(snap["theta_prime"], copy=True)
    snap["theta_prime"][10, 20, 5] = np.nan
    bad.resume = snap
    # a budget that holds one run at a time: the third is admitted only after
    # one of the others has retired
    from oraclev8_b200.serving import footprint_bytes
    eng = ServingEngine(hbm_budget=footprint_bytes(good) * 1.5, chunk=4, realtime=False,
                        keep_final=True)
    recs = {r.rid: r for r in eng.run([good, bad, later])}
    assert sorted(recs) == [0, 1, 2]
    assert recs[1].error == "non-finite state"
    assert recs[0].error is None and recs[2].error is None
    for rid in (0, 2):
        assert all(np.isfinite(recs[rid].final[f]).all() for f in ("u", "v", "w"))


def test_lh82_blowup_matches_the_reference(golden_dir):
    """The LH82 physics of the mid-size workload (WS5, buoyancy, heating,
    theta' noise, dt 20 s) on a 96 x 96 x 64 grid blows up in the reference
    itself (blowup_lh82.npz: the reference's max|u| and max|w| of every step,
    generated by make_golden.py --blowup).  The plain FP64 step follows the
    reference's diagnostics step for step (within 1e-6 until 30 steps before
    the blow-up, while round-off differences are still small against the
    growing mode) and raises its blow-up flag at the same step."""
    import json as _json
    from tests.test_oracle_golden import oracle_initial_state
    from tests.gpu_helpers import b200_config
    from oraclev8_b200.solver import RK3Integrator
    g = np.load(golden_dir / "blowup_lh82.npz")
    c = _json.loads(str(g["config_json"]))
    ref_u, ref_w, blew = g["max_u"], g["max_w"], int(g["blew_step"])
    assert blew > 0
    s0, _ = oracle_initial_state(c)
    integ = RK3Integrator(b200_config(c), Base(c["nz"], c["Lz"]), precision="fp64",
                          blowup_u_max=400.0)
    st = _dev_state(s0, torch.float64)
    flagged = -1
    for n in range(blew + 1):
        st, dg = integ.step(st, c["dt"], n)
        if n < blew - 30:
            assert abs(dg.max_u - ref_u[n]) <= 1e-6 * ref_u[n], (n, dg.max_u, ref_u[n])
            assert abs(dg.max_w - ref_w[n]) <= 1e-6 * max(ref_w[n], 1.0), (n, dg.max_w, ref_w[n])
        if dg.blowup and flagged < 0:
            flagged = n
    assert flagged == blew, (flagged, blew)
