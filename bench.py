"""Benchmark of the LH82 anelastic RK3 step (cell-updates/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp32r|fp64|fp32]
                    [--workload config2|config1|config0] [--impl b200|reference]
                    [--track-hours H]

Default workload: the production-size single run, the one the FP32-refined
versus plain-FP64 target is quoted on -- 1024 x 1024 x 80 cells, dx = 4 km,
0-20 km (dz = 250 m), beta-plane at 25N (f0 = 2 Omega sin 25, beta =
2 Omega cos 25 / R, periodic taper), Holland vortex Vmax 55 m/s / Rmax 30 km /
B 1.8 with wind decaying linearly to zero at 12 km and a uniform 3 m/s
easterly background flow (vortex and Coriolis), WS5 advection, buoyancy,
projection, dt = 15 s.  Synthetic inputs (the reference has no dataset);
every field is larger than L2 (336-671 MB per field), so consecutive steps
stream from HBM.  ``--workload config1`` is the mid-size run (512 x 512 x 64,
dx 5 km, eyewall heating, seeded theta' noise, dt 20 s).

One "step" = one full RK3Integrator.step: two Strang slow half steps (fused
WS5 + Coriolis (+ heating) tendency and forward Euler), three fast stages,
five anelastic projections (FFT x/y + Thomas z + correction) and the
device-side step diagnostics.

Precision (the metric is FP32-refined against plain FP64): the default
``fp32r`` runs the step on an FP32 state and, after its final projection, one
defect correction whose residual divergence is formed in FP64.  The same line
then carries ``fp64_plain`` (the plain FP64 step timed the same way on the
same workload, and the ratio) and ``accuracy`` (per-field error of the FP32
run against the FP64 run after the same steps, and the FP64-evaluated
divergence of both); these two come last in the line.  ``--precision fp64``
times the plain FP64 step alone.

``cufft``: the transforms of one projection (three real-to-complex x
transforms, two complex y transforms and their inverses) done by cuFFT
through torch.fft on the same fields, timed beside this library's pencil
kernels, which also do the projection's arithmetic.  A comparison only.

Ensemble and serving (the metric's latency half, at N = 1): ``ensemble``
serves a sample of the mixed 256-run ensemble through the serving loop
(resident runs, captured step graphs, one stream per run) next to the same
runs served serially in plain FP64; ``serving`` replays a Poisson request
stream with HBM admission and reports p50/p95/p99 time-to-completion.  Sizes
are set by ``--ensemble-runs/--ensemble-hours`` and
``--serving-requests/--serving-scale``; ``--no-ensemble`` skips both.
``--ensemble-physics`` picks the draws' step: the production physics by
default (the LH82 physics of the workloads blows up within hours in the
reference's own algorithm, and blown-up runs retire early), or ``lh82``.

Production physics (``production``; ``--no-production`` skips it): the
reference's build_production_config (centred advection, beta-plane,
biharmonic diffusion, divergence damping, Newtonian cooling, surface drag,
projection, no buoyancy) on the same grid and initial state, with the
intensity cap added after each step as the reference's run loop does; timed
in the bench's precision and in plain FP64, with the slow class's roofline.

``--track-hours H`` (not part of the default run): the workload run for H
hours in FP32-refined and in plain FP64 on the device, with the storm centre
found every hour (find_storm_centre chained through last_pos /
last_raw_pos as run_storm.py:180-190 does); prints one JSON line with the
hourly centre differences, max|w| differences and the final per-field errors.

N > 1: N independent replicas, one per GPU (the path partitions into
independent runs; no collective on the data path).

--impl reference times the reference algorithm on the host CPU (the NumPy
oracle; the reference is pure Python and cannot be installed on the GPU host)
on a bounded sample of the same workload: the workload's full column (same
nz, Lz and physics) on a 128 x 128 horizontal tile at the workload's dx, one
independent sample run per host core.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "config1": dict(nx=512, ny=512, nz=64, dx=5e3, Lz=16e3, dt=20.0,
                    vortex=dict(Vmax=50.0, Rmax=40e3, B=1.6, f=4.99e-5),
                    coriolis=dict(f=4.99e-5, mode="beta_plane", beta=2.15e-11,
                                  periodic_taper=True),
                    heating=dict(Q_max=3.0 / 3600.0, r_eyewall=40e3,
                                 width_r=math.sqrt(2.0) * 15e3, z_peak=6e3,
                                 width_z=math.sqrt(2.0) * 2e3),
                    noise_seed=20261203),
    "config0": dict(nx=128, ny=128, nz=32, dx=20e3, Lz=16e3, dt=60.0,
                    vortex=dict(Vmax=40.0, Rmax=50e3, B=1.5, f=4.99e-5),
                    coriolis=dict(f=4.99e-5, mode="beta_plane", beta=2.15e-11,
                                  periodic_taper=True), heating=None, noise_seed=None),
    "config2": dict(nx=1024, ny=1024, nz=80, dx=4e3, Lz=20e3, dt=15.0,
                    vortex=dict(Vmax=55.0, Rmax=30e3, B=1.8,
                                f=2 * 7.2921e-5 * math.sin(math.radians(25.0)), u_env=-3.0),
                    coriolis=dict(f=2 * 7.2921e-5 * math.sin(math.radians(25.0)),
                                  mode="beta_plane",
                                  beta=2 * 7.2921e-5 * math.cos(math.radians(25.0)) / 6.371e6,
                                  periodic_taper=True, u_env=-3.0),
                    heating=None, noise_seed=None),
}
# a 1024 x 256 x 80 slab of the production grid (same dx, column and physics):
# the case kernel-level ncu captures of the 1024-point pencils run on, its
# fields (84 MB each) still larger than L2 together
WORKLOADS["config2s"] = dict(WORKLOADS["config2"], ny=256)
# Algorithmic field passes per cell-update of one step (one read or write of
# an nx*ny*nz field = 1 pass; w counts as nz; a half-spectrum complex field
# as 1): slow halves 2 x 8, fast stages 3 x 1, projections 5 x 14 = 89, plus
# 2 (heating factors read per slow half) when heating is on.
PASSES_BASE, PASSES_HEAT = 89, 2
SAMPLE_N = 128  # horizontal size of the bounded CPU sample (full column depth)


def grid_of(w):
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    return nx, ny, nz, nx * w["dx"], ny * w["dx"], w["Lz"]


# ---------------------------------------------------------------------------
# configuration builders
# ---------------------------------------------------------------------------

def b200_integrator(w, precision, blowup_u_max=0.0):
    from oraclev8_b200.grid import LorenzStaggering
    from oraclev8_b200.production_config import BaseState
    from oraclev8_b200.solver import (AdvectionComponent, AnelasticProjection,
                                      BuoyancyComponent, CoriolisComponent,
                                      DiabaticHeatingComponent, LH82AnelasticEquationSet,
                                      OperatorConfig, RK3Integrator)
    nx, ny, nz, Lx, Ly, Lz = grid_of(w)
    base = BaseState(nz, Lz)
    kw = dict(equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
              buoyancy=BuoyancyComponent(),
              projection=AnelasticProjection(nx, ny, nz, Lx, Ly, Lz),
              advection=AdvectionComponent(nx, ny, nz, Lx, Ly, Lz, scheme="upwind5h"),
              coriolis=CoriolisComponent(Ly=Ly, ny=ny, **w["coriolis"]))
    if w["heating"]:
        kw["diabatic_heating"] = DiabaticHeatingComponent(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly,
                                                          Lz=Lz, **w["heating"])
    return RK3Integrator(OperatorConfig(**kw), base, precision=precision,
                         blowup_u_max=blowup_u_max), base


def host_initial_state(w, base):
    from oraclev8_b200.vortex_init import HollandVortexInit
    nx, ny, nz, Lx, Ly, Lz = grid_of(w)
    s = HollandVortexInit(**w["vortex"], wind_decay_top=12e3).build_state(
        nx, ny, nz, Lx, Ly, base, device=False)
    if w["noise_seed"] is not None:
        rng = np.random.default_rng(w["noise_seed"])
        s.theta_prime = s.theta_prime + rng.uniform(-0.05, 0.05, (nx, ny, nz))
    return s


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------

class Clocks:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle on a bounded sample (full column, 128 x 128 tile)
# ---------------------------------------------------------------------------

def _sample_integrator(w):
    from oracle import lh82 as O
    nx = ny = min(SAMPLE_N, w["nx"])
    nz, Lz = w["nz"], w["Lz"]
    Lx, Ly = nx * w["dx"], ny * w["dx"]
    z, rho0, th0 = O.build_base_state(nz, Lz)
    cor = dict(w["coriolis"], Ly=Ly, ny=ny)
    cfg = O.StepConfig(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz, coriolis=cor,
                       heating=w["heating"])
    s = O.Holland(**w["vortex"], wind_decay_top=12e3).build_state(nx, ny, nz, Lx, Ly, z,
                                                                   rho0, th0)
    return O.Integrator(cfg, z, rho0, th0), s, nx * ny * nz


def _worker(conn, wname):
    os.environ["OMP_NUM_THREADS"] = "1"
    integ, s, cells = _sample_integrator(WORKLOADS[wname])
    dt = WORKLOADS[wname]["dt"]
    n = 0
    while True:
        cmd = conn.recv()
        if cmd is None:
            break
        t0 = time.perf_counter()
        s, _ = integ.step(s, dt, n)
        n += 1
        conn.send(time.perf_counter() - t0)


def cpu_sample_rate(wname, procs, steps, warmup):
    """Independent sample runs, one per process; returns (cell-updates/s list,
    cells per sample)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    pipes, ps = [], []
    for _ in range(procs):
        a, b = ctx.Pipe()
        p = ctx.Process(target=_worker, args=(b, wname), daemon=True)
        p.start()
        pipes.append(a)
        ps.append(p)
    cells = sample_cells(WORKLOADS[wname])
    rates = []
    try:
        for i in range(warmup + steps):
            t0 = time.perf_counter()
            for c in pipes:
                c.send(1)
            for c in pipes:
                c.recv()
            el = time.perf_counter() - t0
            if i >= warmup:
                rates.append(procs * cells / el)
    finally:
        for c in pipes:
            try:
                c.send(None)
            except Exception:
                pass
        for p in ps:
            p.join(timeout=10)
    return rates, cells


def sample_cells(w):
    n = min(SAMPLE_N, w["nx"])
    return n * n * w["nz"]


def sample_name(w):
    n = min(SAMPLE_N, w["nx"])
    return f"{n}x{n}x{w['nz']}"


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def mem_available_gb():
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable"):
                return int(ln.split()[1]) / 1e6
    except Exception:
        pass
    return 16.0


def reference_procs():
    return max(1, min(host_cores(), 32, int(mem_available_gb() // 2)))


# ---------------------------------------------------------------------------
# per-kernel algorithmic bytes (the kernel's own I/O contract)
# ---------------------------------------------------------------------------

def kernel_bytes(w, S, fast_stages=3, slow_projections=2, shared_stages=False):
    """Algorithmic bytes per launch of each class (the mean over the step's
    launches of the class).  shared_stages: the fast stages' forward x
    transforms come from one launch over the anchor state (three spectra
    written), and each stage's y launch reads three spectra."""
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    n = nx * ny * nz
    nw = nx * ny * (nz + 1)
    ns = (nx // 2 + 1) * ny * nz  # complex half-spectrum elements
    c = 2 * S
    P = slow_projections + fast_stages
    # forward x: a slow projection reads (u, v, w), a stage (u, v, w, b_half)
    fx_slow, fx_stage = (2 * n + nw) * S + 2 * ns * c, (2 * n + 2 * nw) * S + 2 * ns * c
    if shared_stages and fast_stages:
        fx = (slow_projections * fx_slow + fx_stage + ns * c) / (slow_projections + 1)
        fy = (slow_projections * 3 * ns * c + fast_stages * 4 * ns * c) / P
    else:
        fx = (slow_projections * fx_slow + fast_stages * fx_stage) / P
        fy = 3 * ns * c
    # inverse x: the two spectra in; a slow projection reads and writes
    # (u, v, w), a fast stage reads (u, v, w, b_half) and writes (u, v, w);
    # the potential is stored only where the step keeps it (the last fast
    # stage and the last slow projection)
    phi_writes = (1 if fast_stages else 0) + (1 if slow_projections else 0)
    ix = 2 * ns * c + (slow_projections * 2 * (2 * n + nw) * S
                       + fast_stages * ((2 * n + 2 * nw) * S + (2 * n + nw) * S)
                       + phi_writes * n * S) / P
    heat = (nx * ny + nz) * 8 if w["heating"] else 0
    return {
        "fx": fx, "fy": fy, "thomas": 2 * ns * c, "iy": 3 * ns * c, "ix": ix,
        "slow": 2 * (3 * n + nw) * S + heat, "diag": (4 * n + nw) * S,
    }


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------

def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


TRAFFIC_FILE = ROOT / "profiles" / "dram_traffic_per_launch.txt"


def load_traffic(wname, precision):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
    kernel classes, captured by ncu outside this run and committed as text:
    one ``workload precision class bytes`` row per capture (``#`` comments
    give the command).  {} where the file has no row for this workload."""
    out = {}
    if not TRAFFIC_FILE.exists():
        return out
    for ln in TRAFFIC_FILE.read_text().splitlines():
        ln = ln.split("#", 1)[0].split()
        if len(ln) >= 4 and ln[0] == wname and ln[1] == precision:
            out[ln[2]] = float(ln[3])
    return out


def bench_config(args, w, world):
    """The ``config`` object of both arms' lines (identical, so that the
    reference arm times the same named workload)."""
    return {"workload": f"{args.workload}: {w['nx']}x{w['ny']}x{w['nz']} LH82 RK3 step, "
                        f"WS5 + beta-plane + buoyancy + projection"
                        + (" + heating" if w["heating"] else "")
                        + (f", u_env={w['coriolis']['u_env']} m/s" if w["coriolis"].get("u_env")
                           else "") + f", dt={w['dt']}s",
            "precision": args.precision, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (every state field > 126 MB)"}


def max_over_ranks(vals, device):
    """Element-wise maximum of `vals` over the ranks of the default process
    group (the slowest replica's time); the values themselves at one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(x) for x in vals]
    t = torch.tensor([float(x) for x in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def _timed_steps(integ, st, dt, steps, warmup, barrier):
    """W untimed steps, then K steps bracketed by barrier + synchronize and
    timed with CUDA events on the launching stream; per-class kernel times
    from the plan's own launch events."""
    import torch
    for _ in range(warmup):
        integ.step_(st, dt, want_diag=True)
    torch.cuda.synchronize()
    plan = integ.plan
    plan.profile(True)
    l0 = plan.launches
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        integ.step_(st, dt, want_diag=True)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = plan.launches - l0
    prof = plan.profile_read()
    plan.profile(False)
    if not bool(torch.isfinite(st.u).all()):
        raise RuntimeError("non-finite state after the timed steps")
    return ms, launches, prof


def _non_nyquist_max(d):
    """max |d| after removing the Nyquist rows of the horizontal spectrum
    (measurement only; the spectral derivative of the reference cannot act
    on them)."""
    import torch
    nx, ny = d.shape[:2]
    D = torch.fft.fft2(d, dim=(0, 1))
    D[nx // 2] = 0
    D[:, ny // 2] = 0
    return float(torch.fft.ifft2(D, dim=(0, 1)).real.abs().max())


def _precision_report(st, st64, plan64):
    """Per-field error of a single-precision run against the FP64 run from the
    same initial state and step count (max |a - b| / max |b|), and the FP64
    evaluation of the post-step anelastic divergence of both."""
    fields = ("u", "v", "w", "theta_prime", "projection_potential")
    err = {}
    for f in fields:
        a, b = getattr(st, f).double(), getattr(st64, f)
        err[f] = float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))
    d32 = plan64.divergence(st.u.double(), st.v.double(), st.w.double())
    d64 = plan64.divergence(st64.u, st64.v, st64.w)
    return {"rel_err_vs_fp64": err,
            "divergence_non_nyquist_max": {"this": _non_nyquist_max(d32),
                                           "fp64": _non_nyquist_max(d64)},
            "divergence_max": {"this": float(d32.abs().max()), "fp64": float(d64.abs().max())}}


def run_b200(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    w = WORKLOADS[args.workload]
    from oraclev8_b200.solver import State
    integ, base = b200_integrator(w, args.precision)
    hs = host_initial_state(w, base)
    dt = w["dt"]
    dtype = integ.dtype
    S = 8 if args.precision == "fp64" else 4
    dev = torch.device("cuda", torch.cuda.current_device())

    def to_dev(a, dt_=None):
        return torch.as_tensor(a, dtype=dt_ or dtype).to(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    st = State(to_dev(hs.u), to_dev(hs.v), to_dev(hs.w), to_dev(hs.theta_prime),
               to_dev(hs.projection_potential), 0.0)
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    ms, launches, prof = _timed_steps(integ, st, dt, args.steps, args.warmup, barrier)
    companion = None
    if args.precision != "fp64" and not args.no_fp64_companion:
        # the plain FP64 step on the same workload, timed the same way, and the
        # error of this run against it after the same number of steps
        integ64, _ = b200_integrator(w, "fp64")
        f64 = torch.float64
        st64 = State(to_dev(hs.u, f64), to_dev(hs.v, f64), to_dev(hs.w, f64),
                     to_dev(hs.theta_prime, f64), to_dev(hs.projection_potential, f64), 0.0)
        ms64, _, _ = _timed_steps(integ64, st64, dt, args.steps, args.warmup, barrier)
        companion = (ms64, _precision_report(st, st64, integ64.plan))
        del st64, integ64
    production = None
    if not args.no_production:
        production = production_report(args, w, hs, barrier, dev, load_peaks()[0])
    clk = clocks.stop()
    red = max_over_ranks([ms] + ([companion[0]] if companion else []), dev)
    ms = red[0]
    if companion:
        companion = (red[1], companion[1])
    cells = w["nx"] * w["ny"] * w["nz"]
    value = world * cells * args.steps / (ms / 1e3)

    # ---- e2e through the public API with host buffers ---------------------
    # Every step: its input state copied from pinned host memory, one public
    # RK3Integrator.step, its output state copied back to pinned host memory.
    # The copies of neighbouring steps overlap the step on the device (inputs
    # on a copy-in stream into two alternating device sets, outputs on a
    # copy-out stream); the steps themselves run in order on one stream, as
    # they share the plan's scratch.
    fields = (st.u, st.v, st.w, st.theta_prime, st.projection_potential)
    pinned = [torch.empty(tuple(x.shape), dtype=dtype, pin_memory=True) for x in fields]
    outs = [[torch.empty_like(p, pin_memory=True) for p in pinned] for _ in range(2)]
    for p, x in zip(pinned, fields):
        p.copy_(x)
    h2d = sum(p.numel() * p.element_size() for p in pinned)
    devsets = [[torch.empty_like(x) for x in fields] for _ in range(2)]
    comp = torch.cuda.current_stream()
    cin, cout = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_used = [torch.cuda.Event() for _ in range(2)]
    k_e2e = args.steps

    def h2d_into(j):
        with torch.cuda.stream(cin):
            for d_, p in zip(devsets[j], pinned):
                d_.copy_(p, non_blocking=True)
            ev_in[j].record(cin)

    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h2d_into(0)
    for i in range(k_e2e):
        j = i % 2
        if i + 1 < k_e2e:
            if i >= 1:
                cin.wait_event(ev_used[1 - j])  # step i-1 has finished reading that set
            h2d_into(1 - j)
        comp.wait_event(ev_in[j])
        s_out, diag = integ.step(State(*devsets[j], 0.0), dt, step_number=i)
        ev_used[j].record(comp)
        cout.wait_stream(comp)
        with torch.cuda.stream(cout):
            for o, x in zip(outs[j], (s_out.u, s_out.v, s_out.w, s_out.theta_prime,
                                      s_out.projection_potential)):
                x.record_stream(cout)
                o.copy_(x, non_blocking=True)
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    t_e2e = max_over_ranks([t_e2e], dev)[0]
    e2e = world * cells * k_e2e / t_e2e

    # ---- roofline of the dominant kernel ------------------------------------
    peak, peak_kind = load_peaks()
    kb = kernel_bytes(w, S, shared_stages=bool(integ.plan.variants().get("zc4_fxsh")))
    dom = max((c for c in prof if prof[c][1] > 0 and c in kb), key=lambda c: prof[c][0])
    dms, dn = prof[dom]
    ach = kb[dom] / (dms / dn / 1e3) / 1e9
    traffic = load_traffic(args.workload, args.precision).get(dom)
    cufft = None
    if not args.no_cufft and rank == 0:
        cufft = cufft_report(w, args.precision, dev, {c: prof[c][0] for c in prof}, args.steps)
    passes = PASSES_BASE + (PASSES_HEAT if w["heating"] else 0)
    step_gbs = passes * S * cells * args.steps / (ms / 1e3) / 1e9
    line = {
        "metric": "cell-updates/s (RK3 step)",
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32 (f64 residual)" if
        args.precision == "fp32r" else "f32",
        "data": "synthetic (seeded Holland vortex + theta' noise; no dataset in the reference)",
        "config": bench_config(args, w, world),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak,
                     "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                     "traffic": traffic,
                     "traffic_source": ("ncu capture outside this run "
                                        "(profiles/dram_traffic_per_launch.txt)"
                                        if traffic is not None else None),
                     "bytes_per_launch": kb[dom], "avg_launch_ms": dms / dn},
        "step_roofline": {"passes_per_cell": passes, "achieved": step_gbs, "peak": peak,
                          "unit": "GB/s", "frac": step_gbs / peak},
        # every kernel class against the same peak: algorithmic bytes per
        # launch / mean launch time (classes with a byte model only)
        "kernel_rooflines": {c: {"achieved_gbs": kb[c] / (prof[c][0] / prof[c][1] / 1e3) / 1e9,
                                 "frac": kb[c] / (prof[c][0] / prof[c][1] / 1e3) / 1e9 / peak,
                                 "launches_per_step": prof[c][1] / args.steps}
                             for c in kb if c in prof and prof[c][1] > 0},
        "kernels_ms_per_step": {c: prof[c][0] / args.steps for c in prof if prof[c][1]},
        "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": h2d + 8 * 6,
                "note": "public RK3Integrator.step per step: full state H2D from pinned host, "
                        "step, StepDiagnostics, full state D2H to pinned host; copies of "
                        "neighbouring steps overlap the step (copy-in/copy-out streams)"},
        "gpu_launches": launches,
        "kernel_variants": {k: v for k, v in integ.plan.variants().items() if v},
        "clocks": clk,
    }
    if cufft is not None:
        line["cufft"] = cufft
    if production is not None:
        line["production"] = production
    if rank == 0 and world == 1 and not args.no_diagnostics:
        line["diagnostics"] = diagnostics_report(w, st, base)
        line["snapshot"] = snapshot_report(integ, st, dt)
    if not args.no_ensemble:
        ens = ensemble_report(args, load_peaks()[0])
        if rank == 0:
            line["ensemble"], line["serving"] = ens
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rates, sc = cpu_sample_rate(args.workload, 1, 1, 1)
        line["cpu_baseline"] = {
            "value": statistics.median(rates), "unit": "cell-updates/s", "cores": 1,
            "kind": "port",
            "sample": f"oracle (NumPy restatement of the reference, FP64) on "
                      f"{sample_name(w)} (the workload's column depth and physics on a "
                      f"smaller horizontal tile at the same dx), 1 warm-up + "
                      f"1 timed step, 1 process"}
    # the FP32-refined / FP64 comparison last, where a truncated log keeps it
    if companion:
        v64 = world * cells * args.steps / (companion[0] / 1e3)
        line["accuracy"] = dict(companion[1], after_steps=args.warmup + args.steps,
                                note="this run vs the FP64 run from the same initial state; "
                                     "divergence = anelastic divergence evaluated in FP64")
        line["fp64_plain"] = {"value": v64, "unit": "cell-updates/s",
                              "ms_per_step": companion[0] / args.steps,
                              "ratio": value / v64,
                              "note": "plain FP64 step on the same workload and GPU, timed "
                                      "the same way (W warm-up + K timed steps)"}
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def production_report(args, w, hs, barrier, dev, peak_gbs):
    """The reference's production physics on the bench grid.

    build_production_config (centred advection, beta-plane Coriolis,
    biharmonic diffusion, Helmholtz divergence damping, Newtonian cooling,
    surface drag, projection; no buoyancy) stepped on the workload's grid and
    initial state, with the intensity cap added after every step as the
    reference's run loop does (run_storm.py:168-172).  A step here is
    ``RK3Integrator.step_`` + the cap's tendency + the two in-place updates.
    Timed in the bench's precision and in plain FP64, W warm-up + K steps
    each, with CUDA events on the launching stream."""
    import torch
    from oraclev8_b200.production_config import (TAU_CAP, VMAX_CAP_MS, BaseState,
                                                 build_production_config)
    from oraclev8_b200.solver import IntensityCapComponent, RK3Integrator, State
    nx, ny, nz, Lx, Ly, Lz = grid_of(w)
    f0 = w["coriolis"]["f"]
    u_env, v_env = w["coriolis"].get("u_env", 0.0), w["coriolis"].get("v_env", 0.0)
    base = BaseState(nz, Lz)
    cfg = build_production_config(nx, ny, nz, Lx, Ly, Lz, f0, u_env, v_env)
    cap = IntensityCapComponent(v_cap=VMAX_CAP_MS, tau=TAU_CAP, u_env=u_env, v_env=v_env)
    dt = w["dt"]
    runs = {}
    precs = [args.precision] + (["fp64"] if args.precision != "fp64" else [])
    for prec in precs:
        integ = RK3Integrator(cfg, base, precision=prec)
        ty = integ.dtype
        st = State(*(torch.as_tensor(a, dtype=ty).to(dev) for a in
                     (hs.u, hs.v, hs.w, hs.theta_prime, hs.projection_potential)), 0.0)

        def one():
            integ.step_(st, dt, want_diag=True)
            ct = cap.compute_tendency(st, None, None, base, dt)
            st.u.add_(ct.du_dt, alpha=dt)
            st.v.add_(ct.dv_dt, alpha=dt)

        for _ in range(args.warmup):
            one()
        torch.cuda.synchronize()
        plan = integ.plan
        plan.profile(True)
        l0 = plan.launches
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            one()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks([e0.elapsed_time(e1)], dev)[0]
        prof = plan.profile_read()
        plan.profile(False)
        if not bool(torch.isfinite(st.u).all()):
            raise RuntimeError("non-finite state after the production steps")
        # the library's launches plus one intensity-cap kernel per step
        runs[prec] = (ms, plan.launches - l0 + args.steps, prof, st, integ)
    ms, launches, prof, st, _ = runs[args.precision]
    S = 8 if args.precision == "fp64" else 4
    n = nx * ny * nz
    nw = nx * ny * (nz + 1)
    # per slow half: the inner Laplacians (read u, v; write Lu, Lv) and the
    # fused slow kernel (read u, v, w, theta', the damper's Du, Dv and Lu, Lv;
    # write u, v, w, theta')
    slow_bytes = 2 * ((2 * (3 * n + nw) + 4 * n) * S + 4 * n * S)
    slow_ms = prof["slow"][0] / args.steps
    cells = n * args.steps
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rep = {
        "workload": f"production physics (build_production_config: centred advection, "
                    f"beta-plane, nu4 3e11 biharmonic, Helmholtz damping 0.5, cooling 1800 s, "
                    f"drag Cd 1.5e-3 / 1 km, projection, no buoyancy) on the {nx}x{ny}x{nz} "
                    f"grid and initial state, intensity cap 70 m/s / 300 s after each step, "
                    f"dt={dt}s",
        "precision": args.precision,
        "value": world * cells / (ms / 1e3), "unit": "cell-updates/s",
        "ms_per_step": ms / args.steps,
        "gpu_launches": launches,
        "kernels_ms_per_step": {c: prof[c][0] / args.steps for c in prof if prof[c][1]},
        "slow_roofline": {"bound": "hbm", "bytes_per_step": slow_bytes,
                          "achieved": slow_bytes / (slow_ms / 1e3) / 1e9, "peak": peak_gbs,
                          "unit": "GB/s", "frac": slow_bytes / (slow_ms / 1e3) / 1e9 / peak_gbs},
    }
    if "fp64" in runs and args.precision != "fp64":
        ms64, _, _, st64, integ64 = runs["fp64"]
        rep["fp64_plain"] = {"value": world * cells / (ms64 / 1e3), "unit": "cell-updates/s",
                             "ms_per_step": ms64 / args.steps, "ratio": ms64 / ms}
        rep["accuracy"] = dict(_precision_report(st, st64, integ64.plan),
                               after_steps=args.warmup + args.steps)
    return rep


def diagnostics_report(w, st, base, reps=20, cpu_reps=3):
    """The vortex diagnostics read-outs on the bench state (device fields of
    the timed run): ``compute_diagnostics`` and the sub-cell refinement,
    each a synchronous API call (kernels + the host's scalar logic + the
    copies of the scalars), median wall time of ``reps`` calls after two
    warm-up calls; beside them the oracle (NumPy, one core) on the same
    state, median of ``cpu_reps`` calls."""
    import torch
    from oracle import vortex_diag as VD
    from oraclev8_b200 import diagnostics as D
    nx, ny, nz, Lx, Ly, Lz = grid_of(w)
    dx = Lx / nx
    cx, cy = 0.5 * Lx, 0.5 * Ly
    u_env, v_env = w["coriolis"].get("u_env", 0.0), w["coriolis"].get("v_env", 0.0)

    def dev_call():
        d = D.compute_diagnostics(st, base, cx, cy, dx, dx, u_env, v_env, theta_xy_m=(cx, cy))
        return d, D.subcell_refine(st, d["xv_m"], d["yv_m"], dx)

    def med(fn, n):
        ts = []
        for _ in range(n):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts) * 1e3, out

    for _ in range(2):
        dev_call()
    ms, (d, xy) = med(dev_call, reps)
    u = st.u.double().cpu().numpy()
    v = st.v.double().cpu().numpy()
    z = np.asarray(base.z)

    def cpu_call():
        dd = VD.compute_diagnostics(u, v, z, cx, cy, dx, dx, u_env, v_env, theta_xy_m=(cx, cy))
        return dd, VD.subcell_refine(u, v, dd["xv_m"], dd["yv_m"], dx)

    cms, (dref, xyref) = med(cpu_call, cpu_reps)
    return {"calls": "compute_diagnostics + subcell_refine (one diagnostics read-out)",
            "ms_per_readout": ms, "cpu_oracle_ms_per_readout": cms, "cpu_cores": 1,
            "speedup_vs_cpu_oracle": cms / ms,
            "centre_equal_to_oracle": (d["xv_m"], d["yv_m"]) == (dref["xv_m"], dref["yv_m"]),
            "subcell_max_abs_diff_m": float(max(abs(a - b) for a, b in zip(xy, xyref)))}


def snapshot_report(integ, st, dt, steps=12, every=4):
    """Checkpoint cost on the bench state: one synchronous snapshot (device
    to pinned host, median of 5), and ``steps`` public steps with an
    asynchronous snapshot of every ``every``-th state on a side stream
    (each step writes a new state, so the copy overlaps the next steps)
    against the same steps without snapshots; device time with CUDA events."""
    import torch
    from oraclev8_b200 import snapshot as S
    nbytes = sum(getattr(st, f).numel() * getattr(st, f).element_size() for f in S.FIELDS)
    ts = []
    for _ in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S.take_snapshot(st)
        ts.append(time.perf_counter() - t0)
    sync_ms = statistics.median(ts) * 1e3
    side = torch.cuda.Stream()
    pinned = {}

    def run(with_snaps):
        s = st
        copies = []
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for n in range(steps):
            s, _ = integ.step(s, dt, n)
            if with_snaps and (n + 1) % every == 0:
                if copies:
                    copies[-1].result()  # the pinned buffers are reused
                copies.append(S.SnapshotCopy(s, step=n + 1, stream=side, pinned=pinned))
                if not pinned:
                    pinned.update(copies[-1].host)
        e1.record(stream)
        for c in copies:
            c.result()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    run(False)
    base_ms = run(False)
    snap_ms = run(True)
    return {"state_bytes": nbytes, "sync_snapshot_ms": sync_ms,
            "sync_snapshot_gbs": nbytes / (sync_ms / 1e3) / 1e9,
            "steps": steps, "snapshot_every": every,
            "ms_per_step_without": base_ms / steps, "ms_per_step_with_async": snap_ms / steps,
            "note": "async snapshots copy on a side stream into reused pinned buffers while "
                    "the next steps run"}


# the step's components of the ensemble and serving draws
PHYSICS_TEXT = {
    "lh82": "WS5 + beta-plane + buoyancy + projection (LH82 physics)",
    "production": ("production physics (build_production_config: centred advection, "
                   "beta-plane, nu4 biharmonic, Helmholtz damping, cooling, drag, projection; "
                   "no steering wind, no intensity cap)"),
}


def ensemble_report(args, peak_gbs):
    """Ensemble and serving measurements through ``oraclev8_b200.serving``.

    Ensemble: ``--ensemble-runs`` draws of the mixed ensemble (seed 3), each
    ``--ensemble-hours`` long at its CFL time step, FP32-refined, all arriving
    at once; against the same runs served one at a time in plain FP64 through
    ``RK3Integrator.step``.  Serving: ``--serving-requests`` Poisson arrivals
    at 2/s (seed 4), run length U(6, 72) h divided by ``--serving-scale``,
    80% FP32-refined / 20% FP64, 150 GB HBM budget; against the same stream
    served serially in plain FP64."""
    import torch.distributed as dist
    from oraclev8_b200.serving import (RunRequest, ServingEngine, draw_requests,
                                       gather_records, serve_serial_plain, shard_requests,
                                       summarize)
    rank = dist.get_rank() if dist.is_available() and dist.is_initialized() else 0
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    # library, kernels, kernel-form tuning of every grid and the plan pool
    # warm before timing
    ph = args.ensemble_physics
    every = (draw_requests(args.ensemble_runs, 3, hours=args.ensemble_hours, physics=ph)
             + draw_requests(args.serving_requests, 4, rate=2.0, fp32r_frac=0.8, physics=ph))
    ServingEngine.prepare_kernels(every)
    ServingEngine.prepare_kernels([RunRequest(**{**r.__dict__, "precision": "fp64"})
                                   for r in every])
    ServingEngine(realtime=False).run(draw_requests(6, 99, hours=0.2, fp32r_frac=0.5, physics=ph))
    serve_serial_plain(draw_requests(2, 98, hours=0.1, physics=ph), realtime=False)
    # N > 1: whole runs are dealt to the GPUs (no exchange between runs)
    reqs = draw_requests(args.ensemble_runs, 3, hours=args.ensemble_hours, physics=ph)
    mine = shard_requests(reqs, rank, world)
    eng = gather_records(ServingEngine(realtime=False).run(mine))
    ser = gather_records(serve_serial_plain(mine, realtime=False))
    if eng is None:  # not rank 0
        r4 = shard_requests(draw_requests(args.serving_requests, 4,
                                          hours=(6.0 / args.serving_scale,
                                                 72.0 / args.serving_scale),
                                          rate=2.0, fp32r_frac=0.8, physics=ph), rank, world)
        gather_records(ServingEngine(hbm_budget=150e9, realtime=True).run(r4))
        gather_records(serve_serial_plain(r4, realtime=True))
        return None
    eng, ser = summarize(eng), summarize(ser)
    passes = PASSES_BASE  # no heating in the ensemble draws (the production terms not counted)
    ens = {
        "workload": f"{len(reqs)} runs drawn from the mixed ensemble (seed 3), dealt to "
                    f"{world} GPU(s): nx=ny in "
                    f"{{96,128,192,256,384}} at dx 10 km, nz in {{32,48,64}} over 16 km, "
                    f"Vmax U(25,65), Rmax U(20,80) km, B U(1,2), lat U(10,30)N; "
                    f"{args.ensemble_hours:g} h each at dt = 0.8 dx / Vmax; {PHYSICS_TEXT[ph]}; "
                    f"all arrive at t = 0",
        "precision": "fp32r", "engine": eng, "serial_plain_fp64": ser,
        "throughput_ratio_vs_serial_plain": eng["cell_updates_per_s"] / ser["cell_updates_per_s"],
        "roofline": {"bound": "hbm", "passes_per_cell": passes, "bytes_per_cell": passes * 4,
                     "achieved": passes * 4 * eng["cell_updates_per_s"] / 1e9, "peak": peak_gbs,
                     "unit": "GB/s",
                     "frac": passes * 4 * eng["cell_updates_per_s"] / 1e9 / peak_gbs}}
    r4 = shard_requests(draw_requests(args.serving_requests, 4,
                                      hours=(6.0 / args.serving_scale, 72.0 / args.serving_scale),
                                      rate=2.0, fp32r_frac=0.8, physics=ph), rank, world)
    eng4 = summarize(gather_records(ServingEngine(hbm_budget=150e9, realtime=True).run(r4)))
    ser4 = summarize(gather_records(serve_serial_plain(r4, realtime=True)))
    serving = {
        "workload": f"{len(r4)} requests, Poisson arrivals at 2/s (seed 4), ensemble draws, "
                    f"run length U(6,72) h / {args.serving_scale:g}, 80% fp32r / 20% fp64, "
                    f"{PHYSICS_TEXT[ph]}, 150 GB HBM admission budget",
        "engine": eng4, "serial_plain_fp64": ser4,
        "p99_ratio_serial_over_engine": ser4["latency_s"]["p99"] / eng4["latency_s"]["p99"]}
    return ens, serving


def cufft_report(w, precision, dev, kernels_ms, steps, projections=5, reps=5):
    """cuFFT through torch.fft doing the transforms of one projection on the
    workload's grid: R2C along x of three real fields, C2C along y of two of
    the results, the two inverse y transforms and three C2R along x (the
    transform count of this library's pencils), in the step's arithmetic
    precision, timed with CUDA events on the current stream (median of
    ``reps`` after a warm-up).  Beside it, this library's pencil classes per
    projection (fx + fy + iy + ix from the timed steps), which also do the
    projection's arithmetic and its state reads and writes."""
    import torch
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    dt = torch.float64 if precision == "fp64" else torch.float32
    g = torch.Generator(device=dev).manual_seed(5)
    f = [torch.randn(nx, ny, nz, dtype=dt, device=dev, generator=g) for _ in range(3)]

    def once():
        X = [torch.fft.rfft(a, dim=0) for a in f]
        Y = [torch.fft.fft(X[0], dim=1), torch.fft.fft(X[1], dim=1)]
        Z = [torch.fft.ifft(Y[0], dim=1), torch.fft.ifft(Y[1], dim=1)]
        return [torch.fft.irfft(Z[0], n=nx, dim=0), torch.fft.irfft(Z[1], n=nx, dim=0),
                torch.fft.irfft(X[2], n=nx, dim=0)]

    once()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        out = once()
        e1.record(st)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
        del out
    del f
    torch.cuda.empty_cache()
    ours = sum(kernels_ms.get(c, 0.0) for c in ("fx", "fy", "iy", "ix")) / steps / projections
    cu = statistics.median(ts)
    return {"what": "3 R2C x + 2 C2C y + 2 inverse C2C y + 3 C2R x (one projection's "
                    "transforms), torch.fft (cuFFT) on (nx, ny, nz) z-contiguous fields",
            "precision": "fp64" if precision == "fp64" else "fp32",
            "cufft_ms_per_projection": cu,
            "pencils_ms_per_projection": ours,
            "pencils_note": "fx + fy + iy + ix kernel classes of the timed steps / projections; "
                            "they also form the divergence, read and correct the state",
            "ratio_cufft_over_pencils": cu / ours if ours > 0 else None}


def _hour_chunk(steps_per_hour, cap=24):
    return max(c for c in range(1, cap + 1) if steps_per_hour % c == 0)


def track_report(args):
    """The workload run for ``--track-hours`` hours in FP32-refined and in
    plain FP64 on this GPU, with the hourly storm centre of each
    (find_storm_centre chained through last_pos / last_raw_pos, with the
    background flow, as run_storm.py:180-190 does), the hourly max|w| and, at
    the end, the per-field error of the FP32-refined run against the FP64 run
    and the FP64-evaluated non-Nyquist divergence of both.  The steps run as
    captured step graphs of a whole number of steps per hour."""
    import torch
    from oraclev8_b200.solver import State
    from oraclev8_b200.storm_tracker import find_storm_centre
    torch.cuda.set_device(0)
    w = WORKLOADS[args.workload]
    nx, ny, nz, Lx, Ly, Lz = grid_of(w)
    dx = Lx / nx
    dt = w["dt"]
    sph = int(round(3600.0 / dt))
    chunk = _hour_chunk(sph)
    u_env = w["coriolis"].get("u_env", 0.0)
    v_env = w["coriolis"].get("v_env", 0.0)
    prod = args.track_physics == "production"
    runs = {}
    hs = None
    for prec in ("fp64", "fp32r"):
        if prod:
            # the reference's production physics (build_production_config) with
            # the intensity cap added after every step (run_storm.py:146-172)
            from oraclev8_b200.production_config import (TAU_CAP, VMAX_CAP_MS, BaseState,
                                                         build_production_config)
            from oraclev8_b200.solver import IntensityCapComponent, RK3Integrator
            base = BaseState(nz, Lz)
            integ = RK3Integrator(build_production_config(nx, ny, nz, Lx, Ly, Lz,
                                                          w["coriolis"]["f"], u_env, v_env),
                                  base, precision=prec, blowup_u_max=400.0)
            cap = IntensityCapComponent(v_cap=VMAX_CAP_MS, tau=TAU_CAP, u_env=u_env,
                                        v_env=v_env)
        else:
            integ, base = b200_integrator(w, prec, blowup_u_max=400.0)
            cap = None
        if hs is None:
            hs = host_initial_state(w, base)
        ty = integ.dtype
        st = State(*(torch.as_tensor(a, dtype=ty).cuda() for a in
                     (hs.u, hs.v, hs.w, hs.theta_prime, hs.projection_potential)), 0.0)
        runs[prec] = dict(integ=integ, base=base, st=st, cap=cap, last=None, last_raw=None,
                          fixes=[], graph=None if prod else integ.capture(st, dt, chunk))

    def advance_hour(r):
        if r["graph"] is not None:
            for _ in range(sph // chunk):
                r["graph"].launch()
            return
        st = r["st"]
        for _ in range(sph):
            r["integ"].step_(st, dt)
            ct = r["cap"].compute_tendency(st, None, None, r["base"], dt)
            st.u.add_(ct.du_dt, alpha=dt)
            st.v.add_(ct.dv_dt, alpha=dt)
    hours = int(args.track_hours)
    t0 = time.perf_counter()
    for h in range(hours + 1):
        for prec, r in runs.items():
            if r.get("blew_h") is not None:
                continue
            if h > 0:
                advance_hour(r)
            mu = float(r["st"].u.abs().max())
            # a state that is no longer finite (or past the blow-up speed) has
            # no storm centre: the run stops there, as the reference's harness
            # stops it (measure_lh82_phase3.py:129-130)
            if not math.isfinite(mu) or mu > 400.0:
                r["blew_h"] = h
                continue
            (x, y), m, d = find_storm_centre(r["st"], r["base"], nx, ny, dx,
                                             last_pos=r["last"], u_env_ms=u_env,
                                             v_env_ms=v_env, dt_output_s=3600.0,
                                             return_diag=True, last_raw_pos=r["last_raw"])
            r["last"], r["last_raw"] = (x, y), d["theta_raw_m"]
            r["fixes"].append(dict(x=x, y=y, method=m, max_w=float(r["st"].w.abs().max()),
                                   max_u=mu))
        print(f"hour {h}: " + ", ".join(
            f"{p} max|u| {r['fixes'][-1]['max_u']:.2f}" if r.get("blew_h") is None
            else f"{p} blew up by hour {r['blew_h']}" for p, r in runs.items()),
            file=sys.stderr, flush=True)
        if all(r.get("blew_h") is not None for r in runs.values()):
            break
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    f64, f32 = runs["fp64"]["fixes"], runs["fp32r"]["fixes"]
    rows = []
    for h, (a, b) in enumerate(zip(f32, f64)):
        rows.append(dict(h=h, dist_m=float(math.hypot(a["x"] - b["x"], a["y"] - b["y"])),
                         max_w_rel=abs(a["max_w"] - b["max_w"]) / max(b["max_w"], 1e-30),
                         method_fp32r=a["method"], method_fp64=b["method"],
                         x_fp64_km=b["x"] / 1e3, y_fp64_km=b["y"] / 1e3))
    st32, st64 = runs["fp32r"]["st"], runs["fp64"]["st"]
    both_finite = all(r.get("blew_h") is None for r in runs.values())
    rep = _precision_report(st32, st64, runs["fp64"]["integ"].plan) if both_finite else None
    line = {"track": {
        "workload": f"{args.workload}: {nx}x{ny}x{nz}, dt={dt}s, {hours} h = {hours * sph} steps "
                    f"in each precision, "
                    + ("production physics (build_production_config) + intensity cap per step"
                       if prod else f"the workload's physics, step graphs of {chunk} steps"),
        "hours_compared": len(rows) - 1,
        "blew_up_by_hour": {p: r.get("blew_h") for p, r in runs.items()},
        "hours": rows,
        "max_centre_diff_m": max(r["dist_m"] for r in rows),
        "max_w_rel_diff_max": max(r["max_w_rel"] for r in rows),
        "fp64_track_km": [(round(r["x_fp64_km"], 3), round(r["y_fp64_km"], 3)) for r in rows],
        "final": rep,
        "blowup_flag": {p: runs[p]["integ"].plan.blown_up() for p in runs},
        "wall_s": wall}}
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    procs = reference_procs()
    rates, sc = cpu_sample_rate(args.workload, procs, args.steps, args.warmup)
    v = statistics.median(rates)
    cells = w["nx"] * w["ny"] * w["nz"]
    line = {
        "impl": "reference",
        "metric": "cell-updates/s (RK3 step)",
        "value": v,
        "unit": "cell-updates/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": cells / v * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(args, w, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": procs, "kind": "port",
                         "sample": f"{procs} independent oracle runs (NumPy restatement of the "
                                   f"reference, FP64), each {sample_name(w)} (the "
                                   f"workload's column depth on a smaller horizontal tile) "
                                   f"with the workload's physics; one step per process per "
                                   f"bench step"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp32r", choices=["fp64", "fp32", "fp32r"])
    ap.add_argument("--workload", default="config2", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-production", action="store_true",
                    help="skip the production-physics leg")
    ap.add_argument("--no-diagnostics", action="store_true",
                    help="skip the vortex-diagnostics read-out timing")
    ap.add_argument("--no-fp64-companion", action="store_true",
                    help="skip the plain-FP64 timing and accuracy report (profiling runs)")
    ap.add_argument("--ensemble-runs", type=int, default=64)
    ap.add_argument("--ensemble-hours", type=float, default=6.0)
    # the LH82 draws blow up within hours in the reference's own algorithm, so
    # the default measures the physics that stays finite
    ap.add_argument("--ensemble-physics", choices=sorted(PHYSICS_TEXT), default="production")
    ap.add_argument("--serving-requests", type=int, default=32)
    ap.add_argument("--serving-scale", type=float, default=4.0)
    ap.add_argument("--track-hours", type=float, default=0.0,
                    help="run the FP32-refined vs FP64 hourly track comparison instead")
    ap.add_argument("--track-physics", default="workload", choices=["workload", "production"],
                    help="physics of the track comparison: the workload's (LH82 WS5 + buoyancy) "
                         "or the reference's production configuration")
    ap.add_argument("--no-cufft", action="store_true", help="skip the cuFFT comparison")
    args = ap.parse_args()
    if args.track_hours > 0:
        track_report(args)
        return
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
