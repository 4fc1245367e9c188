"""Ensemble and serving loop for many independent vortex runs on one GPU.

The runs come from a request stream (vortex parameters, grid, run length,
precision).  Each run keeps its whole state and its plan resident in HBM from
admission to retirement.  Its steps are recorded once as a CUDA graph of
``chunk`` steps (``RK3Integrator.capture``) and replayed on the run's own
stream, so runs of different sizes overlap on the device.  Admission is by
HBM footprint against a budget; finished runs retire and free their slot for
the next queued request (continuous batching).  Resident runs are fed
shortest-remaining-work first, as many at a time as it takes to fill the GPU.
Per run the loop records arrival, admission and completion times; the summary
gives p50/p95/p99 time-to-completion, queueing delay and aggregate
cell-updates/s.

Request distributions (vortex parameters, grids and CFL time step) follow the
ensemble and serving workloads of the LH82 beta-drift study:
nx = ny in {96, 128, 192, 256, 384} at dx = 10 km, nz in {32, 48, 64} over
16 km, Vmax ~ U(25, 65) m/s, Rmax ~ U(20, 80) km, B ~ U(1, 2), latitude ~
U(10, 30) N giving f0 = 2 Omega sin(lat) and beta = 2 Omega cos(lat) / R
(tendency.py:1160-1164), dt = 0.8 dx / Vmax (run_storm.py:91) rounded down so
that an integer number of steps fills the run.
"""
from __future__ import annotations

import math
import queue as _queue
import threading
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from .snapshot import SnapshotCopy

OMEGA = 7.2921e-5
R_EARTH = 6.371e6
SIZES = (96, 128, 192, 256, 384)
LEVELS = (32, 48, 64)


@dataclass
class RunRequest:
    rid: int
    n: int                  # nx = ny
    nz: int
    vmax: float
    rmax: float
    b: float
    lat_deg: float
    hours: float
    precision: str = "fp32r"  # "fp64" or "fp32r"
    arrival_s: float = 0.0
    dx: float = 10e3
    lz: float = 16e3
    resume: Optional[dict] = None  # snapshot (oraclev8_b200.snapshot) to continue from
    cfl: float = 0.8               # advective CFL number of the time step
    # "lh82": WS5 advection, beta-plane, buoyancy, projection; "production": the
    # reference's build_production_config (centred advection, beta-plane,
    # biharmonic diffusion, divergence damping, cooling, drag, projection)
    physics: str = "lh82"

    @property
    def start_step(self) -> int:
        return int(self.resume.get("step", 0)) if self.resume is not None else 0

    @property
    def f0(self) -> float:
        return 2.0 * OMEGA * math.sin(math.radians(self.lat_deg))

    @property
    def beta(self) -> float:
        return 2.0 * OMEGA * math.cos(math.radians(self.lat_deg)) / R_EARTH

    @property
    def nsteps(self) -> int:
        return max(1, math.ceil(self.hours * 3600.0 / (self.cfl * self.dx / self.vmax) - 1e-9))

    @property
    def dt(self) -> float:
        return self.hours * 3600.0 / self.nsteps

    @property
    def cells(self) -> int:
        return self.n * self.n * self.nz

    @property
    def cell_updates(self) -> int:
        return self.cells * self.nsteps


def draw_requests(count: int, seed: int, hours=24.0, precision="fp32r", rate: float = 0.0,
                  fp32r_frac: float = 1.0, cfl: float = 0.8,
                  physics: str = "lh82") -> "list[RunRequest]":
    """``count`` requests from a seeded stream.  ``hours``: a fixed run length
    or a (lo, hi) uniform range.  ``rate`` > 0 gives Poisson arrivals at that
    many requests per second (else all arrive at 0); ``fp32r_frac`` < 1 tags
    that fraction FP32-refined and the rest FP64 (``precision`` ignored).
    ``cfl``: dt = cfl dx / Vmax (0.8 in the ensemble and serving workloads).
    ``physics``: the step's components, as ``RunRequest.physics``."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for i in range(count):
        n = int(rng.choice(SIZES))
        nz = int(rng.choice(LEVELS))
        vmax = float(rng.uniform(25.0, 65.0))
        rmax = float(rng.uniform(20e3, 80e3))
        b = float(rng.uniform(1.0, 2.0))
        lat = float(rng.uniform(10.0, 30.0))
        h = float(rng.uniform(*hours)) if isinstance(hours, tuple) else float(hours)
        prec = precision
        if fp32r_frac < 1.0:
            prec = "fp32r" if rng.uniform() < fp32r_frac else "fp64"
        if rate > 0.0:
            t += float(rng.exponential(1.0 / rate))
        out.append(RunRequest(i, n, nz, vmax, rmax, b, lat, h, prec, t, cfl=cfl,
                              physics=physics))
    return out


# max|u| in m/s above which a run counts as blown up (measure_lh82_phase3.py:
# 129-130 tests the same after each step); non-finite values always do
BLOWUP_U_MAX = 400.0


def build_run(req: RunRequest, device_dtype=None, blowup_u_max: float = BLOWUP_U_MAX):
    """Integrator and device initial state of a request: WS5 advection,
    beta-plane Coriolis (periodic taper), buoyancy and the anelastic
    projection, or with ``physics="production"`` the reference's production
    configuration (build_production_config, no steering wind); Holland vortex
    at the domain centre with the 12-km linear wind decay.  The plan raises
    its blow-up flag on non-finite values or max|u| > ``blowup_u_max``."""
    from .grid import LorenzStaggering
    from .production_config import BaseState, build_production_config
    from .solver import (AdvectionComponent, AnelasticProjection, BuoyancyComponent,
                         CoriolisComponent, LH82AnelasticEquationSet, OperatorConfig,
                         RK3Integrator)
    from .vortex_init import HollandVortexInit
    n, nz = req.n, req.nz
    L = n * req.dx
    base = BaseState(nz, req.lz)
    if req.physics == "production":
        cfg = build_production_config(n, n, nz, L, L, req.lz, req.f0, 0.0, 0.0)
    elif req.physics == "lh82":
        cfg = OperatorConfig(
            equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
            buoyancy=BuoyancyComponent(), projection=AnelasticProjection(n, n, nz, L, L, req.lz),
            advection=AdvectionComponent(n, n, nz, L, L, req.lz, scheme="upwind5h"),
            coriolis=CoriolisComponent(f=req.f0, mode="beta_plane", beta=req.beta, Ly=L, ny=n,
                                       periodic_taper=True))
    else:
        raise ValueError(f"physics must be 'lh82' or 'production', not {req.physics!r}")
    integ = RK3Integrator(cfg, base, precision=req.precision, blowup_u_max=blowup_u_max)
    if req.resume is not None:
        from .snapshot import state_from_snapshot
        state = state_from_snapshot(req.resume, dtype=integ.dtype)
        if tuple(state.u.shape) != (n, n, nz):
            raise ValueError(f"resume snapshot has shape {tuple(state.u.shape)}, the "
                             f"request {(n, n, nz)}")
    else:
        state = HollandVortexInit(req.vmax, req.rmax, req.b, f=req.f0, wind_decay_top=12e3
                                  ).build_state(n, n, nz, L, L, base, dtype=integ.dtype)
    return integ, state, base


def footprint_bytes(req: RunRequest) -> int:
    """HBM a resident run holds: 5 state fields and the plan's scratch (3
    half-spectrum buffers, 5 anchor and 4 stage fields, 2 temporaries and the
    half-level buoyancy; plus two FP64 spectra for the FP32-refined
    correction; the production physics adds the damper's two tendency fields
    and the biharmonic's two inner Laplacians; single-precision 1024 x 1024
    runs with fast stages add the three spectra of the shared stage
    transforms), in the state dtype."""
    S = 8 if req.precision == "fp64" else 4
    n = req.cells
    ns = (req.n // 2 + 1) * req.n * req.nz
    b = S * (5 * n + 12 * n) + 3 * ns * 2 * S
    if req.physics == "production":  # damper tendencies and the inner Laplacians
        b += 4 * n * S
    if req.precision != "fp64":
        b += 2 * ns * 16
        if req.n == 1024 and req.physics == "lh82":  # buoyancy: the fast stages
            b += 3 * ns * 2 * S
    return int(b * 1.05) + (8 << 20)


@dataclass
class RunRecord:
    rid: int
    n: int
    nz: int
    precision: str
    steps: int
    cells: int
    arrival_s: float
    admit_s: float = math.nan
    done_s: float = math.nan
    final: Optional[dict] = None
    # set when the run's final diagnostics show a blow-up (non-finite state or
    # max|u| above the limit): the run is retired and its slot backfilled
    error: Optional[str] = None

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s

    @property
    def queue_s(self) -> float:
        return self.admit_s - self.arrival_s


@dataclass
class _Active:
    req: RunRequest
    rec: RunRecord
    integ: object
    state: object
    stream: torch.cuda.Stream
    graphs: dict
    left: int
    events: list = field(default_factory=list)
    bytes: int = 0
    t: float = 0.0           # model time after the launched steps
    snaps: list = field(default_factory=list)  # snapshot copies in flight
    flag: Optional[torch.Tensor] = None  # pinned copy of the diagnostics block
    blown: bool = False      # the blow-up flag was seen: no further chunks
    launched: int = 0        # steps launched


class ServingEngine:
    """Continuous-batching loop over a request stream on the current GPU.

    hbm_budget: bytes of resident runs admitted at once.  chunk: steps per
    graph launch.  depth: graph launches kept in flight per run.  realtime:
    honour the arrival times (else every request is available at once).
    keep_final: copy each run's final state to the host when it retires.
    prepare_ahead: admitted runs being set up at once on the preparation
    thread.  inflight_cells: cells of the runs allowed work on the device at
    once; runs are fed shortest remaining work first.
    snapshot_every / snapshot_sink: every ``snapshot_every`` steps (at the
    first graph boundary at or past each multiple) the run's state is copied
    to pinned host memory on the run's own stream, and ``snapshot_sink(rid,
    snapshot)`` receives it once the copy has landed (on the serving thread;
    ``oraclev8_b200.snapshot.save_snapshot`` persists one).  A request whose
    ``resume`` holds such a snapshot continues from it."""

    def __init__(self, hbm_budget: float = 150e9, chunk: int = 16, depth: int = 2,
                 realtime: bool = True, keep_final: bool = False, max_active: int = 256,
                 prepare_ahead: int = 32, inflight_cells: float = 64e6,
                 snapshot_every: int = 0, snapshot_sink=None):
        self.snapshot_every = int(snapshot_every)
        self.snapshot_sink = snapshot_sink
        if self.snapshot_every < 0 or (self.snapshot_every and snapshot_sink is None):
            raise ValueError("snapshot_every needs a snapshot_sink (and must be >= 0)")
        self.budget = float(hbm_budget)
        self.inflight_cells = float(inflight_cells)
        self.prepare_ahead = int(prepare_ahead)
        self.chunk, self.depth = int(chunk), int(depth)
        self.realtime, self.keep_final = bool(realtime), bool(keep_final)
        self.max_active = int(max_active)

    @staticmethod
    def prepare_kernels(requests: "list[RunRequest]") -> int:
        """Create (and drop) one plan per distinct grid and precision of
        ``requests``, so that the kernel-form tuning of each grid (cached per
        process) happens here and not while runs are being served.  Returns
        the number of distinct grids."""
        seen = set()
        for r in requests:
            key = (r.n, r.nz, r.precision)
            if key in seen:
                continue
            seen.add(key)
            integ, _, _ = build_run(r)
            integ.plan.release()
            del integ
        torch.cuda.synchronize()
        return len(seen)

    # -- run lifecycle ---------------------------------------------------------
    def _prepare(self, req: RunRequest) -> _Active:
        """Set a run up (plan, device initial state, step graphs): host work,
        done on the preparation thread while the main loop feeds the GPU."""
        stream = torch.cuda.Stream()
        left = req.nsteps - req.start_step
        if left < 1:
            raise ValueError(f"request {req.rid}: nothing left to run after step "
                             f"{req.start_step} of {req.nsteps}")
        with torch.cuda.stream(stream):
            integ, state, _ = build_run(req)
            graphs = {}
            full = min(self.chunk, left)
            graphs[full] = integ.capture(state, req.dt, full)
            tail = left % full
            if tail:
                graphs[tail] = integ.capture(state, req.dt, tail)
        rec = RunRecord(req.rid, req.n, req.nz, req.precision, req.nsteps, req.cells,
                        req.arrival_s)
        from . import _lib as L
        flag = torch.zeros(L.DIAG_COUNT, dtype=torch.float64, pin_memory=True)
        return _Active(req, rec, integ, state, stream, graphs, left,
                       bytes=footprint_bytes(req), t=float(state.t), flag=flag)

    def _launch(self, a: _Active) -> None:
        k = min(self.chunk, a.left)
        before = a.req.nsteps - a.left
        a.graphs[k].launch(a.stream)
        if a.integ._fast:  # t advances once per step, as the step loop adds it
            for _ in range(k):
                a.t = a.t + a.req.dt
        # the graph's last step updated the plan's blow-up flag: copy the
        # diagnostics block to the run's pinned buffer behind it
        with torch.cuda.stream(a.stream):
            a.integ.plan.read_diag_async(a.flag)
        ev = torch.cuda.Event()
        ev.record(a.stream)
        a.events.append(ev)
        a.left -= k
        a.launched += k
        n = self.snapshot_every
        if n and (a.req.nsteps - a.left) // n > before // n:
            with torch.cuda.stream(a.stream):
                a.snaps.append(SnapshotCopy(a.state, t=a.t, step=a.req.nsteps - a.left,
                                            stream=a.stream))

    def _drain_snapshots(self, a: _Active, wait: bool = False) -> None:
        while a.snaps and (wait or a.snaps[0].ready()):
            self.snapshot_sink(a.req.rid, a.snaps.pop(0).result())

    def _retire(self, a: _Active, now: float) -> RunRecord:
        a.rec.done_s = now
        a.rec.steps = a.launched  # steps this engine ran (fewer for a blown-up run)
        self._drain_snapshots(a, wait=True)
        # the last step of every step graph runs the diagnostics reductions,
        # which keep the plan's sticky blow-up flag (the run's work is done,
        # so this read does not wait on the GPU)
        with torch.cuda.stream(a.stream):
            flag = a.integ.plan.blown_up()
        if flag:
            a.rec.error = ("non-finite state" if flag == 1 else
                           f"max|u| above {a.integ.spec.blowup_u_max:g} m/s")
        if self.keep_final:
            with torch.cuda.stream(a.stream):
                s = a.state
                a.rec.final = {f: getattr(s, f).detach().cpu().numpy() for f in
                               ("u", "v", "w", "theta_prime", "projection_potential")}
        # the run's work is complete: hand its plan memory back to the pool
        # without a device-wide synchronisation
        a.graphs.clear()
        a.integ.plan.release(a.stream)
        a.integ = a.state = None
        return a.rec

    # -- main loop -------------------------------------------------------------
    def run(self, requests: "list[RunRequest]") -> "list[RunRecord]":
        """Serve ``requests`` to completion; returns one record per run.

        The main thread admits requests against the HBM budget (FIFO with
        backfill: a request that fits may pass one that does not) and keeps
        every active run's stream fed with graph launches; a preparation
        thread sets admitted runs up, so host set-up overlaps device work."""
        pending = sorted(requests, key=lambda r: (r.arrival_s, r.rid))
        queue: "list[RunRequest]" = []
        active: "list[_Active]" = []
        done: "list[RunRecord]" = []
        used = 0      # bytes of admitted runs (the admission budget)
        todo: "_queue.Queue" = _queue.Queue()
        ready: "_queue.Queue" = _queue.Queue()
        device = torch.cuda.current_device()

        def worker():
            torch.cuda.set_device(device)
            while True:
                item = todo.get()
                if item is None:
                    return
                req, t_admit = item
                try:
                    a = self._prepare(req)
                    a.rec.admit_s = t_admit
                    ready.put(a)
                except BaseException as e:  # surfaced on the main thread
                    ready.put(e)

        th = threading.Thread(target=worker, daemon=True)
        th.start()
        preparing = 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        try:
            while pending or queue or active or preparing:
                now = time.perf_counter() - t0
                while pending and (not self.realtime or pending[0].arrival_s <= now):
                    queue.append(pending.pop(0))
                admitted, used = admit_from_queue(queue, used, self.budget, len(active),
                                                  preparing, self.max_active,
                                                  self.prepare_ahead)
                for req in admitted:
                    todo.put((req, time.perf_counter() - t0))
                    preparing += 1
                progressed = False
                while True:
                    try:
                        a = ready.get_nowait()
                    except _queue.Empty:
                        break
                    preparing -= 1
                    if isinstance(a, BaseException):
                        raise a
                    active.append(a)
                    progressed = True
                # feed the runs with the least remaining work first (shortest
                # remaining processing time), while the cells of runs with
                # work in flight stay under `inflight_cells`: enough
                # concurrent runs to fill the GPU, without slowing every
                # resident run down by sharing the GPU among all of them
                for a in active:
                    if a.events:
                        a.events = [e for e in a.events if not e.query()]
                    if a.snaps:
                        self._drain_snapshots(a)
                    # a blown-up run gets no further chunks: it retires once
                    # the chunks already queued are done, and its slot is
                    # backfilled (the flag of a completed chunk's copy)
                    if not a.blown and a.left > 0 and float(a.flag[14]) > 0.0:
                        a.blown = True
                        a.left = 0
                for a in runs_to_feed(active, self.inflight_cells):
                    while a.left > 0 and len(a.events) < self.depth:
                        self._launch(a)
                        progressed = True
                for a in list(active):
                    if a.left == 0 and not a.events:
                        done.append(self._retire(a, time.perf_counter() - t0))
                        active.remove(a)
                        used -= a.bytes
                        progressed = True
                # Yield the interpreter: the preparation thread needs it, and
                # a busy polling loop would starve the set-up of queued runs.
                # Every fed run has `depth` graph launches queued, so a poll
                # every millisecond leaves the GPU no gap.
                if not progressed:
                    time.sleep(1e-3)
                elif preparing:
                    time.sleep(100e-6)
        finally:
            todo.put(None)
            th.join()
            torch.cuda.synchronize()
        return done


def admit_from_queue(queue: list, used: int, budget: float, n_active: int, preparing: int,
                     max_active: int, prepare_ahead: int, size=footprint_bytes):
    """Admission of queued requests (FIFO with backfill): in queue order, each
    request that fits the HBM budget beside the admitted runs is taken; one
    that does not fit is skipped, so a later, smaller one can take the room.
    A request larger than the whole budget is admitted alone, when nothing
    else is resident or being set up.  At most `max_active` runs resident or
    in set-up, at most `prepare_ahead` in set-up.  Removes the admitted
    requests from `queue`; returns them in admission order and the new
    number of bytes in use."""
    admitted = []
    i = 0
    while i < len(queue) and n_active + preparing < max_active and preparing < prepare_ahead:
        fb = size(queue[i])
        if used + fb <= budget or not (n_active or preparing):
            admitted.append(queue.pop(i))
            used += fb
            preparing += 1
        else:
            i += 1
    return admitted, used


def runs_to_feed(active: list, inflight_cells: float) -> list:
    """The resident runs that get work this pass: the least remaining work
    (steps left x cells) first, ties by request id.  A run with work in flight
    keeps being fed; an idle one starts only while the cells of the runs with
    work in flight stay under `inflight_cells` (enough concurrent runs to fill
    the GPU without sharing it among every resident run).  Finished runs get
    nothing."""
    busy = sum(a.req.cells for a in active if a.events)
    out = []
    for a in sorted(active, key=lambda x: (x.left * x.req.cells, x.req.rid)):
        if a.left > 0 and (a.events or busy < inflight_cells):
            if not a.events:
                busy += a.req.cells
            out.append(a)
    return out


def shard_requests(requests: "list[RunRequest]", rank: int, world: int
                   ) -> "list[RunRequest]":
    """This rank's share of a request stream served by `world` GPUs: whole runs
    are dealt out (runs never exchange data), largest cell-update count first
    to the least-loaded rank (deterministic on every rank)."""
    if world <= 1:
        return list(requests)
    load = [0] * world
    mine = []
    for r in sorted(requests, key=lambda q: (-q.cell_updates, q.rid)):
        g = min(range(world), key=lambda i: (load[i], i))
        load[g] += r.cell_updates
        if g == rank:
            mine.append(r)
    return sorted(mine, key=lambda q: (q.arrival_s, q.rid))


def gather_records(records: "list[RunRecord]"):
    """All ranks' records on rank 0 (None elsewhere); the records themselves
    without a process group.  Final states are not sent."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return records
    slim = [RunRecord(**{**r.__dict__, "final": None}) for r in records]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(slim, out, dst=0)
    if dist.get_rank() != 0:
        return None
    return [r for part in out for r in part]


def summarize(records: "list[RunRecord]", makespan_s: Optional[float] = None) -> dict:
    lat = np.array([r.latency_s for r in records])
    q = np.array([r.queue_s for r in records])
    cu = float(sum(r.cells * r.steps for r in records))
    span = makespan_s if makespan_s is not None else float(max(r.done_s for r in records))
    pct = lambda a, p: float(np.percentile(a, p))
    return {"runs": len(records), "blown_up": sum(1 for r in records if r.error),
            "cell_updates": cu, "makespan_s": span,
            "cell_updates_per_s": cu / span,
            "latency_s": {"p50": pct(lat, 50), "p95": pct(lat, 95), "p99": pct(lat, 99),
                          "max": float(lat.max())},
            "queue_s": {"p50": pct(q, 50), "p95": pct(q, 95), "p99": pct(q, 99)}}


def serve_serial_plain(requests: "list[RunRequest]", realtime: bool = True
                       ) -> "list[RunRecord]":
    """The comparison the serving loop is measured against: the same stream
    served one run at a time, each in plain FP64 through the public
    ``RK3Integrator.step`` (a new State per step), in arrival order."""
    recs = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for req in sorted(requests, key=lambda r: (r.arrival_s, r.rid)):
        if realtime:
            while time.perf_counter() - t0 < req.arrival_s:
                time.sleep(1e-3)
        r64 = RunRequest(**{**req.__dict__, "precision": "fp64"})
        admit = time.perf_counter() - t0
        integ, state, _ = build_run(r64)
        done, flag = 0, 0
        for n in range(r64.nsteps):
            state, dg = integ.step(state, r64.dt, n)
            done += 1
            # the reference's harnesses stop a run here (measure_lh82_phase3.py:
            # 129-130): max|u| above the limit or not finite
            if dg.blowup:
                flag = dg.blowup
                break
        torch.cuda.synchronize()
        rec = RunRecord(req.rid, req.n, req.nz, "fp64", done, r64.cells,
                        req.arrival_s, admit_s=admit, done_s=time.perf_counter() - t0)
        if flag:
            rec.error = "non-finite state" if flag == 1 else "max|u| above the limit"
        recs.append(rec)
        del integ, state
    return recs
