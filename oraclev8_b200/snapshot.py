"""Full-state snapshots and checkpoints of a run on the B200 backend.

The record is the reference's host snapshot (run_translation_test.py:290-296):
a dict with the scalars ``t``, ``cx``, ``cy`` and the host arrays ``u``,
``v``, ``w``, ``theta_prime``, ``projection_potential`` of the state.  On
disk it is an ``.npz`` with those keys, plus ``step`` (steps taken) and
``format``.  A run restored from it continues bit for bit: the state, its time
and the step counter are all that a step reads.

The device-to-host copy goes into pinned host buffers on a copy stream,
ordered after the step that produced the state, so the next steps run while
the snapshot drains (``SnapshotCopy``).  ``take_snapshot`` is the synchronous
form.

``save_gyre_snapshot`` writes the derived record of the reference's beta-gyre
harness (run_translation_test.py:2104-2125): the column-mean wind, its
centred vorticity, the centre and dx.
"""
from __future__ import annotations

import os
from typing import Optional

import numpy as np
import torch

FIELDS = ("u", "v", "w", "theta_prime", "projection_potential")
FORMAT = "oraclev8_b200.snapshot/1"


class SnapshotCopy:
    """An asynchronous device-to-host copy of one state into pinned buffers.

    By default the copy is enqueued on the producing (current) stream: work
    queued there afterwards, an in-place step included, runs after it, and
    the host does not wait.  With ``stream`` set to a side stream, the copy
    waits for the producing stream and then overlaps the work queued after
    it; the caller must then not overwrite the fields before ``ready()``
    (step a second state, or wait).  ``result()`` waits for the copy and
    returns the snapshot dict, whose arrays are views of the pinned buffers:
    a ``pinned`` dict passed again to a later copy overwrites them, so keep
    (or copy) a result before its buffers are reused."""

    def __init__(self, state, t=None, cx=None, cy=None, step: Optional[int] = None,
                 stream: Optional[torch.cuda.Stream] = None, pinned: Optional[dict] = None):
        dev = state.u.device
        if dev.type != "cuda":
            raise TypeError("SnapshotCopy reads device fields (CUDA torch tensors)")
        self.meta = {"t": float(state.t if t is None else t), "cx": cx, "cy": cy,
                     "step": step}
        produced = torch.cuda.Event()
        produced.record(torch.cuda.current_stream(dev))
        self.stream = stream or torch.cuda.current_stream(dev)
        self.host = {}
        with torch.cuda.stream(self.stream):
            self.stream.wait_event(produced)
            for f in FIELDS:
                x = getattr(state, f)
                buf = pinned.get(f) if pinned else None
                if buf is None or buf.shape != x.shape or buf.dtype != x.dtype:
                    buf = torch.empty(tuple(x.shape), dtype=x.dtype, pin_memory=True)
                x.record_stream(self.stream)
                buf.copy_(x, non_blocking=True)
                self.host[f] = buf
        self.done = torch.cuda.Event()
        self.done.record(self.stream)

    def ready(self) -> bool:
        return self.done.query()

    def result(self) -> dict:
        self.done.synchronize()
        snap = {"t": self.meta["t"], "cx": self.meta["cx"], "cy": self.meta["cy"]}
        snap.update({f: self.host[f].numpy() for f in FIELDS})
        if self.meta["step"] is not None:
            snap["step"] = int(self.meta["step"])
        return snap


def take_snapshot(state, t=None, cx=None, cy=None, step: Optional[int] = None) -> dict:
    """The reference's snapshot dict of a device state (waits for the copy)."""
    return SnapshotCopy(state, t, cx, cy, step).result()


def save_snapshot(path, snap: dict) -> str:
    """Write a snapshot dict as ``.npz`` (the dict's keys, ``format``; cx/cy
    stored as NaN when absent).  Returns the path written."""
    path = os.fspath(path)
    out = {f: np.asarray(snap[f]) for f in FIELDS}
    out["t"] = np.float64(snap["t"])
    for k in ("cx", "cy"):
        out[k] = np.float64(np.nan if snap.get(k) is None else snap[k])
    out["step"] = np.int64(snap.get("step", -1))
    out["format"] = np.array(FORMAT)
    np.savez(path, **out)
    return path if path.endswith(".npz") else path + ".npz"


def load_snapshot(path) -> dict:
    """Read a snapshot written by ``save_snapshot`` (or any ``.npz`` with the
    five field keys and ``t``)."""
    with np.load(os.fspath(path)) as d:
        missing = [k for k in FIELDS + ("t",) if k not in d.files]
        if missing:
            raise ValueError(f"not a snapshot: missing {missing}")
        snap = {f: d[f] for f in FIELDS}
        snap["t"] = float(d["t"])
        for k in ("cx", "cy"):
            v = float(d[k]) if k in d.files else float("nan")
            snap[k] = None if np.isnan(v) else v
        if "step" in d.files and int(d["step"]) >= 0:
            snap["step"] = int(d["step"])
    return snap


def state_from_snapshot(snap: dict, dtype=None, device=None):
    """Device State of a snapshot (its own dtype unless ``dtype`` is given)."""
    from .solver import State
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    fields = []
    for f in FIELDS:
        t = torch.from_numpy(np.ascontiguousarray(snap[f]))
        fields.append((t if dtype is None else t.to(dtype)).to(dev))
    return State(*fields, float(snap["t"]))


def save_gyre_snapshot(path, snap: dict, dx: float) -> str:
    """The beta-gyre harness record (run_translation_test.py:2104-2125):
    column-mean u and v, zeta = dv/dx - du/dy by periodic centred differences
    with spacing dx on both axes, the centre and dx."""
    u2 = np.asarray(snap["u"]).mean(axis=2)
    v2 = np.asarray(snap["v"]).mean(axis=2)
    dvdx = (np.roll(v2, -1, 0) - np.roll(v2, 1, 0)) / (2 * dx)
    dudy = (np.roll(u2, -1, 1) - np.roll(u2, 1, 1)) / (2 * dx)
    path = os.fspath(path)
    np.savez(path, zeta=dvdx - dudy, u=u2, v=v2, cx=snap["cx"], cy=snap["cy"], dx=dx)
    return path if path.endswith(".npz") else path + ".npz"
