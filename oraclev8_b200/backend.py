"""B200 array backend: the drop-in counterpart of oracle_v8/backend.py:39-139.

The reference selects NumPy or CuPy as ``xp``; this backend keeps every
prognostic field as a CUDA ``torch.Tensor`` (z contiguous, C order) and runs
the step through the sm_100a library.  ``ORACLE_B200_PRECISION`` selects the
default device dtype: ``fp64`` (default), ``fp32``, or ``fp32r`` (FP32 state
with one FP64-residual defect correction of the projection per step).
"""
from __future__ import annotations

import os as _os

import numpy as _np
import torch as _torch  # device arrays are torch tensors


class _DeviceArrays:
    """The ``xp`` of this backend: torch, under the NumPy spellings that the
    reference's drivers and harnesses use on device fields (``axis=`` for
    ``roll``, Python scalars as operands of ``maximum``, ``minimum`` and
    ``clip``; run_storm.py:128-137, run_translation_test.py:132-160).  Every
    other name is torch's own."""

    __name__ = "torch"

    def __getattr__(self, name):
        return getattr(_torch, name)

    @staticmethod
    def roll(a, shift, axis=None):
        return _torch.roll(a, shift, dims=axis)

    @staticmethod
    def _pair(a, b):
        if not isinstance(a, _torch.Tensor):
            a = _torch.as_tensor(a, dtype=b.dtype, device=b.device)
        if not isinstance(b, _torch.Tensor):
            b = _torch.as_tensor(b, dtype=a.dtype, device=a.device)
        return a, b

    @classmethod
    def maximum(cls, a, b):
        return _torch.maximum(*cls._pair(a, b))

    @classmethod
    def minimum(cls, a, b):
        return _torch.minimum(*cls._pair(a, b))

    @classmethod
    def clip(cls, a, lo, hi):
        return cls.minimum(cls.maximum(a, lo), hi)


xp = _DeviceArrays()

GPU_AVAILABLE: bool = bool(_torch.cuda.is_available())
PRECISION: str = _os.environ.get("ORACLE_B200_PRECISION", "fp64")
if PRECISION not in ("fp64", "fp32", "fp32r"):
    raise ValueError(f"ORACLE_B200_PRECISION must be fp64, fp32 or fp32r, got {PRECISION!r}")
DTYPE = _torch.float64 if PRECISION == "fp64" else _torch.float32


def _device():
    if not GPU_AVAILABLE:
        raise RuntimeError("the oraclev8_b200 backend needs a CUDA device (no CPU fallback)")
    return _torch.device("cuda", _torch.cuda.current_device())


def to_numpy(arr):
    """Host NumPy copy of a device tensor (backend.py:61-77); other inputs pass through."""
    if isinstance(arr, _torch.Tensor):
        return arr.detach().to("cpu").numpy()
    return arr


def asarray(arr, dtype=None):
    """Move ``arr`` to the CUDA device as a contiguous tensor (backend.py:80-89)."""
    dt = DTYPE if dtype is None else dtype
    if isinstance(dt, _np.dtype) or dt in (float, _np.float64, _np.float32):
        dt = _torch.float64 if _np.dtype(dt) == _np.float64 else _torch.float32
    if isinstance(arr, _torch.Tensor):
        return arr.to(device=_device(), dtype=dt).contiguous()
    return _torch.as_tensor(_np.ascontiguousarray(arr), dtype=dt, device=_device())


def wrap_base(base):
    """Copy of a base-state object (backend.py:92-139).  z, rho0 and theta0
    stay FP64 host arrays: the library uploads its own FP64 copies once per
    plan, so the reference-state profiles are FP64 on the device for both
    precisions."""

    class _DeviceBase:
        pass

    dev = _DeviceBase()
    for attr in ("z", "rho0", "theta0"):
        if hasattr(base, attr):
            setattr(dev, attr, _np.asarray(to_numpy(getattr(base, attr)), dtype=_np.float64))
    for attr in dir(base):
        if attr.startswith("_") or attr in ("z", "rho0", "theta0"):
            continue
        val = getattr(base, attr, None)
        if val is not None:
            setattr(dev, attr, val)
    return dev
