"""Lorenz vertical staggering (oracle_v8/grid/staggering.py:150-244).

The step kernels apply the Lorenz full-to-half average inline (buoyancy,
advection's u_h/v_h); this class keeps the reference's interface for callers
that use it directly.
"""
from __future__ import annotations

import abc
from enum import Enum

import torch


class LevelType(Enum):
    FULL = "full"
    HALF = "half"


class GridStaggering(abc.ABC):
    name = "abstract"

    @abc.abstractmethod
    def level_type(self, variable: str) -> LevelType: ...

    @abc.abstractmethod
    def interpolate_full_to_half(self, field_on_full): ...

    def __repr__(self) -> str:
        return f"<GridStaggering: {self.name}>"


class LorenzStaggering(GridStaggering):
    """u, v, theta', phi on full levels; w on half levels incl. surface and lid."""
    name = "lorenz"

    def level_type(self, variable: str) -> LevelType:
        return LevelType.HALF if variable == "w" else LevelType.FULL

    def interpolate_full_to_half(self, field_on_full):
        """out[..., k] = 0.5 (f[..., k-1] + f[..., k]) for 1 <= k <= nz-1, zero
        at the surface and lid (staggering.py:172-208)."""
        f = field_on_full
        if not isinstance(f, torch.Tensor):
            raise TypeError("LorenzStaggering on the B200 backend expects a device tensor")
        out = torch.zeros(f.shape[:-1] + (f.shape[-1] + 1,), dtype=f.dtype, device=f.device)
        out[..., 1:-1] = 0.5 * (f[..., :-1] + f[..., 1:])
        return out


class CharneyPhillipsStaggering(GridStaggering):
    """Placeholder, as in the reference (staggering.py:211-244)."""
    name = "charney_phillips"

    def level_type(self, variable: str) -> LevelType:
        return LevelType.HALF if variable in ("w", "theta", "theta_prime") else LevelType.FULL

    def interpolate_full_to_half(self, field_on_full):
        raise NotImplementedError("CharneyPhillipsStaggering is a V8.x placeholder.")
