"""OperatorConfig (oracle_v8/solver/operator_config.py:67-230), unchanged
call signature: the slots and their order, the PGC + projection guard and the
stage filters."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class OperatorConfig:
    equation_set: object
    staggering: object
    buoyancy: object = None
    pressure_gradient: object = None
    projection: object = None
    advection: object = None
    coriolis: object = None
    surface_drag: object = None
    sponge_damping: object = None
    horiz_diffusion: object = None
    newtonian_cooling: object = None
    divergence_damping: object = None
    diabatic_heating: object = None
    _unsafe_pgc_override: bool = False

    def __post_init__(self) -> None:
        if (self.pressure_gradient is not None and self.projection is not None
                and not self._unsafe_pgc_override):
            raise ValueError(
                "Invalid V8 configuration: PressureGradientComponent and "
                "AnelasticProjection cannot both be active.  The projection solves for phi "
                "and corrects u_final = u* - grad(phi), which IS the pressure gradient force.")

    def active_components(self) -> list:
        slots = [self.buoyancy, self.pressure_gradient, self.projection, self.advection,
                 self.coriolis, self.surface_drag, self.sponge_damping, self.horiz_diffusion,
                 self.newtonian_cooling, self.divergence_damping, self.diabatic_heating]
        return [c for c in slots if c is not None]

    def fast_components(self) -> list:
        from .tendency import StepStage
        return [c for c in self.active_components() if c.stage == StepStage.PRE_PROJECTION]

    def slow_components(self) -> list:
        from .tendency import StepStage
        return [c for c in self.active_components() if c.stage == StepStage.SLOW]

    def projection_components(self) -> list:
        from .tendency import StepStage
        return [c for c in self.active_components() if c.stage == StepStage.PROJECTION]

    def to_log_dict(self) -> dict:
        return {
            "equation_set": {"name": self.equation_set.name,
                             "class": type(self.equation_set).__name__},
            "staggering": {"name": self.staggering.name,
                           "class": type(self.staggering).__name__},
            "active_components": [c.to_log_dict() for c in self.active_components()],
            "n_pre_projection": len(self.fast_components()),
            "n_projection": len(self.projection_components()),
            "n_slow": len(self.slow_components()),
        }

    def writes_conflicts(self) -> dict:
        writers: dict = {}
        for c in self.active_components():
            for var in c.writes():
                writers.setdefault(getattr(var, "value", str(var)), []).append(c.name)
        return {k: v for k, v in writers.items() if len(v) > 1}

    def __repr__(self) -> str:
        return (f"<OperatorConfig: {self.equation_set.name} on {self.staggering.name} grid, "
                f"{len(self.active_components())} components>")
