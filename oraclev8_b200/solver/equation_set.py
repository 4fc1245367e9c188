"""LH82 anelastic equation set (oracle_v8/solver/equation_set.py:176-319)."""
from __future__ import annotations

import abc
from dataclasses import dataclass

import numpy as np

from ..backend import to_numpy


@dataclass
class ConstraintResidual:
    max_abs: float
    rms: float


class EquationSet(abc.ABC):
    name = "abstract"

    @abc.abstractmethod
    def compute_buoyancy_tendency(self, theta_prime, base, staggering): ...

    @abc.abstractmethod
    def base_state_compatibility(self, base) -> tuple: ...

    def __repr__(self) -> str:
        return f"<EquationSet: {self.name}>"


class LH82AnelasticEquationSet(EquationSet):
    """Continuity div(rho0 u) = 0, Poisson coefficient rho0(z),
    buoyancy b = g theta' / theta0(z)."""
    name = "LH82_anelastic"

    def poisson_coefficient(self, base, staggering):
        raise NotImplementedError("placeholder in the reference (equation_set.py:199-207)")

    def compute_constraint_residual(self, *a, **k):
        raise NotImplementedError("placeholder in the reference (equation_set.py:209-220)")

    def compute_buoyancy_tendency(self, theta_prime, base, staggering):
        """b_half on the w levels, zero at surface and lid (equation_set.py:222-265),
        computed by the device kernel."""
        from .tendency import _plan_for
        p = _plan_for(theta_prime, base)
        return p.buoyancy(theta_prime.contiguous())

    def base_state_compatibility(self, base) -> tuple:
        """equation_set.py:267-319."""
        if base is None:
            return (False, "base state is None")
        for f in ("rho0", "theta0", "z", "integration_scheme"):
            if not hasattr(base, f):
                return (False, f"base state is missing required field: {f!r}")
            if getattr(base, f) is None:
                return (False, f"base state field {f!r} is None")
        ready = getattr(base, "is_load_bearing_ready", None)
        if not callable(ready) or not ready():
            return (False, "base state is not load-bearing ready "
                           f"(integration_scheme={base.integration_scheme!r})")
        r = np.asarray(to_numpy(base.rho0))
        t = np.asarray(to_numpy(base.theta0))
        if not np.all(np.isfinite(r)):
            return (False, "non-finite rho0(z) detected")
        if not np.all(np.isfinite(t)):
            return (False, "non-finite theta0(z) detected")
        if np.any(r <= 0):
            return (False, f"non-positive rho0(z); min = {r.min()}")
        if np.any(t <= 0):
            return (False, f"non-positive theta0(z); min = {t.min()}")
        return (True, "compatible")


class PseudoIncompressibleEquationSet(EquationSet):
    """Placeholder, as in the reference (equation_set.py:322-390)."""
    name = "pseudo_incompressible"

    def compute_buoyancy_tendency(self, theta_prime, base, staggering):
        raise NotImplementedError("PseudoIncompressibleEquationSet is a placeholder")

    def base_state_compatibility(self, base) -> tuple:
        return (False, "pseudo-incompressible equation set is not implemented")
