"""LH82 solver on the B200 backend (import surface of oracle_v8/solver/__init__.py)."""
from .equation_set import (ConstraintResidual, EquationSet, LH82AnelasticEquationSet,
                           PseudoIncompressibleEquationSet)
from .tendency import (AdvectionComponent, AnelasticProjection, BuoyancyComponent,
                       CoriolisComponent, DiabaticHeatingComponent, DiagnosticComponent,
                       HelmholtzDivergenceDampingComponent, HorizontalDiffusionComponent,
                       HyperDiffusionComponent, IntensityCapComponent,
                       NewtonianCoolingComponent, PressureGradientComponent,
                       ProjectionComponent, SpongeDampingComponent, State, StateVar,
                       StepComponent, StepStage, SurfaceDragComponent, Tendency,
                       TendencyComponent, anelastic_divergence)
from .operator_config import OperatorConfig
from .poisson import VariableCoefficientPoissonSolver
from .integrator import RK3Integrator, StepDiagnostics

__all__ = [n for n in dir() if not n.startswith("_")]
