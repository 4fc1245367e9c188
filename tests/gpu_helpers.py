"""Shared helpers of the GPU parity tests."""
import json

import numpy as np
import torch

from oracle import lh82 as O

# FP64 parity bar: max |gpu - ref| <= 1e-12 * max |ref| for every field.
TOL64 = 1e-12


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    a = host(a) if isinstance(a, torch.Tensor) else np.asarray(a)
    b = np.asarray(b)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a.astype(np.float64) - b))) / scale


class Base:
    def __init__(self, nz, Lz):
        self.z, self.rho0, self.theta0 = O.build_base_state(nz, Lz)
        self.integration_scheme = "trapezoid"


def b200_config(c, nx=None):
    """Build an oraclev8_b200 OperatorConfig from a golden case description."""
    from oraclev8_b200.solver import (AdvectionComponent, AnelasticProjection,
                                      BuoyancyComponent, CoriolisComponent,
                                      DiabaticHeatingComponent,
                                      HelmholtzDivergenceDampingComponent,
                                      HorizontalDiffusionComponent, HyperDiffusionComponent,
                                      LH82AnelasticEquationSet, NewtonianCoolingComponent,
                                      OperatorConfig, SpongeDampingComponent,
                                      SurfaceDragComponent)
    from oraclev8_b200.grid import LorenzStaggering
    nx, ny, nz, Lx, Ly, Lz = c["nx"], c["ny"], c["nz"], c["Lx"], c["Ly"], c["Lz"]
    kw = dict(equation_set=LH82AnelasticEquationSet(), staggering=LorenzStaggering(),
              projection=AnelasticProjection(nx, ny, nz, Lx, Ly, Lz))
    if c.get("buoyancy"):
        kw["buoyancy"] = BuoyancyComponent()
    if c.get("advection"):
        kw["advection"] = AdvectionComponent(nx, ny, nz, Lx, Ly, Lz, scheme=c["advection"])
    if c.get("coriolis"):
        ck = dict(c["coriolis"])
        if ck.get("mode") == "beta_plane":
            ck.update(Ly=Ly, ny=ny)
        kw["coriolis"] = CoriolisComponent(**ck)
    if c.get("damping") is not None:
        kw["divergence_damping"] = HelmholtzDivergenceDampingComponent(
            epsilon=c["damping"], Lx=Lx, Ly=Ly, nx=nx, ny=ny)
    if c.get("heating"):
        kw["diabatic_heating"] = DiabaticHeatingComponent(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly,
                                                          Lz=Lz, **c["heating"])
    if c.get("drag"):
        kw["surface_drag"] = SurfaceDragComponent(**c["drag"])
    if c.get("sponge"):
        kw["sponge_damping"] = SpongeDampingComponent(Lz=Lz, **c["sponge"])
    if c.get("laplacian") is not None:
        kw["horiz_diffusion"] = HorizontalDiffusionComponent(c["laplacian"], Lx, Ly, nx, ny)
    if c.get("hyper") is not None:
        kw["horiz_diffusion"] = HyperDiffusionComponent(c["hyper"], Lx, Ly, nx, ny)
    if c.get("cooling") is not None:
        kw["newtonian_cooling"] = NewtonianCoolingComponent(tau=c["cooling"])
    return OperatorConfig(**kw)


def load_case(golden_dir, name):
    g = np.load(golden_dir / f"steps_{name}.npz")
    return g, json.loads(str(g["config_json"]))
