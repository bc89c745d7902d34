"""The benchmark workloads (seeded synthetic inputs with the shapes and physics of
the reference drivers), as (metrics, bcs, models, numerics, state, dt, steps).

  cavity_disk          lid-driven cavity with one ACDI disk, FP64, N=64, 200 steps
                       (run_sugiyama_lid_driven_cavity.jl:309-448)
  filament_kolmogorov  wall-supported filament under Kolmogorov forcing, UWCDI,
                       periodic x, N=256, 1000 steps
                       (run_wall_supported_filament_kolmogorov_flow.jl:371-557)
  cavity_disks20       cavity physics with 20 seeded disks of radius 0.05, N=1024
  channel_growth       open channel [0,2]x[0,1], 1024x512, growth and resource
  cavity_disk_sensitivity  cavity_disk at N=256 to T=2 with (G, lid speed, disk centre)
                       as parameters, for the finite-difference sensitivities
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .boundary import AdvectiveOutflow, BoundaryConditionSetup, Dirichlet, Neumann, Periodic
from .imex import FSIBoundaryConditions, FSIModels, FSIState
from .init import initialize_circle, initialize_circles, seeded_disk_centers, sharp_wall_rectangle
from .mesh import build_mesh_metrics, generate_grid
from .models import (ConstantDiffusivity, ConstantViscosity, GeometricStructureExtension,
                     IMEXNumerics, IsotropicGrowthTensor, JainACDIPhaseField, KolmogorovBodyForce,
                     LinearInternalTensorStress, LinearSolverOptions, NoCapillarity, NoRelaxation,
                     PirozzoliUWCDIPhaseField, SaturatingResourceConsumption,
                     SaturatingResourceGrowth)

DISKS20_SEED = 20240611


@dataclass
class Workload:
    name: str
    grid: object
    metrics: object
    bcs: FSIBoundaryConditions
    models: FSIModels
    numerics: IMEXNumerics
    state: FSIState
    dt: float
    steps: int
    needs_compatible_start: bool = False

    @property
    def cells(self) -> int:
        return self.metrics.Nx * self.metrics.Ny


def _numerics(projection_reltol, velocity_reltol, precision, extension=True):
    ls = LinearSolverOptions(velocity_method="gmres", reltol=velocity_reltol, maxiter=800,
                             restart=100, direct_fallback=True, fallback_reltol=1e-6)
    ext = GeometricStructureExtension(20.0, 4.0, safety_cutoff=1e-6)
    kw = {"structure_extension": ext} if extension else {}
    return IMEXNumerics(linear_solvers=ls, projection_reltol=projection_reltol,
                        projection_maxiter=3000, projection_restart=50, precision=precision, **kw)


def _cavity_bcs(lid_speed=1.0):
    wall, lid = Dirichlet(0.0), Dirichlet(float(lid_speed))
    noflux = BoundaryConditionSetup(Neumann(0.0), Neumann(0.0), Neumann(0.0), Neumann(0.0))
    return FSIBoundaryConditions(
        BoundaryConditionSetup(wall, wall, wall, lid), BoundaryConditionSetup(wall, wall, wall, wall),
        noflux, noflux, {"xx": noflux, "yy": noflux, "xy": noflux})


def _cavity_models(h, modulus=0.1):
    return FSIModels(viscosity=ConstantViscosity(0.01), tensor_relaxation=NoRelaxation(),
                     elastic_stress=LinearInternalTensorStress(modulus), capillarity=NoCapillarity(),
                     phase_field_method=JainACDIPhaseField(1.0, 0.51 * h, delta_normal=1e-14,
                                                           dynamic_gamma=False))


def _rest_state(Nx, Ny, phi, resource=None):
    return FSIState(np.zeros((Nx + 1, Ny), order="F"), np.zeros((Nx, Ny + 1), order="F"), phi,
                    np.zeros((Nx, Ny), order="F") if resource is None else resource,
                    np.ones((Nx, Ny), order="F"), np.ones((Nx, Ny), order="F"),
                    np.zeros((Nx, Ny), order="F"))


def cavity_disk(N=64, steps=200, projection_reltol=1e-10, velocity_reltol=1e-8, precision="fp64"):
    grid = generate_grid(1.0, 1.0, N, N)
    metrics = build_mesh_metrics(grid)
    h = 1.0 / N
    phi = initialize_circle(grid, (0.6, 0.5), 0.2, 1.5 * h)
    modulus = 0.1
    dt = 0.2 * h / max(1.0, math.sqrt(modulus / 1.0))
    return Workload("cavity_disk", grid, metrics, _cavity_bcs(), _cavity_models(h, modulus),
                    _numerics(projection_reltol, velocity_reltol, precision), _rest_state(N, N, phi),
                    dt, steps)


def cavity_disk_sensitivity(N=256, params=(0.1, 1.0, 0.6, 0.5), T=2.0, projection_reltol=1e-10,
                            velocity_reltol=1e-8, precision="fp64"):
    """The differentiation configuration: the cavity_disk physics with its shear
    modulus G, lid speed and initial disk centre (x, y) taken from `params`, run to
    time T at the fixed step dt = 0.2/N, so that perturbing G leaves dt alone."""
    G, lid, cx, cy = (float(v) for v in params)
    grid = generate_grid(1.0, 1.0, N, N)
    metrics = build_mesh_metrics(grid)
    h = 1.0 / N
    phi = initialize_circle(grid, (cx, cy), 0.2, 1.5 * h)
    dt = 0.2 * h
    steps = int(round(T / dt))
    return Workload("cavity_disk_sensitivity", grid, metrics, _cavity_bcs(lid), _cavity_models(h, G),
                    _numerics(projection_reltol, velocity_reltol, precision), _rest_state(N, N, phi),
                    dt, steps)


def cavity_disks20(N=1024, steps=500, projection_reltol=1e-10, velocity_reltol=1e-8, precision="fp64",
                   seed=DISKS20_SEED):
    grid = generate_grid(1.0, 1.0, N, N)
    metrics = build_mesh_metrics(grid)
    h = 1.0 / N
    centers = seeded_disk_centers(20, 0.05, h, seed)
    phi = initialize_circles(grid, centers, 0.05, 1.5 * h)
    modulus = 0.1
    dt = 0.2 * h / max(1.0, math.sqrt(modulus))
    return Workload("cavity_disks20", grid, metrics, _cavity_bcs(), _cavity_models(h, modulus),
                    _numerics(projection_reltol, velocity_reltol, precision), _rest_state(N, N, phi),
                    dt, steps)


def filament_kolmogorov(N=256, steps=1000, projection_reltol=1e-10, velocity_reltol=1e-8,
                        precision="fp64"):
    grid = generate_grid(1.0, 1.0, N, N)
    metrics = build_mesh_metrics(grid, periodic_x=True)
    h = 1.0 / N
    px, wall = Periodic(), Dirichlet(0.0)
    bc_phi = BoundaryConditionSetup(px, px, Dirichlet(1.0), Dirichlet(0.0))
    bc_u = BoundaryConditionSetup(px, px, wall, wall)
    bc_q = BoundaryConditionSetup(px, px, Neumann(0.0), Neumann(0.0))
    bc_s1 = BoundaryConditionSetup(px, px, Dirichlet(1.0), Dirichlet(1.0))
    bc_s0 = BoundaryConditionSetup(px, px, Dirichlet(0.0), Dirichlet(0.0))
    bcs = FSIBoundaryConditions(bc_u, bc_u, bc_q, bc_phi, {"xx": bc_s1, "yy": bc_s1, "xy": bc_s0})
    models = FSIModels(viscosity=ConstantViscosity(0.01), tensor_relaxation=NoRelaxation(),
                       elastic_stress=LinearInternalTensorStress(1.0), capillarity=NoCapillarity(),
                       phase_field_method=PirozzoliUWCDIPhaseField(1.0, delta_normal=1e-14),
                       body_force=KolmogorovBodyForce(0.1, 4.0 * math.pi))
    phi = sharp_wall_rectangle(grid, 0.5, 0.04, 0.4)
    dt = 0.2 * h / max(1.0, math.sqrt(1.0))
    return Workload("filament_kolmogorov", grid, metrics, bcs, models,
                    _numerics(projection_reltol, velocity_reltol, precision), _rest_state(N, N, phi),
                    dt, steps)


def channel_growth(N=512, steps=300, projection_reltol=1e-10, velocity_reltol=1e-8, precision="fp64"):
    Nx, Ny = 2 * N, N
    grid = generate_grid(2.0, 1.0, Nx, Ny)
    metrics = build_mesh_metrics(grid)
    h = 1.0 / N
    y = np.asarray(grid.y_p)
    inflow = 4.0 * y * (1.0 - y)
    wall = Dirichlet(0.0)
    bc_u = BoundaryConditionSetup(Dirichlet(inflow), Dirichlet(inflow), wall, wall)
    bc_v = BoundaryConditionSetup(wall, wall, wall, wall)
    bc_q = BoundaryConditionSetup(Neumann(0.0), Dirichlet(0.0), Neumann(0.0), Neumann(0.0))
    bc_phi = BoundaryConditionSetup(Neumann(0.0), Neumann(0.0), Neumann(0.0), Neumann(0.0))
    bc_c = BoundaryConditionSetup(Dirichlet(1.0), AdvectiveOutflow(1.0), Neumann(0.0), Neumann(0.0))
    s1 = BoundaryConditionSetup(Dirichlet(1.0), Dirichlet(1.0), Dirichlet(1.0), Dirichlet(1.0))
    s0 = BoundaryConditionSetup(Dirichlet(0.0), Dirichlet(0.0), Dirichlet(0.0), Dirichlet(0.0))
    bcs = FSIBoundaryConditions(bc_u, bc_v, bc_q, bc_phi, bc_c, {"xx": s1, "yy": s1, "xy": s0})
    models = FSIModels(growth_source=SaturatingResourceGrowth(0.1, 0.5),
                       growth_tensor=IsotropicGrowthTensor(), viscosity=ConstantViscosity(0.01),
                       diffusivity=ConstantDiffusivity(0.01),
                       resource_consumption=SaturatingResourceConsumption(0.05, 0.5),
                       elastic_stress=LinearInternalTensorStress(0.5),
                       phase_field_method=JainACDIPhaseField(1.0, 0.51 * h, delta_normal=1e-14,
                                                             dynamic_gamma=False))
    phi = initialize_circle(grid, (0.5, 0.5), 0.15, 1.5 * h)
    state = _rest_state(Nx, Ny, phi, np.ones((Nx, Ny), order="F"))
    state.U[...] = inflow[None, :]
    dt = 0.2 * h / max(1.0, math.sqrt(0.5))
    return Workload("channel_growth", grid, metrics, bcs, models,
                    _numerics(projection_reltol, velocity_reltol, precision), state, dt, steps,
                    needs_compatible_start=True)


WORKLOADS = {"cavity_disk": cavity_disk, "filament_kolmogorov": filament_kolmogorov,
             "cavity_disks20": cavity_disks20, "channel_growth": channel_growth}
