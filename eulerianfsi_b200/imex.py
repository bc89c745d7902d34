"""Host-side mirror of EulerianFSI.jl's TimeIntegrationIMEX API
(TimeIntegrationIMEX.jl:53-65) over the CUDA library's C-ABI.

``integrate_step`` and ``make_velocity_compatible`` mutate the state in place, as
the Julia ``integrate_step!`` / ``make_velocity_compatible!`` do.  Fields are
numpy float64 arrays indexed ``[i, j]`` with i along x, stored column-major
(Fortran order) so their memory layout equals the Julia matrices'.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import _abi
from .boundary import BoundaryConditionSetup, fill_setup, is_periodic_x, is_periodic_y
from .errors import ArgumentError, DimensionMismatch, raise_status
from .mesh import MeshMetrics
from .models import (AbstractPhaseFieldMethod, IMEXNumerics, IsotropicGrowthTensor,
                     LegacySplitPhaseFieldMethod, NoBodyForce, NoCapillarity, NoDiffusion,
                     NoElasticStress, NoGrowth, NoInterfaceFlux, NoRelaxation,
                     NoResourceConsumption, NoViscosity, fill_models, fill_numerics)


def field64(a, shape=None) -> np.ndarray:
    """Column-major float64 view/copy of `a` (no copy when already conforming)."""
    out = np.asfortranarray(a, dtype=np.float64)
    if shape is not None and out.shape != tuple(shape):
        raise DimensionMismatch(f"expected shape {tuple(shape)}; received {out.shape}")
    return out


class FSIState:
    """FSIState(U, V, phi, resource, sigma_xx, sigma_yy, sigma_xy), or the legacy
    six-array form without `resource` (TimeIntegrationIMEX.jl:103-118)."""

    def __init__(self, U, V, phi, *rest):
        if len(rest) == 3:
            resource = np.zeros(np.shape(phi))
            sxx, syy, sxy = rest
        elif len(rest) == 4:
            resource, sxx, syy, sxy = rest
        else:
            raise ArgumentError("FSIState takes 6 or 7 arrays")
        self.U, self.V, self.phi = field64(U), field64(V), field64(phi)
        self.resource = field64(resource)
        self.sigma_xx, self.sigma_yy, self.sigma_xy = field64(sxx), field64(syy), field64(sxy)

    def arrays(self):
        return (self.U, self.V, self.phi, self.resource, self.sigma_xx, self.sigma_yy, self.sigma_xy)

    def copy(self):
        return FSIState(*(a.copy(order="F") for a in self.arrays()))


class FSIBoundaryConditions:
    """FSIBoundaryConditions(U, V, correction, phi, resource, sigma) and the 5-argument
    form reusing the phase-field boundaries for the resource (TimeIntegrationIMEX.jl:127-147).
    `sigma` is a mapping or object with xx, yy and xy entries."""

    def __init__(self, U, V, correction, phi, *rest):
        if len(rest) == 1:
            resource, sigma = phi, rest[0]
        elif len(rest) == 2:
            resource, sigma = rest
        else:
            raise ArgumentError("FSIBoundaryConditions takes 5 or 6 arguments")
        get = (lambda k: sigma[k]) if isinstance(sigma, dict) else (lambda k: getattr(sigma, k))
        for key in ("xx", "yy", "xy"):
            try:
                get(key)
            except (KeyError, AttributeError):
                raise ArgumentError(f"sigma boundary data require an `{key}` entry.") from None
        self.U, self.V, self.correction, self.phi, self.resource = U, V, correction, phi, resource
        self.sigma = {k: get(k) for k in ("xx", "yy", "xy")}


@dataclass
class FSIModels:
    """FSIModels(; kwargs...) (TimeIntegrationIMEX.jl:156-208)."""
    growth_source: Any = field(default_factory=NoGrowth)
    growth_tensor: Any = field(default_factory=IsotropicGrowthTensor)
    viscosity: Any = field(default_factory=NoViscosity)
    diffusivity: Any = field(default_factory=NoDiffusion)
    resource_consumption: Any = field(default_factory=NoResourceConsumption)
    tensor_relaxation: Any = field(default_factory=NoRelaxation)
    elastic_stress: Any = field(default_factory=NoElasticStress)
    capillarity: Any = field(default_factory=NoCapillarity)
    phase_field_method: Any = None
    interface_flux: Any = field(default_factory=NoInterfaceFlux)
    body_force: Any = field(default_factory=NoBodyForce)

    def __post_init__(self):
        if self.phase_field_method is None:
            self.phase_field_method = LegacySplitPhaseFieldMethod(self.interface_flux)
        elif not isinstance(self.interface_flux, NoInterfaceFlux):
            raise ArgumentError("Specify either phase_field_method or the legacy interface_flux keyword, not both.")
        if not isinstance(self.phase_field_method, AbstractPhaseFieldMethod):
            raise ArgumentError("phase_field_method must be an AbstractPhaseFieldMethod.")


@dataclass
class StepReport:
    """StepReport (TimeIntegrationIMEX.jl:318-327)."""
    maximum_projection_constraint_linf: float
    maximum_growth_trace_error: float
    minimum_phi: float
    maximum_phi: float
    minimum_resource: float
    minimum_sigma_eigenvalue: float
    maximum_abs_sigma_determinant_error: float
    non_spd_cells: int

    @classmethod
    def from_c(cls, r: _abi.StepReportC) -> "StepReport":
        return cls(r.maximum_projection_constraint_linf, r.maximum_growth_trace_error, r.minimum_phi,
                   r.maximum_phi, r.minimum_resource, r.minimum_sigma_eigenvalue,
                   r.maximum_abs_sigma_determinant_error, int(r.non_spd_cells))


@dataclass
class ProjectionResult:
    """ProjectionResult (Projection.jl:31-37)."""
    correction: np.ndarray
    linear_relative_residual: float
    constraint_linf: float
    constraint_l2: float
    compatibility_defect: float


@dataclass
class IMEXWorkspace:
    """The part of IMEXWorkspace (TimeIntegrationIMEX.jl:333-441) that is observable
    across calls: the projection warm start.  Every other buffer lives on the device."""
    correction: np.ndarray


def allocate_imex_workspace(metrics: MeshMetrics) -> IMEXWorkspace:
    return IMEXWorkspace(np.zeros((metrics.Nx, metrics.Ny), order="F"))


class ConfigBlock:
    """An `efsi_config` plus the numpy buffers its pointers refer to."""

    def __init__(self, metrics: MeshMetrics, bcs: FSIBoundaryConditions, models: FSIModels,
                 numerics: IMEXNumerics):
        self.keep: list = []
        cfg = _abi.Config()
        cfg.abi_version = _abi.ABI_VERSION
        m = cfg.mesh
        m.Nx, m.Ny, m.Lx, m.Ly = metrics.Nx, metrics.Ny, metrics.Lx, metrics.Ly
        m.periodic_x, m.periodic_y = int(metrics.periodic_x), int(metrics.periodic_y)
        for name, attr in (("dx_f", "dx_f"), ("dx_c", "dx_c"), ("dy_f", "dy_f"), ("dy_c", "dy_c"),
                           ("wL_c2fx", "wL_c2fx"), ("wR_c2fx", "wR_c2fx"), ("wB_c2fy", "wB_c2fy"),
                           ("wT_c2fy", "wT_c2fy"), ("wL_f2cx", "wL_f2cx"), ("wR_f2cx", "wR_f2cx"),
                           ("wB_f2cy", "wB_f2cy"), ("wT_f2cy", "wT_f2cy"),
                           ("dx_west_corner", "dx_west_corner"), ("dx_east_corner", "dx_east_corner"),
                           ("dy_south_corner", "dy_south_corner"), ("dy_north_corner", "dy_north_corner")):
            arr = np.ascontiguousarray(getattr(metrics, attr), dtype=np.float64)
            self.keep.append(arr)
            setattr(m, name, _abi.dptr(arr))
        Nx, Ny = metrics.Nx, metrics.Ny
        fill_setup(cfg.bc_U, bcs.U, Ny, Nx + 1, self.keep)
        fill_setup(cfg.bc_V, bcs.V, Ny + 1, Nx, self.keep)
        fill_setup(cfg.bc_correction, bcs.correction, Ny, Nx, self.keep)
        fill_setup(cfg.bc_phi, bcs.phi, Ny, Nx, self.keep)
        fill_setup(cfg.bc_resource, bcs.resource, Ny, Nx, self.keep)
        fill_setup(cfg.bc_sigma_xx, bcs.sigma["xx"], Ny, Nx, self.keep)
        fill_setup(cfg.bc_sigma_yy, bcs.sigma["yy"], Ny, Nx, self.keep)
        fill_setup(cfg.bc_sigma_xy, bcs.sigma["xy"], Ny, Nx, self.keep)
        fill_models(cfg.models, models)
        fill_numerics(cfg.numerics, numerics)
        self.config = cfg


class Handle:
    """Owns one library context (CUDA library, or any object exposing the same
    prefixed entry points)."""

    def __init__(self, lib, prefix: str, block: ConfigBlock, metrics: MeshMetrics):
        self.lib, self.prefix, self.block, self.metrics = lib, prefix, block, metrics
        h = C.c_void_p()
        st = self._fn("create")(C.byref(block.config), C.byref(h))
        if st != _abi.OK:
            msg = self._fn("last_error")(None)
            raise_status(st, msg.decode() if msg else "")
        self.h = h

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def call(self, name, *args):
        st = self._fn(name)(self.h, *args)
        if st != _abi.OK:
            msg = self._fn("last_error")(self.h)
            raise_status(st, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._fn("destroy")(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state transfer --
    def shapes(self):
        Nx, Ny = self.metrics.Nx, self.metrics.Ny
        return [(Nx + 1, Ny), (Nx, Ny + 1)] + [(Nx, Ny)] * 5

    def upload(self, state: FSIState):
        arrs = [field64(a, s) for a, s in zip(state.arrays(), self.shapes())]
        self.call("upload_state", *[_abi.dptr(a) for a in arrs])

    def download(self, state: FSIState):
        for a, s in zip(state.arrays(), self.shapes()):
            if a.shape != s or not a.flags.f_contiguous or a.dtype != np.float64:
                raise DimensionMismatch("state arrays must be float64, Fortran-ordered, correctly sized")
        self.call("download_state", *[_abi.dptr(a) for a in state.arrays()])

    def set_correction(self, q):
        q = field64(q, (self.metrics.Nx, self.metrics.Ny))
        self.call("set_correction", _abi.dptr(q))

    def get_correction(self):
        q = np.zeros((self.metrics.Nx, self.metrics.Ny), order="F")
        self.call("get_correction", _abi.dptr(q))
        return q

    def stats(self):
        s = _abi.Stats()
        self.call("get_stats", C.byref(s))
        return {"projection_iterations": list(s.projection_iterations),
                "velocity_iterations": list(s.velocity_iterations),
                "resource_iterations": list(s.resource_iterations),
                "kernel_launches": int(s.kernel_launches), "device_ms": float(s.device_ms),
                "site_launches": int(s.site_launches), "site_ms": float(s.site_ms),
                "site_bytes": float(s.site_bytes), "step_bytes": float(s.step_bytes)}


@dataclass
class IMEXContext:
    """IMEXContext (TimeIntegrationIMEX.jl:304-311): the configuration plus the
    device context that holds the preassembled projection hierarchy."""
    metrics: MeshMetrics
    bcs: FSIBoundaryConditions
    models: FSIModels
    numerics: IMEXNumerics
    config: ConfigBlock
    handle: Handle


def _validate_periodicity(metrics: MeshMetrics, bcs: FSIBoundaryConditions):  # :447-466
    for name, bc in (("U", bcs.U), ("V", bcs.V), ("correction", bcs.correction), ("phi", bcs.phi),
                     ("resource", bcs.resource), ("sigma_xx", bcs.sigma["xx"]),
                     ("sigma_yy", bcs.sigma["yy"]), ("sigma_xy", bcs.sigma["xy"])):
        if not isinstance(bc, BoundaryConditionSetup):
            raise ArgumentError(f"{name} boundary conditions must be a BoundaryConditionSetup.")
        if metrics.periodic_x != is_periodic_x(bc):
            raise ArgumentError(f"{name} boundary conditions do not match MeshMetrics periodicity in x.")
        if metrics.periodic_y != is_periodic_y(bc):
            raise ArgumentError(f"{name} boundary conditions do not match MeshMetrics periodicity in y.")


def build_imex_context(metrics: MeshMetrics, bcs: FSIBoundaryConditions, models: FSIModels, *,
                       numerics: IMEXNumerics | None = None, use_projection_amg: bool = True,
                       backend: str = "cuda") -> IMEXContext:
    """build_imex_context (TimeIntegrationIMEX.jl:468-493) with the device backend.
    `use_projection_amg` is accepted for signature compatibility; the device solves the
    projection with its own solvers (`IMEXNumerics.projection_solver`: the direct
    fast-diagonalisation solve where the grid allows it, multigrid-preconditioned CG
    otherwise)."""
    numerics = numerics if numerics is not None else IMEXNumerics()
    if backend != "cuda":
        raise ArgumentError("the only backend of this library is 'cuda'")
    _validate_periodicity(metrics, bcs)
    block = ConfigBlock(metrics, bcs, models, numerics)
    handle = Handle(_abi.load_library(), "efsi_", block, metrics)
    return IMEXContext(metrics, bcs, models, numerics, block, handle)


def _validate_state(state: FSIState, metrics: MeshMetrics):  # :495-523
    Nx, Ny = metrics.Nx, metrics.Ny
    if state.U.shape != (Nx + 1, Ny):
        raise DimensionMismatch(f"state.U must have size {(Nx + 1, Ny)}; received {state.U.shape}.")
    if state.V.shape != (Nx, Ny + 1):
        raise DimensionMismatch(f"state.V must have size {(Nx, Ny + 1)}; received {state.V.shape}.")
    for name in ("phi", "resource", "sigma_xx", "sigma_yy", "sigma_xy"):
        if getattr(state, name).shape != (Nx, Ny):
            raise DimensionMismatch(f"state.{name} must have size {(Nx, Ny)}.")


def make_velocity_compatible(state: FSIState, context: IMEXContext, work: IMEXWorkspace) -> ProjectionResult:
    """make_velocity_compatible! (TimeIntegrationIMEX.jl:1088-1109); U and V of
    `state` are replaced by the projected velocity."""
    _validate_state(state, context.metrics)
    h = context.handle
    h.upload(state)
    h.set_correction(work.correction)
    r = _abi.ProjectionResultC()
    h.call("make_velocity_compatible", C.byref(r))
    h.download(state)
    work.correction[...] = h.get_correction()
    return ProjectionResult(work.correction.copy(order="F"), r.linear_relative_residual,
                            r.constraint_linf, r.constraint_l2, r.compatibility_defect)


def integrate_step(state: FSIState, t: float, dt: float, context: IMEXContext,
                   work: IMEXWorkspace) -> StepReport:
    """integrate_step! (TimeIntegrationIMEX.jl:1152-1256): advances `state` in place
    from t to t+dt on the device and returns the StepReport.  The workspace
    correction (the projection warm start) travels with the state."""
    _validate_state(state, context.metrics)
    h = context.handle
    arrs = [field64(a, s) for a, s in zip(state.arrays(), h.shapes())]
    q = field64(work.correction, (context.metrics.Nx, context.metrics.Ny))
    rep = _abi.StepReportC()
    h.call("integrate_step_host", *[_abi.dptr(a) for a in arrs], _abi.dptr(q), float(t), float(dt),
           C.byref(rep))
    for dst, src in zip(state.arrays(), arrs):
        if dst is not src:
            dst[...] = src
    if q is not work.correction:
        work.correction[...] = q
    return StepReport.from_c(rep)
