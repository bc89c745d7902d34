"""Constitutive, phase-field, forcing and numerics types mirroring the reference
constructors (names, arguments, defaults and ArgumentError checks)."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from . import _abi
from .errors import ArgumentError


def _finite(x, msg):
    x = float(x)
    if not math.isfinite(x):
        raise ArgumentError(msg)
    return x


# ---- GrowthModels.jl:47-168 ---------------------------------------------------
class AbstractGrowthSource:
    pass


@dataclass(frozen=True)
class NoGrowth(AbstractGrowthSource):
    pass


@dataclass(frozen=True)
class ConstantIntrinsicGrowth(AbstractGrowthSource):
    rate: float

    def __post_init__(self):
        _finite(self.rate, "Intrinsic growth rate must be finite.")


@dataclass(frozen=True)
class SaturatingResourceGrowth(AbstractGrowthSource):
    rate: float
    half_saturation: float

    def __post_init__(self):
        _finite(self.rate, "Resource-limited growth rate must be finite.")
        _finite(self.half_saturation, "Growth half-saturation constant must be finite.")
        if not self.half_saturation > 0:
            raise ArgumentError("Growth half-saturation constant must be strictly positive.")


class AbstractGrowthTensorModel:
    pass


@dataclass(frozen=True)
class IsotropicGrowthTensor(AbstractGrowthTensorModel):
    pass


@dataclass(frozen=True)
class DirectionalGrowthTensor(AbstractGrowthTensorModel):
    direction_x: float
    direction_y: float

    def __post_init__(self):
        tx, ty = float(self.direction_x), float(self.direction_y)
        if not (math.isfinite(tx) and math.isfinite(ty)):
            raise ArgumentError("Directional-growth components must be finite.")
        mag = math.hypot(tx, ty)
        if not mag > 0:
            raise ArgumentError("Directional growth requires a non-zero direction vector.")
        object.__setattr__(self, "direction_x", tx / mag)
        object.__setattr__(self, "direction_y", ty / mag)


# ---- TransportConstitutive.jl:78-397 --------------------------------------------
class AbstractViscosityModel:
    pass


@dataclass(frozen=True)
class NoViscosity(AbstractViscosityModel):
    pass


@dataclass(frozen=True)
class ConstantViscosity(AbstractViscosityModel):
    value: float

    def __post_init__(self):
        _finite(self.value, "Viscosity must be finite.")
        if not self.value > 0:
            raise ArgumentError("Viscosity must be strictly positive.")


@dataclass(frozen=True)
class HarmonicPhaseViscosity(AbstractViscosityModel):
    fluid_value: float
    structure_value: float

    def __post_init__(self):
        _finite(self.fluid_value, "Fluid viscosity must be finite.")
        _finite(self.structure_value, "Structure viscosity must be finite.")
        if not (self.fluid_value > 0 and self.structure_value > 0):
            raise ArgumentError("Viscosities must be strictly positive.")


class AbstractDiffusivityModel:
    pass


@dataclass(frozen=True)
class NoDiffusion(AbstractDiffusivityModel):
    pass


@dataclass(frozen=True)
class ConstantDiffusivity(AbstractDiffusivityModel):
    value: float

    def __post_init__(self):
        _finite(self.value, "Diffusivity must be finite.")
        if not self.value > 0:
            raise ArgumentError("Diffusivity must be strictly positive.")


@dataclass(frozen=True)
class HarmonicPhaseDiffusivity(AbstractDiffusivityModel):
    fluid_value: float
    structure_value: float

    def __post_init__(self):
        _finite(self.fluid_value, "Fluid diffusivity must be finite.")
        _finite(self.structure_value, "Structure diffusivity must be finite.")
        if not (self.fluid_value > 0 and self.structure_value > 0):
            raise ArgumentError("Diffusivities must be strictly positive.")


class AbstractResourceConsumption:
    pass


@dataclass(frozen=True)
class NoResourceConsumption(AbstractResourceConsumption):
    pass


@dataclass(frozen=True)
class SaturatingResourceConsumption(AbstractResourceConsumption):
    rate: float
    half_saturation: float

    def __post_init__(self):
        _finite(self.rate, "Consumption rate must be finite.")
        _finite(self.half_saturation, "Consumption half-saturation constant must be finite.")
        if not self.rate >= 0:
            raise ArgumentError("Consumption rate must be non-negative.")
        if not self.half_saturation > 0:
            raise ArgumentError("Consumption half-saturation constant must be strictly positive.")


class AbstractBodyForce:
    pass


@dataclass(frozen=True)
class NoBodyForce(AbstractBodyForce):
    pass


@dataclass(frozen=True)
class ConstantBodyForce(AbstractBodyForce):
    fx: float
    fy: float

    def __post_init__(self):
        _finite(self.fx, "Body-force x-component must be finite.")
        _finite(self.fy, "Body-force y-component must be finite.")


@dataclass(frozen=True)
class KolmogorovBodyForce(AbstractBodyForce):
    amplitude: float
    wavenumber: float
    phase: float = 0.0

    def __post_init__(self):
        _finite(self.amplitude, "Kolmogorov-force amplitude must be finite.")
        _finite(self.wavenumber, "Kolmogorov-force wavenumber must be finite.")
        if not self.wavenumber > 0:
            raise ArgumentError("Kolmogorov-force wavenumber must be positive.")
        _finite(self.phase, "Kolmogorov-force phase must be finite.")


# ---- StructuralConstitutive.jl:15-48 ------------------------------------------
class AbstractTensorRelaxation:
    pass


@dataclass(frozen=True)
class NoRelaxation(AbstractTensorRelaxation):
    pass


@dataclass(frozen=True)
class MaxwellRelaxation(AbstractTensorRelaxation):
    rate: float

    def __post_init__(self):
        _finite(self.rate, "Maxwell relaxation rate must be finite.")
        if not self.rate >= 0:
            raise ArgumentError("Maxwell relaxation rate must be non-negative.")


class AbstractElasticStressModel:
    pass


@dataclass(frozen=True)
class NoElasticStress(AbstractElasticStressModel):
    pass


@dataclass(frozen=True)
class LinearInternalTensorStress(AbstractElasticStressModel):
    coefficient: float

    def __post_init__(self):
        _finite(self.coefficient, "Elastic-stress coefficient must be finite.")
        if not self.coefficient >= 0:
            raise ArgumentError("Elastic-stress coefficient must be non-negative.")


# ---- Capillarity.jl:15-41 -------------------------------------------------------
class AbstractCapillarity:
    pass


@dataclass(frozen=True)
class NoCapillarity(AbstractCapillarity):
    pass


@dataclass(frozen=True)
class DiffuseAreaCapillarity(AbstractCapillarity):
    coefficient: float
    delta_normal: float = 1e-6
    smoothing_passes: int = 0

    def __post_init__(self):
        _finite(self.coefficient, "coefficient must be finite.")
        if not self.coefficient >= 0:
            raise ArgumentError("coefficient must be nonnegative.")
        _finite(self.delta_normal, "delta_normal must be finite.")
        if not self.delta_normal > 0:
            raise ArgumentError("delta_normal must be positive.")
        if int(self.smoothing_passes) < 0:
            raise ArgumentError("smoothing_passes must be nonnegative.")


# ---- InterfaceRegularization.jl:17-63 and PhaseFieldMethods.jl:22-120 -----------
class AbstractInterfaceFlux:
    pass


@dataclass(frozen=True)
class NoInterfaceFlux(AbstractInterfaceFlux):
    pass


@dataclass(frozen=True)
class ConservativeDiffuseInterfaceFlux(AbstractInterfaceFlux):
    inverse_peclet: float
    epsilon: float
    delta_normal: float = 1e-6

    def __post_init__(self):
        for v, n in ((self.inverse_peclet, "inverse_peclet"), (self.epsilon, "epsilon"),
                     (self.delta_normal, "delta_normal")):
            _finite(v, f"{n} must be finite.")
        if not self.inverse_peclet >= 0:
            raise ArgumentError("inverse_peclet must be non-negative.")
        if not self.epsilon > 0:
            raise ArgumentError("epsilon must be strictly positive.")
        if not self.delta_normal > 0:
            raise ArgumentError("delta_normal must be strictly positive.")


class AbstractPhaseFieldMethod:
    pass


@dataclass(frozen=True)
class LegacySplitPhaseFieldMethod(AbstractPhaseFieldMethod):
    interface_flux: AbstractInterfaceFlux


@dataclass(frozen=True)
class NoPhaseFieldRegularization(AbstractPhaseFieldMethod):
    pass


@dataclass(frozen=True)
class CurrentCDIPhaseField(AbstractPhaseFieldMethod):
    inverse_peclet: float
    epsilon: float
    delta_normal: float = 1e-6

    def __post_init__(self):
        ConservativeDiffuseInterfaceFlux(self.inverse_peclet, self.epsilon, self.delta_normal)

    @property
    def flux(self):
        return ConservativeDiffuseInterfaceFlux(self.inverse_peclet, self.epsilon, self.delta_normal)


@dataclass(frozen=True)
class JainACDIPhaseField(AbstractPhaseFieldMethod):
    gamma: float
    epsilon: float
    psi_floor: float = 1e-100
    delta_normal: float = 1e-14
    dynamic_gamma: bool = True

    def __post_init__(self):
        if not (math.isfinite(self.gamma) and self.gamma >= 0):
            raise ArgumentError("gamma must be finite and non-negative.")
        if not (math.isfinite(self.epsilon) and self.epsilon > 0):
            raise ArgumentError("epsilon must be finite and strictly positive.")
        if not (math.isfinite(self.psi_floor) and 0.0 < self.psi_floor < 0.5):
            raise ArgumentError("psi_floor must lie strictly between 0 and 0.5.")
        if not (math.isfinite(self.delta_normal) and self.delta_normal > 0):
            raise ArgumentError("delta_normal must be finite and strictly positive.")


@dataclass(frozen=True)
class PirozzoliUWCDIPhaseField(AbstractPhaseFieldMethod):
    alpha: float = 1.0
    delta_normal: float = 1e-14
    normal_reconstruction: str = "standard"

    def __post_init__(self):
        if not (math.isfinite(self.alpha) and self.alpha >= 1.0):
            raise ArgumentError("alpha must be finite and >= 1 for the published UWCDI stability range.")
        if not (math.isfinite(self.delta_normal) and self.delta_normal > 0):
            raise ArgumentError("delta_normal must be finite and strictly positive.")
        if self.normal_reconstruction not in ("standard", "youngs", "smoothed9"):
            raise ArgumentError("normal_reconstruction must be :standard, :youngs, or :smoothed9.")


def jain_equilibrium_initialization_epsilon(model: JainACDIPhaseField) -> float:
    return 2.0 * model.epsilon


def phase_field_label(model) -> str:
    if isinstance(model, NoPhaseFieldRegularization):
        return "upwind_no_regularization"
    if isinstance(model, CurrentCDIPhaseField):
        return "current_cdi"
    if isinstance(model, JainACDIPhaseField):
        return "jain_acdi"
    if isinstance(model, PirozzoliUWCDIPhaseField):
        return "pirozzoli_uwcdi"
    if isinstance(model, LegacySplitPhaseFieldMethod):
        return "legacy_split_" + type(model.interface_flux).__name__
    raise ArgumentError("unknown phase-field method")


# ---- StructureTensor.jl:59-131 --------------------------------------------------
class AbstractStructureExtension:
    pass


@dataclass(frozen=True)
class NoStructureExtension(AbstractStructureExtension):
    pass


@dataclass(frozen=True)
class IdentityOutsideStructure(AbstractStructureExtension):
    cutoff: float

    def __post_init__(self):
        _finite(self.cutoff, "Structure-extension cutoff must be finite.")
        if not 0 <= self.cutoff <= 1:
            raise ArgumentError("Structure-extension cutoff must lie in [0, 1].")


@dataclass(frozen=True)
class GeometricStructureExtension(AbstractStructureExtension):
    max_rate: float
    exponent: float = 4.0
    safety_cutoff: float = 1e-6

    def __post_init__(self):
        _finite(self.max_rate, "Geometric extension rate must be finite.")
        if not self.max_rate >= 0:
            raise ArgumentError("Geometric extension rate must be non-negative.")
        _finite(self.exponent, "Geometric extension exponent must be finite.")
        if not self.exponent > 0:
            raise ArgumentError("Geometric extension exponent must be positive.")
        _finite(self.safety_cutoff, "Geometric extension safety cutoff must be finite.")
        if not 0.0 <= self.safety_cutoff < 1.0:
            raise ArgumentError("Geometric extension safety cutoff must lie in [0, 1).")


# ---- TimeIntegrationIMEX.jl:71-301 ------------------------------------------------
@dataclass(frozen=True)
class FourStageIMEXFractionalStep:
    pass


@dataclass(frozen=True)
class LinearSolverOptions:
    """LinearSolverOptions (TimeIntegrationIMEX.jl:211-252).  On the device every
    implicit system is SPD after symmetric Dirichlet elimination and is solved by
    preconditioned CG, each system with its own method: `:direct` maps to a relative
    residual of 1e-13 (the exact solution within round-off, at most
    EFSI_LINEAR_HARD_CAP iterations), `:gmres` to `reltol` and `maxiter`.  The
    result is then judged as _solve_linear_system! judges it (:602-641): a relative
    residual |A x - b| / max(|b|, eps) that is non-finite or above `fallback_reltol`
    continues with the `:direct` iteration when `direct_fallback` is set and
    otherwise raises SolverError (the reference's ErrorException)."""
    velocity_method: str = "direct"
    resource_method: str = "gmres"
    reltol: float = 1e-8
    maxiter: int = 800
    restart: int = 100
    direct_fallback: bool = True
    fallback_reltol: float = 1e-6
    verbose: bool = False

    def __post_init__(self):
        if self.velocity_method not in ("direct", "gmres"):
            raise ArgumentError("velocity_method must be :direct or :gmres.")
        if self.resource_method not in ("direct", "gmres"):
            raise ArgumentError("resource_method must be :direct or :gmres.")
        if not self.reltol > 0:
            raise ArgumentError("Linear-solver reltol must be positive.")
        if not self.maxiter > 0:
            raise ArgumentError("Linear-solver maxiter must be positive.")
        if not self.restart > 0:
            raise ArgumentError("Linear-solver restart must be positive.")
        if not self.fallback_reltol > 0:
            raise ArgumentError("fallback_reltol must be positive.")



@dataclass(frozen=True)
class IMEXNumerics:
    """IMEXNumerics (TimeIntegrationIMEX.jl:262-301) plus two device options of this
    library: the precision form (``precision="fp64"`` for the plain step, ``"mixed"`` for
    FP32 solver bulk with FP64 state, residuals, inner products and refinement) and the
    projection solver (``projection_solver="auto"``: the direct fast-diagonalisation
    solve where the grid has power-of-two sizes and one boundary kind per side of the
    correction potential, the multigrid CG elsewhere; ``"multigrid"``: always the CG).
    Both projection solvers stop on the relative residual ``projection_reltol``."""
    scheme: FourStageIMEXFractionalStep = field(default_factory=FourStageIMEXFractionalStep)
    linear_solvers: LinearSolverOptions = field(default_factory=LinearSolverOptions)
    structure_extension: AbstractStructureExtension = field(default_factory=NoStructureExtension)
    projection_reltol: float = 1e-10
    projection_maxiter: int = 3000
    projection_restart: int = 50
    stage1_constraint_atol: float = 5e-8
    stage1_constraint_rtol: float = 1e-8
    check_stage1_constraint: bool = True
    precision: str = "fp64"
    projection_solver: str = "auto"

    def __post_init__(self):
        if not self.projection_reltol > 0:
            raise ArgumentError("projection_reltol must be positive.")
        if not self.projection_maxiter > 0:
            raise ArgumentError("projection_maxiter must be positive.")
        if not self.projection_restart > 0:
            raise ArgumentError("projection_restart must be positive.")
        if not self.stage1_constraint_atol >= 0:
            raise ArgumentError("stage1_constraint_atol must be non-negative.")
        if not self.stage1_constraint_rtol >= 0:
            raise ArgumentError("stage1_constraint_rtol must be non-negative.")
        if self.precision not in ("fp64", "mixed"):
            raise ArgumentError("precision must be 'fp64' or 'mixed'.")
        if self.projection_solver not in ("auto", "multigrid"):
            raise ArgumentError("projection_solver must be 'auto' or 'multigrid'.")


# ---- flattening into the C structs ------------------------------------------------
def fill_models(out: _abi.Models, m) -> None:
    g = m.growth_source
    if isinstance(g, NoGrowth):
        out.growth_source = _abi.GROWTH_NONE
    elif isinstance(g, ConstantIntrinsicGrowth):
        out.growth_source, out.growth_rate = _abi.GROWTH_CONSTANT, g.rate
    elif isinstance(g, SaturatingResourceGrowth):
        out.growth_source, out.growth_rate, out.growth_half_saturation = (
            _abi.GROWTH_SATURATING, g.rate, g.half_saturation)
    else:
        raise ArgumentError(f"unsupported growth source {g!r}")
    t = m.growth_tensor
    if isinstance(t, IsotropicGrowthTensor):
        out.growth_tensor = _abi.GTENSOR_ISOTROPIC
    elif isinstance(t, DirectionalGrowthTensor):
        out.growth_tensor, out.growth_direction_x, out.growth_direction_y = (
            _abi.GTENSOR_DIRECTIONAL, t.direction_x, t.direction_y)
    else:
        raise ArgumentError(f"unsupported growth tensor {t!r}")
    v = m.viscosity
    if isinstance(v, NoViscosity):
        out.viscosity = _abi.VISC_NONE
    elif isinstance(v, ConstantViscosity):
        out.viscosity, out.viscosity_fluid = _abi.VISC_CONSTANT, v.value
    elif isinstance(v, HarmonicPhaseViscosity):
        out.viscosity, out.viscosity_fluid, out.viscosity_structure = (
            _abi.VISC_HARMONIC, v.fluid_value, v.structure_value)
    else:
        raise ArgumentError(f"unsupported viscosity {v!r}")
    d = m.diffusivity
    if isinstance(d, NoDiffusion):
        out.diffusivity = _abi.DIFF_NONE
    elif isinstance(d, ConstantDiffusivity):
        out.diffusivity, out.diffusivity_fluid = _abi.DIFF_CONSTANT, d.value
    elif isinstance(d, HarmonicPhaseDiffusivity):
        out.diffusivity, out.diffusivity_fluid, out.diffusivity_structure = (
            _abi.DIFF_HARMONIC, d.fluid_value, d.structure_value)
    else:
        raise ArgumentError(f"unsupported diffusivity {d!r}")
    c = m.resource_consumption
    if isinstance(c, NoResourceConsumption):
        out.resource_consumption = _abi.CONSUMPTION_NONE
    elif isinstance(c, SaturatingResourceConsumption):
        out.resource_consumption, out.consumption_rate, out.consumption_half_saturation = (
            _abi.CONSUMPTION_SATURATING, c.rate, c.half_saturation)
    else:
        raise ArgumentError(f"unsupported consumption {c!r}")
    r = m.tensor_relaxation
    if isinstance(r, NoRelaxation):
        out.tensor_relaxation = _abi.RELAX_NONE
    elif isinstance(r, MaxwellRelaxation):
        out.tensor_relaxation, out.relaxation_rate = _abi.RELAX_MAXWELL, r.rate
    else:
        raise ArgumentError(f"unsupported relaxation {r!r}")
    e = m.elastic_stress
    if isinstance(e, NoElasticStress):
        out.elastic_stress = _abi.ELASTIC_NONE
    elif isinstance(e, LinearInternalTensorStress):
        out.elastic_stress, out.elastic_coefficient = _abi.ELASTIC_LINEAR, e.coefficient
    else:
        raise ArgumentError(f"unsupported elastic stress {e!r}")
    k = m.capillarity
    if isinstance(k, NoCapillarity):
        out.capillarity = _abi.CAP_NONE
    elif isinstance(k, DiffuseAreaCapillarity):
        out.capillarity, out.capillary_coefficient = _abi.CAP_DIFFUSE_AREA, k.coefficient
        out.capillary_delta_normal, out.capillary_smoothing_passes = k.delta_normal, int(k.smoothing_passes)
    else:
        raise ArgumentError(f"unsupported capillarity {k!r}")
    pf = m.phase_field_method
    if isinstance(pf, LegacySplitPhaseFieldMethod):
        pf = (NoPhaseFieldRegularization() if isinstance(pf.interface_flux, NoInterfaceFlux)
              else CurrentCDIPhaseField(pf.interface_flux.inverse_peclet, pf.interface_flux.epsilon,
                                        pf.interface_flux.delta_normal))
    if isinstance(pf, NoPhaseFieldRegularization):
        out.phase_field_method = _abi.PF_UPWIND
    elif isinstance(pf, CurrentCDIPhaseField):
        out.phase_field_method = _abi.PF_CDI
        out.pf_param[0], out.pf_param[1], out.pf_param[2] = pf.inverse_peclet, pf.epsilon, pf.delta_normal
    elif isinstance(pf, JainACDIPhaseField):
        out.phase_field_method = _abi.PF_ACDI
        out.pf_param[0], out.pf_param[1], out.pf_param[2], out.pf_param[3] = (
            pf.gamma, pf.epsilon, pf.psi_floor, pf.delta_normal)
        out.pf_option = int(bool(pf.dynamic_gamma))
    elif isinstance(pf, PirozzoliUWCDIPhaseField):
        out.phase_field_method = _abi.PF_UWCDI
        out.pf_param[0], out.pf_param[1] = pf.alpha, pf.delta_normal
        out.pf_option = {"standard": _abi.NORMALS_STANDARD, "youngs": _abi.NORMALS_YOUNGS,
                         "smoothed9": _abi.NORMALS_SMOOTHED9}[pf.normal_reconstruction]
    else:
        raise ArgumentError("phase_field_method must be an AbstractPhaseFieldMethod.")
    b = m.body_force
    if isinstance(b, NoBodyForce):
        out.body_force = _abi.FORCE_NONE
    elif isinstance(b, ConstantBodyForce):
        out.body_force = _abi.FORCE_CONSTANT
        out.body_force_param[0], out.body_force_param[1] = b.fx, b.fy
    elif isinstance(b, KolmogorovBodyForce):
        out.body_force = _abi.FORCE_KOLMOGOROV
        out.body_force_param[0], out.body_force_param[1], out.body_force_param[2] = (
            b.amplitude, b.wavenumber, b.phase)
    else:
        raise ArgumentError(f"unsupported body force {b!r}")


def fill_numerics(out: _abi.Numerics, n: IMEXNumerics) -> None:
    if not isinstance(n.scheme, FourStageIMEXFractionalStep):
        raise ArgumentError(f"Unsupported IMEX scheme {type(n.scheme).__name__}.")
    e = n.structure_extension
    if isinstance(e, NoStructureExtension):
        out.structure_extension = _abi.EXT_NONE
    elif isinstance(e, IdentityOutsideStructure):
        out.structure_extension, out.extension_cutoff = _abi.EXT_IDENTITY_OUTSIDE, e.cutoff
    elif isinstance(e, GeometricStructureExtension):
        out.structure_extension = _abi.EXT_GEOMETRIC
        out.extension_rate, out.extension_exponent, out.extension_cutoff = (
            e.max_rate, e.exponent, e.safety_cutoff)
    else:
        raise ArgumentError(f"unsupported structure extension {e!r}")
    out.projection_reltol = n.projection_reltol
    out.projection_maxiter = int(n.projection_maxiter)
    out.stage1_constraint_atol = n.stage1_constraint_atol
    out.stage1_constraint_rtol = n.stage1_constraint_rtol
    out.check_stage1_constraint = int(bool(n.check_stage1_constraint))
    ls = n.linear_solvers
    method = {"direct": _abi.LINEAR_DIRECT, "gmres": _abi.LINEAR_GMRES}
    out.velocity_method = method[ls.velocity_method]
    out.resource_method = method[ls.resource_method]
    out.linear_reltol = ls.reltol
    out.linear_maxiter = int(ls.maxiter)
    out.direct_fallback = int(bool(ls.direct_fallback))
    out.fallback_reltol = ls.fallback_reltol
    out.precision = _abi.PRECISION_MIXED if n.precision == "mixed" else _abi.PRECISION_FP64
    out.projection_solver = (_abi.PROJECTION_MULTIGRID if n.projection_solver == "multigrid"
                             else _abi.PROJECTION_AUTO)
