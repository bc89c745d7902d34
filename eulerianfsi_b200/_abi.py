"""ctypes mirror of ``include/efsi.h`` and the loader of the CUDA library.

The structures below must match the C declarations byte for byte; a CPU test
compiles a C translation unit against the header and compares ``sizeof`` and
field offsets with these definitions.
"""
from __future__ import annotations

import ctypes as C
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_int32, c_int64, c_uint8, c_void_p

ABI_VERSION = 2

# status codes
OK, ARG, DIM, SOLVE, DOMAIN, CUDA, UNSUPPORTED = range(7)

# boundary-condition kinds
BC_PERIODIC, BC_DIRICHLET, BC_NEUMANN, BC_MIXED, BC_ADVECTIVE_OUTFLOW = range(5)

GROWTH_NONE, GROWTH_CONSTANT, GROWTH_SATURATING = range(3)
GTENSOR_ISOTROPIC, GTENSOR_DIRECTIONAL = range(2)
VISC_NONE, VISC_CONSTANT, VISC_HARMONIC = range(3)
DIFF_NONE, DIFF_CONSTANT, DIFF_HARMONIC = range(3)
CONSUMPTION_NONE, CONSUMPTION_SATURATING = range(2)
RELAX_NONE, RELAX_MAXWELL = range(2)
ELASTIC_NONE, ELASTIC_LINEAR = range(2)
CAP_NONE, CAP_DIFFUSE_AREA = range(2)
PF_UPWIND, PF_CDI, PF_ACDI, PF_UWCDI = range(4)
NORMALS_STANDARD, NORMALS_YOUNGS, NORMALS_SMOOTHED9 = range(3)
FORCE_NONE, FORCE_CONSTANT, FORCE_KOLMOGOROV = range(3)
EXT_NONE, EXT_IDENTITY_OUTSIDE, EXT_GEOMETRIC = range(3)
PRECISION_FP64, PRECISION_MIXED = range(2)
LINEAR_DIRECT, LINEAR_GMRES = range(2)
LINEAR_HARD_CAP = 10000
PROJECTION_AUTO, PROJECTION_MULTIGRID = range(2)
STEP_GRAPH, STEP_HOST = range(2)

_dp = POINTER(c_double)


class BCSide(Structure):
    _fields_ = [("type", c_int32), ("n", c_int32), ("value", _dp), ("neumann", _dp),
                ("mask", POINTER(c_uint8))]


class BCSetup(Structure):
    _fields_ = [("left", BCSide), ("right", BCSide), ("bottom", BCSide), ("top", BCSide)]


class Mesh(Structure):
    _fields_ = [("Nx", c_int32), ("Ny", c_int32), ("Lx", c_double), ("Ly", c_double),
                ("periodic_x", c_int32), ("periodic_y", c_int32)] + [
        (name, _dp) for name in (
            "dx_f", "dx_c", "dy_f", "dy_c",
            "wL_c2fx", "wR_c2fx", "wB_c2fy", "wT_c2fy",
            "wL_f2cx", "wR_f2cx", "wB_f2cy", "wT_f2cy",
            "dx_west_corner", "dx_east_corner", "dy_south_corner", "dy_north_corner")]


class Models(Structure):
    _fields_ = [
        ("growth_source", c_int32), ("growth_rate", c_double), ("growth_half_saturation", c_double),
        ("growth_tensor", c_int32), ("growth_direction_x", c_double), ("growth_direction_y", c_double),
        ("viscosity", c_int32), ("viscosity_fluid", c_double), ("viscosity_structure", c_double),
        ("diffusivity", c_int32), ("diffusivity_fluid", c_double), ("diffusivity_structure", c_double),
        ("resource_consumption", c_int32), ("consumption_rate", c_double),
        ("consumption_half_saturation", c_double),
        ("tensor_relaxation", c_int32), ("relaxation_rate", c_double),
        ("elastic_stress", c_int32), ("elastic_coefficient", c_double),
        ("capillarity", c_int32), ("capillary_coefficient", c_double),
        ("capillary_delta_normal", c_double), ("capillary_smoothing_passes", c_int32),
        ("phase_field_method", c_int32), ("pf_param", c_double * 4), ("pf_option", c_int32),
        ("body_force", c_int32), ("body_force_param", c_double * 3),
    ]


class Numerics(Structure):
    _fields_ = [
        ("structure_extension", c_int32), ("extension_rate", c_double),
        ("extension_exponent", c_double), ("extension_cutoff", c_double),
        ("projection_reltol", c_double), ("projection_maxiter", c_int32),
        ("stage1_constraint_atol", c_double), ("stage1_constraint_rtol", c_double),
        ("check_stage1_constraint", c_int32),
        ("linear_reltol", c_double), ("linear_maxiter", c_int32),
        ("precision", c_int32), ("velocity_method", c_int32), ("resource_method", c_int32),
        ("direct_fallback", c_int32), ("fallback_reltol", c_double), ("projection_solver", c_int32),
        ("reserved", c_int32 * 3),
    ]


class Config(Structure):
    _fields_ = [("abi_version", c_int32), ("mesh", Mesh)] + [
        (name, BCSetup) for name in (
            "bc_U", "bc_V", "bc_correction", "bc_phi", "bc_resource",
            "bc_sigma_xx", "bc_sigma_yy", "bc_sigma_xy")] + [
        ("models", Models), ("numerics", Numerics)]


class StepReportC(Structure):
    _fields_ = [
        ("maximum_projection_constraint_linf", c_double),
        ("maximum_growth_trace_error", c_double),
        ("minimum_phi", c_double), ("maximum_phi", c_double),
        ("minimum_resource", c_double), ("minimum_sigma_eigenvalue", c_double),
        ("maximum_abs_sigma_determinant_error", c_double),
        ("non_spd_cells", c_int64),
    ]


class ProjectionResultC(Structure):
    _fields_ = [("linear_relative_residual", c_double), ("constraint_linf", c_double),
                ("constraint_l2", c_double), ("compatibility_defect", c_double)]


class Stats(Structure):
    _fields_ = [("projection_iterations", c_int32 * 4), ("velocity_iterations", c_int32 * 4),
                ("resource_iterations", c_int32 * 4), ("kernel_launches", c_int64),
                ("device_ms", c_double), ("site_launches", c_int64), ("site_ms", c_double),
                ("site_bytes", c_double), ("step_bytes", c_double)]


class GradientC(Structure):
    _fields_ = [("elastic_coefficient", c_double), ("U_bottom", _dp), ("U_top", _dp), ("V_left", _dp),
                ("V_right", _dp)]


DIAG_MAX_MODES = 8


class DiagConfig(Structure):
    _fields_ = [("density", c_double), ("elastic_modulus", c_double), ("sigma_core_cutoff", c_double),
                ("sigma_interface_cutoff", c_double), ("sigma_safety_cutoff", c_double),
                ("h_interface", c_double), ("nmax", c_int32), ("reserved", c_int32 * 3)]


class TensorRegion(Structure):
    _fields_ = [("cells", c_int64)] + [(n, c_double) for n in (
        "area", "determinant_min", "determinant_max", "max_abs_determinant_error",
        "mean_abs_determinant_error", "lambda_min", "lambda_max")] + [
        ("non_spd_cells", c_int64), ("max_effective_stress", c_double), ("mean_effective_stress", c_double)]


class Diagnostics(Structure):
    _fields_ = [(n, c_double) for n in (
        "x_centroid", "y_centroid", "phase_integral", "perimeter_proxy", "mixed_layer_measure",
        "effective_interface_width", "effective_interface_cells", "covariance_major", "covariance_minor",
        "aspect_ratio", "orientation_radians", "R0")] + [
        ("Rc", c_double * DIAG_MAX_MODES), ("Rs", c_double * DIAG_MAX_MODES),
        ("amplitudes", c_double * DIAG_MAX_MODES)] + [(n, c_double) for n in (
            "phi_minimum", "phi_maximum", "lower_violation", "upper_violation")] + [
        ("out_of_bounds_cells", c_int64)] + [(n, c_double) for n in (
            "maximum_speed", "kinetic_energy", "divergence_linf", "divergence_l2", "max_abs_U", "max_abs_V")] + [
        ("tensor", TensorRegion * 4)]


SITES = ["phase", "momentum", "structure", "visc_apply", "visc_cg", "visc_init", "pcg_matvec",
         "pcg_update", "vcycle", "proj_rhs", "proj_finish", "combine", "vel_rhs", "finalize", "spectral"]


# Entry points shared by the CUDA library (prefix "efsi_") and the CPU oracle
# (prefix "oracle_"): name -> (restype, argtypes)
_H = c_void_p
SIGNATURES = {
    "create": (c_int32, [POINTER(Config), POINTER(c_void_p)]),
    "destroy": (None, [_H]),
    "last_error": (c_char_p, [_H]),
    "upload_state": (c_int32, [_H] + [_dp] * 7),
    "download_state": (c_int32, [_H] + [_dp] * 7),
    "set_correction": (c_int32, [_H, _dp]),
    "get_correction": (c_int32, [_H, _dp]),
    "make_velocity_compatible": (c_int32, [_H, POINTER(ProjectionResultC)]),
    "integrate_step": (c_int32, [_H, c_double, c_double, POINTER(StepReportC)]),
    "project": (c_int32, [_H, _dp, _dp, _dp, POINTER(ProjectionResultC)]),
    "phase_field_rhs": (c_int32, [_H, _dp, _dp, _dp, _dp, _dp]),
    "structure_tensor_rhs": (c_int32, [_H] + [_dp] * 10),
    "momentum_explicit_rhs": (c_int32, [_H, c_double] + [_dp] * 9),
    "apply_viscous_operator": (c_int32, [_H, _dp, _dp, _dp]),
    "get_stats": (c_int32, [_H, POINTER(Stats)]),
    "uwcdi_strang_step": (c_int32, [_H, _dp, _dp, _dp, c_double, c_int32, _dp]),
    "state_diagnostics": (c_int32, [_H, POINTER(DiagConfig), POINTER(Diagnostics)]),
}
CUDA_ONLY = {
    "set_timed_site": (c_int32, [_H, c_int32]),
    "set_step_mode": (c_int32, [_H, c_int32]),
    "forward_checkpointed": (c_int32, [_H, c_double, _dp, c_int32, c_int32, POINTER(StepReportC)]),
    "backward": (c_int32, [_H] + [_dp] * 12 + [c_void_p]),
    "tendencies_adjoint": (c_int32, [_H] + [_dp] * 20 + [c_void_p]),
    "project_adjoint": (c_int32, [_H] + [_dp] * 4),
    "integrate_step_host": (c_int32, [_H] + [_dp] * 8 + [c_double, c_double, POINTER(StepReportC)]),
    "step_n": (c_int32, [_H, c_double, _dp, c_int32, POINTER(StepReportC)]),
    # no handle: device pointers in, device result out (allocates nothing)
    "divergence_residual_noalloc": (c_int32, [c_int32, c_int32, c_double, c_double, c_void_p, c_void_p,
                                              c_void_p, c_void_p, c_void_p]),
}

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(PACKAGE_DIR, "libefsi.so")


def bind(lib: C.CDLL, prefix: str, extra: dict | None = None) -> C.CDLL:
    table = dict(SIGNATURES)
    if extra:
        table.update(extra)
    for name, (res, args) in table.items():
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


def load_library() -> C.CDLL:
    """Load the in-tree CUDA library; there is no fallback implementation."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY_PATH):
            raise RuntimeError(
                f"CUDA library {LIBRARY_PATH} is missing: build it with "
                "`python -m eulerianfsi_b200.build` (nvcc, sm_100a). The device step has no CPU fallback.")
        _LIB = bind(C.CDLL(LIBRARY_PATH), "efsi_", CUDA_ONLY)
    return _LIB


def dptr(a):
    """Pointer to the first element of a contiguous float64 numpy array (or NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(_dp)
