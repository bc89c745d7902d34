"""Driver diagnostics of the cavity benchmarks on the device-resident state.

The reference computes these on the host every output step
(scripts/benchmarks/run_sugiyama_lid_driven_cavity.jl:484-934); here one call
reduces them on the GPU and returns a few hundred bytes, so a time loop run with
``efsi_step_n`` needs no state download.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

from . import _abi

REGIONS = ("global_region", "core", "interface", "tail")


@dataclass
class DiagnosticsConfig:
    """Parameters of the diagnostics (BenchmarkConfig fields of the cavity driver)."""
    density: float = 1.0
    elastic_modulus: float = 0.1
    sigma_core_cutoff: float = 0.9
    sigma_interface_cutoff: float = 0.1
    sigma_safety_cutoff: float = 1e-6
    h_interface: float = 1.0
    nmax: int = 4

    def to_c(self) -> _abi.DiagConfig:
        if not 0 <= self.nmax <= _abi.DIAG_MAX_MODES:
            raise ValueError("nmax must lie in 0..8")
        c = _abi.DiagConfig()
        for name in ("density", "elastic_modulus", "sigma_core_cutoff", "sigma_interface_cutoff",
                     "sigma_safety_cutoff", "h_interface"):
            setattr(c, name, float(getattr(self, name)))
        c.nmax = int(self.nmax)
        return c


def to_dict(d: _abi.Diagnostics, nmax: int) -> dict:
    out = {}
    for name, _ in _abi.Diagnostics._fields_:
        if name in ("Rc", "Rs", "amplitudes"):
            out[name] = list(getattr(d, name))[:nmax]
        elif name == "tensor":
            for r, region in enumerate(REGIONS):
                t = d.tensor[r]
                out[region] = {f: getattr(t, f) for f, _ in _abi.TensorRegion._fields_}
        else:
            out[name] = getattr(d, name)
    return out


def state_diagnostics(handle, config: DiagnosticsConfig | None = None) -> dict:
    """phase_centroid, phase_geometry_diagnostics, phase_bound_diagnostics,
    flow_diagnostics, tensor_diagnostics_detailed and the speed maxima of
    comparison_timestep_bounds for the state held by `handle` (a context handle of
    the CUDA library, or of the oracle)."""
    config = config or DiagnosticsConfig()
    c = config.to_c()
    d = _abi.Diagnostics()
    handle.call("state_diagnostics", C.byref(c), C.byref(d))
    return to_dict(d, config.nmax)


def comparison_timestep_bounds(max_abs_U: float, max_abs_V: float, *, hx: float, hy: float, U_lid: float,
                               elastic_modulus: float, density: float, cfl_hyperbolic: float, Pe_gamma: float,
                               cfl_interface_compression: float, cfl_interface_diffusion: float,
                               cdi_epsilon: float, acdi_gamma: float, acdi_epsilon: float, uwcdi_alpha: float,
                               dt_max: float) -> dict:
    """comparison_timestep_bounds (run_sugiyama_lid_driven_cavity.jl:852-934), with
    the velocity maxima taken from state_diagnostics."""
    eps = 2.220446049250313e-16
    hmin = min(hx, hy)
    max_adv = max(U_lid, max_abs_U, max_abs_V)
    wave = math.sqrt(elastic_modulus / density)
    hyper = max(max_adv, wave, eps)
    dt_h = cfl_hyperbolic * hmin / hyper
    inv_pe = 1.0 / Pe_gamma
    dt_cdi_c = cfl_interface_compression * hmin / inv_pe
    nu_cdi = 0.5 * cdi_epsilon * inv_pe
    dt_cdi_d = cfl_interface_diffusion * (1.0 / (2.0 * nu_cdi * (1.0 / hx ** 2 + 1.0 / hy ** 2)))
    dt_acdi_c = cfl_interface_compression * hmin / max(acdi_gamma, eps)
    nu_acdi = acdi_gamma * acdi_epsilon
    dt_acdi_d = (cfl_interface_diffusion / (2.0 * nu_acdi * (1.0 / hx ** 2 + 1.0 / hy ** 2))
                 if nu_acdi > 0.0 else math.inf)
    uw_lim = 1.0 / (1.0 + 1.0 / uwcdi_alpha)
    dt_uw = uw_lim * hmin / max(max_adv, eps)
    labels = ("hyperbolic", "current_cdi_compression", "current_cdi_diffusion", "acdi_compression",
              "acdi_diffusion", "uwcdi", "dt_max")
    values = (dt_h, dt_cdi_c, dt_cdi_d, dt_acdi_c, dt_acdi_d, dt_uw, dt_max)
    k = min(range(len(values)), key=lambda n: values[n])  # first minimum, as findmin
    return {"hyperbolic": dt_h, "cdi_compression": dt_cdi_c, "cdi_diffusion": dt_cdi_d,
            "acdi_compression": dt_acdi_c, "acdi_diffusion": dt_acdi_d, "uwcdi": dt_uw,
            "selected": values[k], "limiting_constraint": labels[k], "max_advection_speed": max_adv,
            "elastic_wave_speed": wave, "gamma_acdi": acdi_gamma}
