"""Differentiation form of the IMEX step: the discrete adjoint behind an rrule.

``rrule_integrate_steps(state, t0, dts, context)`` is the Python counterpart of the
``ChainRulesCore.rrule`` a Julia caller binds (the reference has no adjoint): it runs
the steps forward on the device with sqrt(n) checkpoints (``efsi_forward_checkpointed``)
and returns the final state with a pullback.  The pullback maps the cotangent of the
final state to the cotangent of the initial state and of the parameters it
differentiates: the elastic coefficient G of LinearInternalTensorStress and the
tangential wall velocity data (U bottom/top, V left/right).  It recomputes each
segment between checkpoints once, recording its stage fields, and sweeps it
backwards (``efsi_backward``): transposed explicit stencils, transposed projections
(a Poisson solve with the same SPD operator) and transposed viscous solves.

The model set it differentiates is the one ``efsi_backward`` accepts: ACDI with a
fixed mobility, constant or no viscosity, linear elastic stress, Maxwell relaxation,
any structure extension and body force; growth, resource transport and capillarity
raise UnsupportedError.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from .imex import FSIState, IMEXContext, field64


@dataclass
class ParameterGradient:
    """Cotangents of the differentiated parameters."""
    elastic_coefficient: float
    U_bottom: np.ndarray
    U_top: np.ndarray
    V_left: np.ndarray
    V_right: np.ndarray


def _gradient_struct(Nx, Ny):
    g = _abi.GradientC()
    arrays = {"U_bottom": np.zeros(Nx + 1), "U_top": np.zeros(Nx + 1),
              "V_left": np.zeros(Ny + 1), "V_right": np.zeros(Ny + 1)}
    for k, a in arrays.items():
        setattr(g, k, _abi.dptr(a))
    return g, arrays


def forward_checkpointed(state: FSIState, t0: float, dts, context: IMEXContext, every: int = 0,
                         correction=None) -> list:
    """Advance `state` in place through the steps `dts` (device-resident, one
    checkpoint every `every` steps, 0 = ceil(sqrt(n))) and return the StepReports.
    `correction` is the projection warm start (zeros when None)."""
    from .imex import StepReport
    h = context.handle
    m = context.metrics
    h.upload(state)
    h.set_correction(np.zeros((m.Nx, m.Ny), order="F") if correction is None else correction)
    dts = np.ascontiguousarray(dts, dtype=np.float64)
    n = len(dts)
    reps = (_abi.StepReportC * n)()
    h.call("forward_checkpointed", float(t0), _abi.dptr(dts), n, int(every), reps)
    h.download(state)
    return [StepReport.from_c(r) for r in reps]


def backward(context: IMEXContext, cotangent: FSIState | dict):
    """Pullback of the last forward_checkpointed run on `context`: the cotangent of the
    final state (an FSIState, or a dict of its U, V, phi, sigma_* arrays; missing
    entries are zero) -> (cotangent of the initial state as an FSIState,
    ParameterGradient)."""
    h = context.handle
    m = context.metrics
    Nx, Ny = m.Nx, m.Ny
    shapes = {"U": (Nx + 1, Ny), "V": (Nx, Ny + 1), "phi": (Nx, Ny), "sigma_xx": (Nx, Ny),
              "sigma_yy": (Nx, Ny), "sigma_xy": (Nx, Ny)}
    get = (lambda k: getattr(cotangent, k)) if isinstance(cotangent, FSIState) else cotangent.get
    seeds = {k: (field64(get(k), s) if get(k) is not None else None) for k, s in shapes.items()}
    out = {k: np.zeros(s, order="F") for k, s in shapes.items()}
    g, arrays = _gradient_struct(Nx, Ny)
    names = ("U", "V", "phi", "sigma_xx", "sigma_yy", "sigma_xy")
    h.call("backward", *[_abi.dptr(seeds[k]) for k in names], *[_abi.dptr(out[k]) for k in names], C.byref(g))
    grad_state = FSIState(out["U"], out["V"], out["phi"], np.zeros((Nx, Ny), order="F"), out["sigma_xx"],
                          out["sigma_yy"], out["sigma_xy"])
    return grad_state, ParameterGradient(float(g.elastic_coefficient), **arrays)


def rrule_integrate_steps(state: FSIState, t0: float, dts, context: IMEXContext, every: int = 0):
    """(final state, pullback) of n steps from `state` (left unchanged), the shape of
    ChainRulesCore.rrule(integrate_steps, state, t0, dts, context)."""
    final = state.copy()
    forward_checkpointed(final, t0, dts, context, every)

    def pullback(cotangent):
        return backward(context, cotangent)

    return final, pullback


def tendencies_adjoint(context: IMEXContext, fields: FSIState, lam: dict):
    """Transposed Jacobian of one stage's explicit tendencies at `fields`: `lam` maps
    "Eu", "Ev", "Iu", "Iv" (compact rows, Nx x Ny), "Ephi", "Exx", "Eyy", "Exy" to
    their cotangents (missing = zero); returns (cotangent of the six stage fields as a
    dict, ParameterGradient).  The dot-product tests of the transposed stencils use it."""
    h = context.handle
    m = context.metrics
    Nx, Ny = m.Nx, m.Ny
    shapes = {"U": (Nx + 1, Ny), "V": (Nx, Ny + 1)}
    arrs = [field64(a, shapes.get(k, (Nx, Ny))) for k, a in
            (("U", fields.U), ("V", fields.V), ("phi", fields.phi), ("sxx", fields.sigma_xx),
             ("syy", fields.sigma_yy), ("sxy", fields.sigma_xy))]
    keys = ("Eu", "Ev", "Iu", "Iv", "Ephi", "Exx", "Eyy", "Exy")
    seeds = [field64(lam[k], (Nx, Ny)) if lam.get(k) is not None else None for k in keys]
    out = {"U": np.zeros((Nx + 1, Ny), order="F"), "V": np.zeros((Nx, Ny + 1), order="F")}
    for k in ("phi", "sigma_xx", "sigma_yy", "sigma_xy"):
        out[k] = np.zeros((Nx, Ny), order="F")
    g, arrays = _gradient_struct(Nx, Ny)
    h.call("tendencies_adjoint", *[_abi.dptr(a) for a in arrs], *[_abi.dptr(a) for a in seeds],
           *[_abi.dptr(out[k]) for k in ("U", "V", "phi", "sigma_xx", "sigma_yy", "sigma_xy")], C.byref(g))
    return out, ParameterGradient(float(g.elastic_coefficient), **arrays)


def project_adjoint(context: IMEXContext, lam_U, lam_V):
    """Transposed efsi_project: cotangent of the input faces from that of the output."""
    h = context.handle
    m = context.metrics
    lu = field64(lam_U, (m.Nx + 1, m.Ny))
    lv = field64(lam_V, (m.Nx, m.Ny + 1))
    ou = np.zeros((m.Nx + 1, m.Ny), order="F")
    ov = np.zeros((m.Nx, m.Ny + 1), order="F")
    h.call("project_adjoint", _abi.dptr(lu), _abi.dptr(lv), _abi.dptr(ou), _abi.dptr(ov))
    return ou, ov
