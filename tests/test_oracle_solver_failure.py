"""The oracle's restatement of _solve_linear_system! (TimeIntegrationIMEX.jl:602-641):
an unconverged GMRES-method solve whose relative residual exceeds fallback_reltol
throws the reference's ErrorException text without direct_fallback, and falls back
to the exact solve with it.  CPU only; the CUDA step is held to the same behaviour
in tests/test_gpu_solver_failure.py."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import _abi, workloads
from eulerianfsi_b200.imex import ConfigBlock, Handle
from oracle.oracle import load
from tests.helpers import fz, rel_l2


def _oracle(w, **ls_kw):
    ls = dataclasses.replace(w.numerics.linear_solvers, **ls_kw)
    num = dataclasses.replace(w.numerics, linear_solvers=ls, projection_reltol=1e-13)
    h = Handle(load(), "oracle_", ConfigBlock(w.metrics, w.bcs, w.models, num), w.metrics)
    st = w.state.copy()
    h.upload(st)
    h.set_correction(fz(w.metrics.Nx, w.metrics.Ny))
    return h, st


def test_oracle_velocity_failure_message():
    w = workloads.cavity_disk(N=12)
    h, _ = _oracle(w, velocity_method="gmres", reltol=1e-8, maxiter=1, direct_fallback=False)
    with pytest.raises(ef.SolverError, match="velocity stage 2 GMRES residual is too large"):
        h.call("integrate_step", 0.0, w.dt, C.byref(_abi.StepReportC()))


def test_oracle_resource_failure_message():
    w = workloads.channel_growth(N=8)
    h, _ = _oracle(w, velocity_method="direct", resource_method="gmres", reltol=1e-12, maxiter=1,
                   direct_fallback=False, fallback_reltol=1e-15)
    h.call("make_velocity_compatible", C.byref(_abi.ProjectionResultC()))
    h.set_correction(fz(w.metrics.Nx, w.metrics.Ny))
    with pytest.raises(ef.SolverError, match="resource stage 2 GMRES residual is too large"):
        h.call("integrate_step", 0.0, w.dt, C.byref(_abi.StepReportC()))


def test_oracle_fallback_equals_direct():
    w = workloads.cavity_disk(N=12)
    out = []
    for kw in (dict(velocity_method="gmres", reltol=1e-8, maxiter=1, direct_fallback=True),
               dict(velocity_method="direct")):
        h, st = _oracle(w, **kw)
        h.call("integrate_step", 0.0, w.dt, C.byref(_abi.StepReportC()))
        h.download(st)
        out.append(st)
    for name in ("U", "V", "phi", "sigma_xx", "sigma_yy", "sigma_xy"):
        assert rel_l2(getattr(out[0], name), getattr(out[1], name)) <= 1e-11, name


def test_linear_solver_options_flatten_per_system():
    ls = ef.LinearSolverOptions(velocity_method="direct", resource_method="gmres", reltol=1e-5, maxiter=17,
                                direct_fallback=False, fallback_reltol=1e-4)
    n = _abi.Numerics()
    ef.models.fill_numerics(n, ef.IMEXNumerics(linear_solvers=ls))
    assert (n.velocity_method, n.resource_method) == (_abi.LINEAR_DIRECT, _abi.LINEAR_GMRES)
    assert (n.linear_reltol, n.linear_maxiter, n.direct_fallback, n.fallback_reltol) == (1e-5, 17, 0, 1e-4)
