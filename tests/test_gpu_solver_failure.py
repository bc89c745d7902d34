"""Linear-solve failure semantics of the CUDA step, against _solve_linear_system!
(TimeIntegrationIMEX.jl:602-641): a velocity or resource solve that ends with a
relative residual |A x - b| / max(|b|, eps) above fallback_reltol either falls back
to the exact (DIRECT) solve or raises the reference's ErrorException ("... GMRES
residual is too large"), leaving the state as it was.  The velocity and resource
systems take their tolerances from their own methods.

Every failure here is made on the host (an iteration cap of one or two); the device
loops are bounded and nothing faults."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import _abi, workloads
from tests.gpu_util import pair, rel_err
from tests.helpers import fz

pytestmark = pytest.mark.gpu

FIELDS = ("U", "V", "phi", "resource", "sigma_xx", "sigma_yy", "sigma_xy")


def _with_solvers(numerics, **ls_kw):
    ls = dataclasses.replace(numerics.linear_solvers, **ls_kw)
    return dataclasses.replace(numerics, linear_solvers=ls, projection_reltol=1e-13, projection_maxiter=3000)


def _context(w, numerics):
    ctx = ef.build_imex_context(w.metrics, w.bcs, w.models, numerics=numerics)
    return ctx, ef.allocate_imex_workspace(w.metrics)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_velocity_solve_failure_raises_and_keeps_state(precision):
    w = workloads.cavity_disk(N=16)
    num = dataclasses.replace(_with_solvers(w.numerics, velocity_method="gmres", reltol=1e-8, maxiter=2,
                                            direct_fallback=False), precision=precision)
    ctx, work = _context(w, num)
    st = w.state.copy()
    before = st.copy()
    with pytest.raises(ef.SolverError, match="velocity stage 2 GMRES residual is too large"):
        ef.integrate_step(st, 0.0, w.dt, ctx, work)
    for name in FIELDS:
        np.testing.assert_array_equal(getattr(st, name), getattr(before, name))
    # the context is still usable: the same state steps with a solvable configuration
    ctx2, work2 = _context(w, _with_solvers(w.numerics, velocity_method="direct"))
    ef.integrate_step(st, 0.0, w.dt, ctx2, work2)
    assert np.all(np.isfinite(st.U))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_velocity_solve_fallback_matches_oracle(precision):
    """An iteration cap below what the solve needs, with direct_fallback: the DIRECT
    continuation gives the exact predictor, so two steps agree with the oracle's direct
    solves to 1e-10.  The cap is 2 CG iterations for FP64; the precision form meets
    1e-8 at 16^2 in two launches (one Chebyshev launch and its FP64 refinement), so its
    cap is one launch."""
    w = workloads.cavity_disk(N=16)
    cap = 2 if precision == "fp64" else 1
    num_gpu = dataclasses.replace(_with_solvers(w.numerics, velocity_method="gmres", reltol=1e-8, maxiter=cap,
                                                direct_fallback=True), precision=precision)
    num_ora = _with_solvers(w.numerics, velocity_method="direct")
    gpu, _ = pair(w.metrics, w.bcs, w.models, num_gpu)
    _, ora = pair(w.metrics, w.bcs, w.models, num_ora)
    states = []
    for h in (gpu, ora):
        st = w.state.copy()
        h.upload(st)
        h.set_correction(fz(w.metrics.Nx, w.metrics.Ny))
        t = 0.0
        for _ in range(2):
            rep = _abi.StepReportC()
            h.call("integrate_step", t, w.dt, C.byref(rep))
            t += w.dt
        h.download(st)
        states.append(st)
    assert max(gpu.stats()["velocity_iterations"][1:4]) > cap  # the continuation ran past the cap
    tol = 1e-10 if precision == "fp64" else 1e-8
    for name in FIELDS:
        assert rel_err(getattr(states[0], name), getattr(states[1], name)) <= tol, name


def test_resource_solve_failure_raises_and_keeps_state():
    w = workloads.channel_growth(N=16)
    num = _with_solvers(w.numerics, velocity_method="direct", resource_method="gmres", reltol=1e-12, maxiter=1,
                        direct_fallback=False, fallback_reltol=1e-15)
    ctx, work = _context(w, num)
    st = w.state.copy()
    ef.make_velocity_compatible(st, ctx, work)
    work.correction[...] = 0.0
    before = st.copy()
    with pytest.raises(ef.SolverError, match="resource stage 2 GMRES residual is too large"):
        ef.integrate_step(st, 0.0, w.dt, ctx, work)
    for name in FIELDS:
        np.testing.assert_array_equal(getattr(st, name), getattr(before, name))


def test_unconverged_solve_within_fallback_tolerance_is_accepted():
    """The reference accepts a GMRES result that stops at maxiter if its relative
    residual is within fallback_reltol; so does the device step."""
    w = workloads.cavity_disk(N=16)
    num = _with_solvers(w.numerics, velocity_method="gmres", reltol=1e-14, maxiter=12, direct_fallback=False,
                        fallback_reltol=1e-2)
    ctx, work = _context(w, num)
    st = w.state.copy()
    ef.integrate_step(st, 0.0, w.dt, ctx, work)
    assert np.all(np.isfinite(st.U))


def test_velocity_and_resource_methods_are_separate():
    """Velocity :direct with resource :gmres at a loose reltol, then the reverse: each
    system's iteration count follows its own method."""
    w = workloads.channel_growth(N=32)
    its = {}
    for key, kw in {"vdir": dict(velocity_method="direct", resource_method="gmres"),
                    "rdir": dict(velocity_method="gmres", resource_method="direct")}.items():
        num = _with_solvers(w.numerics, reltol=1e-3, maxiter=800, **kw)
        gpu, _ = pair(w.metrics, w.bcs, w.models, num)
        st = w.state.copy()
        gpu.upload(st)
        gpu.set_correction(fz(w.metrics.Nx, w.metrics.Ny))
        r = _abi.ProjectionResultC()
        gpu.call("make_velocity_compatible", C.byref(r))
        rep = _abi.StepReportC()
        gpu.call("integrate_step", 0.0, w.dt, C.byref(rep))
        s = gpu.stats()
        its[key] = (sum(s["velocity_iterations"]), sum(s["resource_iterations"]))
    assert its["vdir"][0] > its["rdir"][0]
    assert its["vdir"][1] < its["rdir"][1]
