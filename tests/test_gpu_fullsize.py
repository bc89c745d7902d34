"""The benchmark workloads at their full sizes on the GPU.

* One FP64 step of the 1024 x 1024 twenty-disk cavity and of the 1024 x 512 growth
  channel against the FP64 oracle, solves converged to 1e-13 on both sides: every
  field within 1e-10 relative L2.
* Size-independent properties over 20 device-resident steps of the 1024 x 1024
  cavity, in both precision forms: phase mass conserved to 1e-12 relative, the
  projected velocity satisfies the divergence constraint, every structure tensor stays
  SPD, every field stays finite."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from eulerianfsi_b200 import _abi, workloads
from tests.gpu_util import pair
from tests.helpers import fz
from tests.test_gpu_parity import STEP_TOL, _assert_states

pytestmark = pytest.mark.gpu


def _tight(numerics):
    ls = dataclasses.replace(numerics.linear_solvers, velocity_method="gmres", reltol=1e-13, maxiter=4000)
    return dataclasses.replace(numerics, linear_solvers=ls, projection_reltol=1e-13, projection_maxiter=3000)


@pytest.mark.parametrize("name", ["cavity_disks20", "channel_growth"])
def test_full_size_step_against_oracle(name):
    w = workloads.cavity_disks20(N=1024) if name == "cavity_disks20" else workloads.channel_growth(N=512)
    gpu, ora = pair(w.metrics, w.bcs, w.models, _tight(w.numerics))
    out = []
    for h in (gpu, ora):
        st = w.state.copy()
        h.upload(st)
        h.set_correction(fz(w.metrics.Nx, w.metrics.Ny))
        if w.needs_compatible_start:
            h.call("make_velocity_compatible", C.byref(_abi.ProjectionResultC()))
        rep = _abi.StepReportC()
        h.call("integrate_step", 0.0, w.dt, C.byref(rep))
        h.download(st)
        out.append(st)
    _assert_states(out[0], out[1], STEP_TOL)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_full_size_properties_over_twenty_steps(precision):
    w = workloads.cavity_disks20(N=1024, precision=precision)
    gpu, _ = pair(w.metrics, w.bcs, w.models, w.numerics)
    st = w.state.copy()
    gpu.upload(st)
    gpu.set_correction(fz(1024, 1024))
    n = 20
    dts = (C.c_double * n)(*([w.dt] * n))
    reps = (_abi.StepReportC * n)()
    gpu.call("step_n", 0.0, dts, n, reps)
    gpu.download(st)
    area = np.outer(w.metrics.dx_c, w.metrics.dy_c)
    m0, m1 = float(np.sum(w.state.phi * area)), float(np.sum(st.phi * area))
    assert abs(m1 - m0) <= 1e-12 * m0, (m0, m1)
    # The bound is the reference's own acceptance test of a projected velocity: the
    # stage-1 check of the next step (TimeIntegrationIMEX.jl:1111-1127) rejects
    # max |div v - G| above atol + rtol * max(max|G|, 1) (5e-8 + 1e-8 here).
    num = w.numerics
    accept = num.stage1_constraint_atol + num.stage1_constraint_rtol
    for r in reps:
        assert r.maximum_projection_constraint_linf <= accept, r.maximum_projection_constraint_linf
        assert r.minimum_sigma_eigenvalue > 0.0 and r.non_spd_cells == 0
    for a in st.arrays():
        assert np.all(np.isfinite(a))
    hx = hy = 1.0 / 1024
    div = (st.U[1:, :] - st.U[:-1, :]) / hx + (st.V[:, 1:] - st.V[:, :-1]) / hy
    # the host's divergence of the returned velocity is the constraint the step reported
    # (to the rounding of the terms whose difference it is)
    scale = float(np.max(np.abs(st.U))) / hx + float(np.max(np.abs(st.V))) / hy
    assert float(np.max(np.abs(div))) <= reps[n - 1].maximum_projection_constraint_linf + 1e-12 * scale
    assert float(np.max(np.abs(div))) <= accept
