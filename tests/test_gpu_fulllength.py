"""Full-length runs of the benchmark configurations against the FP64 oracle.

* C1, the filament in Kolmogorov flow (256 x 256, 1000 steps): both precision forms
  against the oracle's final state (tests/golden/filament_N256_s1000.npz, made by
  tests/golden/make_fulllength.py), every solve converged to 1e-13 on both sides:
  1e-8 relative L2 per field for the FP64 step, 1e-6 for the precision form.
* C2, the 20-disk cavity (1024 x 1024, 500 steps) and C3, the growth channel
  (1024 x 512, 300 steps), at their benchmark tolerances: the precision form against
  the FP64 step after the full run (1e-6 per field), and a segment of steps from the
  FP64 run's final state on the GPU and on the oracle (solves converged to 1e-13 on
  both sides, 1e-10 per field), which pins the step at the end of the trajectory.
"""
import ctypes as C
import dataclasses
import os

import numpy as np
import pytest

from eulerianfsi_b200 import _abi, workloads
from tests.gpu_util import pair, rel_err
from tests.helpers import fz

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("U", "V", "phi", "resource", "sigma_xx", "sigma_yy", "sigma_xy")


def _tight(numerics, precision=None):
    ls = dataclasses.replace(numerics.linear_solvers, velocity_method="gmres", reltol=1e-13, maxiter=2000)
    kw = {} if precision is None else {"precision": precision}
    return dataclasses.replace(numerics, linear_solvers=ls, projection_reltol=1e-13, projection_maxiter=3000, **kw)


def _run_gpu(w, numerics, steps, compatible=False):
    gpu, _ = pair(w.metrics, w.bcs, w.models, numerics)
    st = w.state.copy()
    gpu.upload(st)
    gpu.set_correction(fz(w.metrics.Nx, w.metrics.Ny))
    if compatible:
        gpu.call("make_velocity_compatible", C.byref(_abi.ProjectionResultC()))
        gpu.set_correction(fz(w.metrics.Nx, w.metrics.Ny))
    dts = (C.c_double * steps)(*([w.dt] * steps))
    gpu.call("step_n", 0.0, dts, steps, None)
    gpu.download(st)
    return st, gpu.get_correction()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 1e-6)])
def test_config1_full_length_against_oracle(precision, tol):
    ref = np.load(os.path.join(HERE, "golden", "filament_N256_s1000.npz"))
    w = workloads.filament_kolmogorov(N=256, steps=1000)
    assert int(ref["steps"]) == w.steps and float(ref["dt"]) == w.dt
    st, _ = _run_gpu(w, _tight(w.numerics, precision), w.steps)
    errs = {f: rel_err(getattr(st, f), ref[f]) for f in FIELDS}
    print(f"C1 {precision} vs oracle after {w.steps} steps:", {f: f"{e:.2e}" for f, e in errs.items()})
    for f, e in errs.items():
        assert e <= tol, (f, e)


def _segment_against_oracle(w, start, q, steps, t0):
    """`steps` steps from state `start` (correction q) on the GPU and on the oracle,
    solves converged to 1e-13 on both sides."""
    gpu, ora = pair(w.metrics, w.bcs, w.models, _tight(w.numerics, "fp64"))
    out = []
    for h in (gpu, ora):
        st = start.copy()
        h.upload(st)
        h.set_correction(q)
        for k in range(steps):
            rep = _abi.StepReportC()
            h.call("integrate_step", t0 + k * w.dt, w.dt, C.byref(rep))
        h.download(st)
        out.append(st)
    return out


@pytest.mark.parametrize("config", ["C2", "C3"])
def test_precision_forms_full_length_and_final_segment(config):
    if config == "C2":
        make = lambda p: workloads.cavity_disks20(N=1024, precision=p)
        compatible, seg = False, 2
    else:
        make = lambda p: workloads.channel_growth(N=512, precision=p)
        compatible, seg = True, 2
    w64, wmx = make("fp64"), make("mixed")
    a, q = _run_gpu(w64, w64.numerics, w64.steps, compatible)
    b, _ = _run_gpu(wmx, wmx.numerics, wmx.steps, compatible)
    errs = {f: rel_err(getattr(b, f), getattr(a, f)) for f in FIELDS}
    print(f"{config} precision form vs FP64 after {w64.steps} steps:", {f: f"{e:.2e}" for f, e in errs.items()})
    for f, e in errs.items():
        assert e <= 1e-6, (config, f, e)
    g, o = _segment_against_oracle(w64, a, q, seg, w64.steps * w64.dt)
    errs = {f: rel_err(getattr(g, f), getattr(o, f)) for f in FIELDS}
    print(f"{config} FP64 vs oracle, {seg} steps from step {w64.steps}:", {f: f"{e:.2e}" for f, e in errs.items()})
    for f, e in errs.items():
        assert e <= 1e-10, (config, f, e)
