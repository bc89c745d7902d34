"""ctypes front end of the FP64 CPU oracle (oracle/liboracle_efsi.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg as the checker.  The oracle exports the same entry points as the
CUDA library with the prefix ``oracle_`` (see oracle/imex.cpp), so the package's
config builder and handle wrapper drive both.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import numpy as np

from eulerianfsi_b200 import _abi
from eulerianfsi_b200.imex import ConfigBlock, FSIState, Handle, StepReport, ProjectionResult

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_efsi.so")
_dp = C.POINTER(C.c_double)

EXTRA = {
    "structure_extension_rhs": (C.c_int32, [C.c_double, C.c_double, C.c_int32] + [_dp] * 7 + [C.c_char_p, C.c_int32]),
    "apply_structure_extension": (C.c_int32, [C.c_int32, C.c_double, C.c_int32] + [_dp] * 4),
    "relaxation_rhs": (None, [C.c_double, C.c_int32] + [_dp] * 6),
    "structure_tensor_diagnostics": (None, [C.c_int32] + [_dp] * 4),
    "body_force": (C.c_int32, [C.c_void_p, C.c_double, _dp, _dp]),
    "resource_explicit_rhs": (C.c_int32, [C.c_void_p] + [_dp] * 5),
    "constitutive_fields": (C.c_int32, [C.c_void_p] + [_dp] * 11),
    "divergence": (C.c_int32, [C.c_void_p, _dp, _dp, _dp]),
    "tensor_cell_diagnostics": (C.c_int32, [C.c_double] * 5 + [_dp]),
}

_LIB = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ only); make rebuilds it when a source
    or the ABI header is newer than the library."""
    if force and os.path.exists(LIB_PATH):
        os.remove(LIB_PATH)
    if force or not os.path.exists(LIB_PATH) or shutil.which("make"):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def load():
    global _LIB
    if _LIB is None:
        build()
        _LIB = _abi.bind(C.CDLL(LIB_PATH), "oracle_", EXTRA)
    return _LIB


def dp(a):
    return _abi.dptr(a)


class Oracle:
    """One oracle context built from a workload's configuration."""

    def __init__(self, metrics, bcs, models, numerics):
        self.block = ConfigBlock(metrics, bcs, models, numerics)
        self.metrics = metrics
        self.handle = Handle(load(), "oracle_", self.block, metrics)

    def upload(self, state: FSIState):
        self.handle.upload(state)

    def download(self, state: FSIState):
        self.handle.download(state)

    def step(self, t, dt) -> StepReport:
        r = _abi.StepReportC()
        self.handle.call("integrate_step", float(t), float(dt), C.byref(r))
        return StepReport.from_c(r)

    def make_velocity_compatible(self):
        r = _abi.ProjectionResultC()
        self.handle.call("make_velocity_compatible", C.byref(r))
        return ProjectionResult(self.handle.get_correction(), r.linear_relative_residual,
                                r.constraint_linf, r.constraint_l2, r.compatibility_defect)

    def call(self, name, *args):
        self.handle.call(name, *args)

    def stats(self):
        return self.handle.stats()
