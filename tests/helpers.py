"""Shared builders for the tests (small periodic / walled problems)."""
import ctypes as C

import numpy as np

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import _abi


def dp(a):
    return _abi.dptr(a)


def periodic_problem(N, model, Lx=1.0, Ly=1.0, **model_kw):
    grid = ef.generate_grid(Lx, Ly, N, N)
    metrics = ef.build_mesh_metrics(grid, periodic_x=True, periodic_y=True)
    p = ef.Periodic()
    bc = ef.BoundaryConditionSetup(p, p, p, p)
    bcs = ef.FSIBoundaryConditions(bc, bc, bc, bc, {"xx": bc, "yy": bc, "xy": bc})
    models = ef.FSIModels(phase_field_method=model, **model_kw) if model is not None else ef.FSIModels(**model_kw)
    return grid, metrics, bcs, models


def fz(*shape):
    return np.zeros(shape, order="F")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    return num / den if den > 0 else num
