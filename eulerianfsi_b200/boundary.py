"""Boundary-condition types mirroring BoundaryConditions.jl:23-136, and their
flattening into the C-ABI's per-side value arrays."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any

import numpy as np

from . import _abi
from .errors import ArgumentError, DimensionMismatch


class AbstractBoundaryCondition:
    pass


@dataclass(frozen=True)
class Periodic(AbstractBoundaryCondition):
    pass


@dataclass(frozen=True)
class Dirichlet(AbstractBoundaryCondition):
    value: Any = 0.0


@dataclass(frozen=True)
class Neumann(AbstractBoundaryCondition):
    value: Any = 0.0


@dataclass(frozen=True)
class MixedBoundary(AbstractBoundaryCondition):
    dirichlet_mask: Any
    dirichlet_value: Any
    neumann_value: Any


@dataclass(frozen=True)
class AdvectiveOutflow(AbstractBoundaryCondition):
    backflow_value: Any = 0.0


class BoundaryConditionSetup:
    """Four-sided container (BoundaryConditions.jl:51-83)."""

    def __init__(self, left, right, bottom, top):
        for side in (left, right, bottom, top):
            if not isinstance(side, AbstractBoundaryCondition):
                raise ArgumentError("boundary sides must be boundary-condition objects")
        if isinstance(left, Periodic) != isinstance(right, Periodic):
            raise ArgumentError("Periodic boundaries in the x-direction must be specified as an opposing pair.")
        if isinstance(bottom, Periodic) != isinstance(top, Periodic):
            raise ArgumentError("Periodic boundaries in the y-direction must be specified as an opposing pair.")
        self.left, self.right, self.bottom, self.top = left, right, bottom, top

    def sides(self):
        return (self.left, self.right, self.bottom, self.top)

    def __repr__(self):
        return f"BoundaryConditionSetup({self.left!r}, {self.right!r}, {self.bottom!r}, {self.top!r})"


def is_periodic_x(bc: BoundaryConditionSetup) -> bool:
    return isinstance(bc.left, Periodic)


def is_periodic_y(bc: BoundaryConditionSetup) -> bool:
    return isinstance(bc.bottom, Periodic)


def has_dirichlet(bc: BoundaryConditionSetup) -> bool:
    """BoundaryConditions.jl:92-98."""
    for s in bc.sides():
        if isinstance(s, Dirichlet):
            return True
        if isinstance(s, MixedBoundary) and any(bool(v) for v in np.asarray(s.dirichlet_mask).ravel()):
            return True
    return False


def evaluate_boundary_data(value, n: int) -> np.ndarray:
    """Flatten Julia-style boundary data (number, vector or callable of the 1-based
    boundary index, BoundaryConditions.jl:124-136) into n float64 values."""
    if value is None:
        return np.zeros(n)
    if np.isscalar(value):
        return np.full(n, float(value))
    if callable(value):
        return np.array([float(value(k)) for k in range(1, n + 1)])
    arr = np.asarray(value, dtype=np.float64).ravel()
    if arr.size < n:
        raise DimensionMismatch(f"boundary data has {arr.size} entries; the side needs {n}")
    return np.ascontiguousarray(arr[:n])


_KIND = {Periodic: _abi.BC_PERIODIC, Dirichlet: _abi.BC_DIRICHLET, Neumann: _abi.BC_NEUMANN,
         MixedBoundary: _abi.BC_MIXED, AdvectiveOutflow: _abi.BC_ADVECTIVE_OUTFLOW}


def fill_setup(dst: _abi.BCSetup, bc: BoundaryConditionSetup, n_lr: int, n_bt: int, keep: list) -> None:
    """Write one BoundaryConditionSetup into the C struct; arrays are kept alive in `keep`."""
    for name, side, n in (("left", bc.left, n_lr), ("right", bc.right, n_lr),
                          ("bottom", bc.bottom, n_bt), ("top", bc.top, n_bt)):
        out = getattr(dst, name)
        out.type = _KIND[type(side)]
        out.n = n
        if isinstance(side, Periodic):
            out.n = 0
            continue
        if isinstance(side, MixedBoundary):
            val = evaluate_boundary_data(side.dirichlet_value, n)
            neu = evaluate_boundary_data(side.neumann_value, n)
            mask = np.ascontiguousarray(np.asarray(side.dirichlet_mask, dtype=np.uint8).ravel())
            if mask.size < n:
                raise DimensionMismatch("MixedBoundary mask shorter than the side")
            keep += [val, neu, mask]
            out.value = _abi.dptr(val)
            out.neumann = _abi.dptr(neu)
            out.mask = mask.ctypes.data_as(C.POINTER(C.c_uint8))
        else:
            raw = side.backflow_value if isinstance(side, AdvectiveOutflow) else side.value
            val = evaluate_boundary_data(raw, n)
            keep.append(val)
            out.value = _abi.dptr(val)
