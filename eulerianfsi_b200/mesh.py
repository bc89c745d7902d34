"""MAC grid and mesh metrics, mirroring EulerianFSI.jl's MeshGeneration module
(MeshGeneration.jl:17-372).  Arrays use 0-based indices; values are computed with
the same floating-point expressions as the reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .errors import ArgumentError, DimensionMismatch

SUPPORTED_STRETCHING_METHODS = (
    "uniform", "tanh_edges", "sinh_center", "chebyshev_edges", "drop_centered",
    "boundary_layer_bottom")


@dataclass
class MACGrid:
    """MACGrid (MeshGeneration.jl:17-39)."""
    Lx: float
    Ly: float
    Nx: int
    Ny: int
    dx_nominal: float
    dy_nominal: float
    x_p: np.ndarray
    y_p: np.ndarray
    x_u: np.ndarray
    y_u: np.ndarray
    x_v: np.ndarray
    y_v: np.ndarray


@dataclass
class MeshMetrics:
    """MeshMetrics (MeshGeneration.jl:41-73)."""
    dx_f: np.ndarray
    dx_c: np.ndarray
    dy_f: np.ndarray
    dy_c: np.ndarray
    wL_c2fx: np.ndarray
    wR_c2fx: np.ndarray
    wB_c2fy: np.ndarray
    wT_c2fy: np.ndarray
    wL_f2cx: np.ndarray
    wR_f2cx: np.ndarray
    wB_f2cy: np.ndarray
    wT_f2cy: np.ndarray
    dx_west_corner: np.ndarray
    dx_east_corner: np.ndarray
    dy_south_corner: np.ndarray
    dy_north_corner: np.ndarray
    periodic_x: bool
    periodic_y: bool
    Nx: int
    Ny: int
    Lx: float
    Ly: float


def _stretch_parameter(method: str, gamma):  # MeshGeneration.jl:85-105
    if method not in SUPPORTED_STRETCHING_METHODS:
        raise ArgumentError(f"Unsupported stretching method: {method}.")
    if method in ("uniform", "chebyshev_edges"):
        return 0.0
    value = (0.5 if method == "drop_centered" else 2.0) if gamma is None else float(gamma)
    if method == "drop_centered":
        if not (0.0 <= value < 1.0):
            raise ArgumentError("For :drop_centered, the stretching parameter must satisfy 0 <= gamma < 1.")
    elif not value > 0.0:
        raise ArgumentError(f"For {method}, the stretching parameter gamma must be positive.")
    return value


def map_coordinate(xi: float, L: float, method: str, gamma: float) -> float:
    """MeshGeneration.jl:108-132."""
    if not (0.0 <= xi <= 1.0):
        raise ArgumentError("Logical coordinate xi must lie in [0,1].")
    if method == "uniform":
        return L * xi
    if method == "tanh_edges":
        return L * 0.5 * (1.0 + math.tanh(gamma * (xi - 0.5)) / math.tanh(gamma / 2.0))
    if method == "sinh_center":
        return L * 0.5 * (1.0 + math.sinh(gamma * (xi - 0.5)) / math.sinh(gamma / 2.0))
    if method == "chebyshev_edges":
        return L * 0.5 * (1.0 - math.cos(math.pi * xi))
    if method == "drop_centered":
        return L * (0.5 + (1.0 - gamma) * (xi - 0.5) + gamma * 16.0 * (xi - 0.5) ** 5)
    if method == "boundary_layer_bottom":
        return L * (1.0 - math.tanh(gamma * (1.0 - xi)) / math.tanh(gamma))
    raise ArgumentError(f"Unsupported stretching method: {method}")


def generate_grid(Lx, Ly, Nx, Ny, *, stretch_x="uniform", stretch_y="uniform", gamma_x=None,
                  gamma_y=None) -> MACGrid:
    """generate_grid (MeshGeneration.jl:179-233)."""
    Lx, Ly, Nx, Ny = float(Lx), float(Ly), int(Nx), int(Ny)
    if not Lx > 0.0:
        raise ArgumentError("Lx must be positive.")
    if not Ly > 0.0:
        raise ArgumentError("Ly must be positive.")
    if Nx < 2:
        raise ArgumentError("Nx must be at least 2.")
    if Ny < 2:
        raise ArgumentError("Ny must be at least 2.")
    gx = _stretch_parameter(stretch_x, gamma_x)
    gy = _stretch_parameter(stretch_y, gamma_y)
    x_u = np.array([map_coordinate((i - 1.0) / Nx, Lx, stretch_x, gx) for i in range(1, Nx + 2)])
    y_v = np.array([map_coordinate((j - 1.0) / Ny, Ly, stretch_y, gy) for j in range(1, Ny + 2)])
    x_u[0], x_u[-1], y_v[0], y_v[-1] = 0.0, Lx, 0.0, Ly
    x_p = np.array([map_coordinate((i - 0.5) / Nx, Lx, stretch_x, gx) for i in range(1, Nx + 1)])
    y_p = np.array([map_coordinate((j - 0.5) / Ny, Ly, stretch_y, gy) for j in range(1, Ny + 1)])
    for arr, name in ((x_p, "Cell-center x"), (y_p, "Cell-center y"), (x_u, "x-face"), (y_v, "y-face")):
        if not np.all(np.diff(arr) > 0.0):
            raise ArgumentError(f"{name}-coordinates must be strictly increasing.")
    if not (np.all(x_u[:-1] < x_p) and np.all(x_p < x_u[1:])):
        raise ArgumentError("Each x cell center must lie strictly between its adjacent x-faces.")
    if not (np.all(y_v[:-1] < y_p) and np.all(y_p < y_v[1:])):
        raise ArgumentError("Each y cell center must lie strictly between its adjacent y-faces.")
    return MACGrid(Lx, Ly, Nx, Ny, Lx / Nx, Ly / Ny, x_p, y_p, x_u, y_p.copy(), x_p.copy(), y_v)


def _axis_metrics(centers, faces, L, periodic):  # MeshGeneration.jl:237-335
    N = len(centers)
    if len(faces) != N + 1:
        raise DimensionMismatch("A staggered axis with N cell centers must contain N+1 faces.")
    h_c = np.diff(faces)
    h_f = np.empty(N + 1)
    wrapped = centers[0] + L - centers[-1]
    h_f[0] = wrapped if periodic else 2.0 * (centers[0] - faces[0])
    for i in range(1, N):
        h_f[i] = centers[i] - centers[i - 1]
    h_f[N] = wrapped if periodic else 2.0 * (faces[N] - centers[N - 1])
    wm, wp = np.empty(N + 1), np.empty(N + 1)
    if periodic:
        dm = faces[0] + L - centers[-1]
        dp = centers[0] - faces[0]
        wm[0], wp[0] = dp / (dm + dp), dm / (dm + dp)
    else:
        wm[0], wp[0] = 0.0, 1.0
    for i in range(1, N):
        dm = faces[i] - centers[i - 1]
        dp = centers[i] - faces[i]
        wm[i], wp[i] = dp / (dm + dp), dm / (dm + dp)
    if periodic:
        dm = faces[N] - centers[N - 1]
        dp = centers[0] + L - faces[N]
        wm[N], wp[N] = dp / (dm + dp), dm / (dm + dp)
    else:
        wm[N], wp[N] = 1.0, 0.0
    fm, fp = np.empty(N), np.empty(N)
    for i in range(N):
        dm = centers[i] - faces[i]
        dp = faces[i + 1] - centers[i]
        fm[i], fp[i] = dp / (dm + dp), dm / (dm + dp)
    cm, cp = np.empty(N + 1), np.empty(N + 1)
    cp[0] = centers[0] - faces[0]
    cm[0] = faces[0] + L - centers[-1] if periodic else cp[0]
    for i in range(1, N):
        cm[i] = faces[i] - centers[i - 1]
        cp[i] = centers[i] - faces[i]
    cm[N] = faces[N] - centers[N - 1]
    cp[N] = centers[0] + L - faces[N] if periodic else cm[N]
    if not np.all(h_c > 0.0):
        raise ArgumentError("All cell widths must be positive.")
    if not np.all(h_f > 0.0):
        raise ArgumentError("All center-to-center distances must be positive.")
    return h_f, h_c, wm, wp, fm, fp, cm, cp


def build_mesh_metrics(grid: MACGrid, *, periodic_x: bool = False, periodic_y: bool = False) -> MeshMetrics:
    """build_mesh_metrics (MeshGeneration.jl:340-372)."""
    xf, xc, xwm, xwp, xfm, xfp, xcm, xcp = _axis_metrics(grid.x_p, grid.x_u, grid.Lx, periodic_x)
    yf, yc, ywm, ywp, yfm, yfp, ycm, ycp = _axis_metrics(grid.y_p, grid.y_v, grid.Ly, periodic_y)
    return MeshMetrics(xf, xc, yf, yc, xwm, xwp, ywm, ywp, xfm, xfp, yfm, yfp, xcm, xcp, ycm, ycp,
                       bool(periodic_x), bool(periodic_y), grid.Nx, grid.Ny, grid.Lx, grid.Ly)


def is_uniform(metrics: MeshMetrics, rtol: float = 1e-12) -> bool:
    """True when every cell has the same width in x and in y (the device step's requirement)."""
    hx = metrics.Lx / metrics.Nx
    hy = metrics.Ly / metrics.Ny
    return bool(np.all(np.abs(metrics.dx_c - hx) <= rtol * hx) and
                np.all(np.abs(metrics.dy_c - hy) <= rtol * hy))
