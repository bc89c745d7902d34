"""Initial phase fields (InterfaceInitialization.jl:36-295 and the drivers' sharp
indicators).  One-time host set-up, vectorised with numpy."""
from __future__ import annotations

import numpy as np

from .errors import ArgumentError
from .mesh import MACGrid


def _periodic_displacement(coord, center, length, periodic):  # InterfaceInitialization.jl:36-44
    delta = coord - center
    return np.mod(delta + 0.5 * length, length) - 0.5 * length if periodic else delta


def profile_from_distance(distance, epsilon):  # :46-49
    return np.clip(0.5 * (1.0 - np.tanh(distance / epsilon)), 0.0, 1.0)


def _centers(grid: MACGrid):
    X = np.asarray(grid.x_p)[:, None] * np.ones((1, grid.Ny))
    Y = np.ones((grid.Nx, 1)) * np.asarray(grid.y_p)[None, :]
    return X, Y


def circle_distance(grid: MACGrid, center, radius, periodic_x=False, periodic_y=False):
    X, Y = _centers(grid)
    dx = _periodic_displacement(X, float(center[0]), grid.Lx, periodic_x)
    dy = _periodic_displacement(Y, float(center[1]), grid.Ly, periodic_y)
    return np.hypot(dx, dy) - float(radius)


def initialize_circle(grid: MACGrid, center, radius, epsilon, *, periodic_x=False, periodic_y=False):
    """initialize_circle (InterfaceInitialization.jl:74-95)."""
    if not (np.isfinite(epsilon) and epsilon > 0):
        raise ArgumentError("epsilon must be positive.")
    if not radius > 0:
        raise ArgumentError("radius must be positive.")
    d = circle_distance(grid, center, radius, periodic_x, periodic_y)
    return np.asfortranarray(profile_from_distance(d, float(epsilon)))


def initialize_circles(grid: MACGrid, centers, radius, epsilon):
    """Several disks: the phase field is the maximum of the single-disk profiles."""
    phi = np.zeros((grid.Nx, grid.Ny))
    for c in centers:
        phi = np.maximum(phi, profile_from_distance(circle_distance(grid, c, radius), float(epsilon)))
    return np.asfortranarray(phi)


def sharp_circle_indicator(grid: MACGrid, center, radius):
    """run_sugiyama_lid_driven_cavity.jl:450-457."""
    X, Y = _centers(grid)
    return np.asfortranarray((np.hypot(X - center[0], Y - center[1]) <= radius).astype(np.float64))


def sharp_wall_rectangle(grid: MACGrid, center_x, width, height, periodic_x=True):
    """Sharp indicator of a rectangle standing on the bottom wall (the wall-supported
    filament of run_wall_supported_filament_kolmogorov_flow.jl:481-500 without the cap)."""
    X, Y = _centers(grid)
    dx = _periodic_displacement(X, float(center_x), grid.Lx, periodic_x)
    inside = (np.abs(dx) <= 0.5 * width) & (Y <= height)
    return np.asfortranarray(inside.astype(np.float64))


def seeded_disk_centers(count, radius, h, seed, Lx=1.0, Ly=1.0, max_tries=200000):
    """Rejection-sampled non-overlapping disk centres: centre distance >= 2r + 4h and
    margin r + 4h from every wall; deterministic for a given seed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    margin = radius + 4.0 * h
    dmin = 2.0 * radius + 4.0 * h
    out = []
    tries = 0
    while len(out) < count:
        tries += 1
        if tries > max_tries:
            raise ArgumentError("could not place the requested disks")
        c = (rng.uniform(margin, Lx - margin), rng.uniform(margin, Ly - margin))
        if all(np.hypot(c[0] - p[0], c[1] - p[1]) >= dmin for p in out):
            out.append(c)
    return out
