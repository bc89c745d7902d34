"""Finite-difference sensitivities of the cavity-disk objective, run as replica
ensembles.

Objective: the disk's y-centroid at the final time (phase_centroid,
scripts/benchmarks/run_sugiyama_lid_driven_cavity.jl:496-509) plus 0.1 times a
neo-Hookean elastic energy of the structure tensor,

    J(p) = y_c(phi_T) + 0.1 * sum_cells phi (G/2) (tr sigma - 2 - log det sigma) dA,

with p = (shear modulus G, lid speed, initial disk centre x, y).  A central
difference with step h = rel_h * |p| along a unit direction d is
(J(p + h d) - J(p - h d)) / (2 h).  The perturbed forward runs are independent, so
the set of them is spread over the ranks of a process group (run k on rank
k mod world).  The only exchange is one all-gather of the scalar results.

Forward runs for finite differences use tight solver tolerances (1e-13) by
default.  At a looser tolerance the change of an iteration count between p + h d
and p - h d shifts J by about tolerance * |J|, which h = 1e-6 |p| turns into a
derivative error of about tolerance / 1e-6.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Callable, Sequence

import numpy as np

from . import workloads
from .errors import ArgumentError, DomainError
from .imex import FSIState, build_imex_context

PARAMETERS = ("shear_modulus", "lid_speed", "center_x", "center_y")
DEFAULT_PARAMETERS = (0.1, 1.0, 0.6, 0.5)
ENERGY_WEIGHT = 0.1
FD_RELTOL = 1e-13


def objective(state: FSIState, workload, shear_modulus: float) -> float:
    """J of a final state: y-centroid of phi plus ENERGY_WEIGHT times the elastic
    energy sum phi (G/2)(tr sigma - 2 - log det sigma) dA."""
    area = np.outer(workload.metrics.dx_c, workload.metrics.dy_c)
    phi = state.phi
    mass = float(np.sum(phi * area))
    if not mass > np.finfo(np.float64).eps:
        raise ArgumentError("Phase integral is too small to define a centroid.")
    y_p = np.asarray(workload.grid.y_p)
    y_centroid = float(np.sum(phi * area * y_p[None, :])) / mass
    det = state.sigma_xx * state.sigma_yy - state.sigma_xy ** 2
    if not np.all(det > 0.0):
        raise DomainError("structure tensor is not SPD; its elastic energy is undefined")
    density = 0.5 * shear_modulus * (state.sigma_xx + state.sigma_yy - 2.0 - np.log(det))
    return y_centroid + ENERGY_WEIGHT * float(np.sum(phi * density * area))


def objective_cotangent(state: FSIState, workload, shear_modulus: float):
    """(J, dJ/d(final state) as a dict of cell arrays, dJ/dG at fixed state) of the
    objective above: the centroid term differentiates to dA (y - y_c) / M, the energy
    term to w (G/2)(tr - 2 - log det) dA in phi and w phi (G/2)(1 - s_yy/det,
    1 - s_xx/det, 2 s_xy/det) dA in the tensor components."""
    area = np.outer(workload.metrics.dx_c, workload.metrics.dy_c)
    phi, sxx, syy, sxy = state.phi, state.sigma_xx, state.sigma_yy, state.sigma_xy
    mass = float(np.sum(phi * area))
    if not mass > np.finfo(np.float64).eps:
        raise ArgumentError("Phase integral is too small to define a centroid.")
    y_p = np.asarray(workload.grid.y_p)[None, :]
    y_centroid = float(np.sum(phi * area * y_p)) / mass
    det = sxx * syy - sxy ** 2
    if not np.all(det > 0.0):
        raise DomainError("structure tensor is not SPD; its elastic energy is undefined")
    half_g = 0.5 * shear_modulus
    density = half_g * (sxx + syy - 2.0 - np.log(det))
    energy = float(np.sum(phi * density * area))
    J = y_centroid + ENERGY_WEIGHT * energy
    w = ENERGY_WEIGHT * area
    cot = {"phi": np.asfortranarray(area * (y_p - y_centroid) / mass + w * density),
           "sigma_xx": np.asfortranarray(w * phi * half_g * (1.0 - syy / det)),
           "sigma_yy": np.asfortranarray(w * phi * half_g * (1.0 - sxx / det)),
           "sigma_xy": np.asfortranarray(w * phi * half_g * (2.0 * sxy / det))}
    dJ_dG = ENERGY_WEIGHT * energy / shear_modulus if shear_modulus != 0.0 else 0.0
    return J, cot, dJ_dG


def circle_center_derivative(grid, center, radius, epsilon):
    """d(phi_0)/d(center x) and /d(center y) of initialize_circle's tanh profile
    phi_0 = (1 - tanh((|x - c| - r) / eps)) / 2."""
    X = np.asarray(grid.x_p)[:, None] * np.ones((1, grid.Ny))
    Y = np.ones((grid.Nx, 1)) * np.asarray(grid.y_p)[None, :]
    dx, dy = X - center[0], Y - center[1]
    rho = np.hypot(dx, dy)
    t = np.tanh((rho - radius) / epsilon)
    g = np.where(rho > 0.0, 0.5 * (1.0 - t * t) / (epsilon * np.where(rho > 0.0, rho, 1.0)), 0.0)
    return g * dx, g * dy


def adjoint_gradient(N: int = 256, T: float = 2.0, p=DEFAULT_PARAMETERS, reltol: float = FD_RELTOL,
                     every: int = 0, timings: dict | None = None) -> dict:
    """J and dJ/dp for p = (G, lid speed, centre x, y) from one checkpointed forward run
    and one reverse sweep of the discrete adjoint.  `timings` receives the device
    milliseconds of the forward run and of the reverse sweep (which includes its
    recomputation of every checkpoint segment)."""
    from . import adjoint
    G, lid, cx, cy = (float(v) for v in p)
    w = workloads.cavity_disk_sensitivity(N, tuple(p), T, projection_reltol=reltol, velocity_reltol=reltol)
    ctx = build_imex_context(w.metrics, w.bcs, w.models, numerics=w.numerics)
    state = w.state.copy()
    adjoint.forward_checkpointed(state, 0.0, np.full(w.steps, w.dt), ctx, every)
    forward_ms = ctx.handle.stats()["device_ms"]
    J, cot, dJdG_direct = objective_cotangent(state, w, G)
    grad_state, pg = adjoint.backward(ctx, cot)
    backward_ms = ctx.handle.stats()["device_ms"]
    ctx.handle.close()
    h = 1.0 / N
    dcx, dcy = circle_center_derivative(w.grid, (cx, cy), 0.2, 1.5 * h)
    # the lid speed is the (uniform) U-top wall datum: every entry moves with it
    gradient = [pg.elastic_coefficient + dJdG_direct, float(np.sum(pg.U_top)),
                float(np.sum(grad_state.phi * dcx)), float(np.sum(grad_state.phi * dcy))]
    if timings is not None:
        timings.update(forward_ms=forward_ms, backward_ms=backward_ms)
    return {"J": J, "gradient": gradient, "steps": w.steps, "forward_ms": forward_ms, "backward_ms": backward_ms}


def cuda_final_state(w, timings: list | None = None) -> FSIState:
    """Run workload `w` for w.steps device-resident steps on the CUDA library and
    return the final state; the run's device milliseconds are appended to
    `timings` when given."""
    ctx = build_imex_context(w.metrics, w.bcs, w.models, numerics=w.numerics)
    h = ctx.handle
    state = w.state.copy()
    h.upload(state)
    h.set_correction(np.zeros((w.metrics.Nx, w.metrics.Ny), order="F"))
    dts = (C.c_double * w.steps)(*([w.dt] * w.steps))
    h.call("step_n", 0.0, dts, int(w.steps), None)
    if timings is not None:
        timings.append(h.stats()["device_ms"])
    h.download(state)
    h.close()
    return state


def make_evaluator(N: int = 256, T: float = 2.0, run: Callable | None = None, reltol: float = FD_RELTOL,
                   precision: str = "fp64", timings: list | None = None) -> Callable[[Sequence[float]], float]:
    """J as a function of p for the cavity_disk_sensitivity workload of size N to
    time T; `run(workload) -> final FSIState` defaults to the CUDA library (whose
    device milliseconds per run go to `timings`)."""
    run = run or (lambda w: cuda_final_state(w, timings))

    def evaluate(p):
        w = workloads.cavity_disk_sensitivity(N, tuple(p), T, projection_reltol=reltol, velocity_reltol=reltol,
                                              precision=precision)
        return objective(run(w), w, float(p[0]))

    return evaluate


def seeded_direction(seed: int, n: int = len(PARAMETERS)) -> np.ndarray:
    """Unit direction drawn from a seeded normal distribution."""
    d = np.random.default_rng(seed).standard_normal(n)
    return d / np.linalg.norm(d)


def difference_points(p, directions, rel_h: float):
    """[p, p + h d_0, p - h d_0, p + h d_1, ...] and h = rel_h * |p|."""
    p = np.asarray(p, dtype=np.float64)
    h = rel_h * float(np.linalg.norm(p))
    if not h > 0.0:
        raise ArgumentError("the finite-difference step must be positive")
    points = [p.copy()]
    for d in np.atleast_2d(np.asarray(directions, dtype=np.float64)):
        points += [p + h * d, p - h * d]
    return points, h


def _world(group):
    if group is None:
        return 1, 0
    import torch.distributed as dist
    return dist.get_world_size(group), dist.get_rank(group)


def ensemble(evaluate, points, group=None) -> np.ndarray:
    """J at every point.  Point k runs on rank k mod world; the results meet in one
    all-gather, so every rank returns the full vector."""
    world, rank = _world(group)
    vals = np.zeros(len(points))
    for k in range(rank, len(points), world):
        vals[k] = evaluate(points[k])
    if world == 1:
        return vals
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    mine = torch.tensor(vals, dtype=torch.float64, device=device)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = np.zeros(len(points))
    for k in range(len(points)):
        out[k] = float(parts[k % world][k].item())
    return out


def central_differences(evaluate, p, directions, rel_h: float = 1e-6, group=None):
    """(J(p), [D_d J(p) for each direction d]) by central differences, the runs
    spread over `group`."""
    points, h = difference_points(p, directions, rel_h)
    vals = ensemble(evaluate, points, group)
    n = (len(points) - 1) // 2
    derivs = np.array([(vals[1 + 2 * k] - vals[2 + 2 * k]) / (2.0 * h) for k in range(n)])
    return float(vals[0]), derivs


def gradient_check(evaluate, p=DEFAULT_PARAMETERS, seed: int = 0, rel_h: float = 1e-6, group=None) -> dict:
    """Finite-difference gradient (one central difference per parameter) and the
    directional derivative along a seeded unit direction, from one ensemble of
    2 * (len(p) + 1) + 1 forward runs.  `rel_diff` compares the directional
    derivative with gradient . direction."""
    n = len(p)
    d = seeded_direction(seed, n)
    dirs = np.vstack([np.eye(n), d[None, :]])
    J, D = central_differences(evaluate, p, dirs, rel_h, group)
    grad = D[:n]
    directional = float(D[n])
    dot = float(grad @ d)
    return {"J": J, "gradient": grad.tolist(), "direction": d.tolist(), "directional": directional,
            "gradient_dot_direction": dot,
            "rel_diff": abs(directional - dot) / max(abs(directional), math.ulp(1.0)),
            "runs": 2 * (n + 1) + 1, "h": rel_h * float(np.linalg.norm(p))}
