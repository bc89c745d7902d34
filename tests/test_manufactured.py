"""Manufactured solutions with exact discrete answers, on the oracle (CPU) and through
the CUDA library (GPU).  They pin both implementations against closed forms, not
against each other:

* the viscous operator (`Operators.jl:929-1083`) on quadratic velocity fields: second
  differences and the mixed difference of quadratics are exact, so every row away from
  the boundary equals 2 mu u_xx + mu u_yy + mu v_xy and mu v_xx + 2 mu v_yy + mu u_xy;
* the projection (`Projection.jl:170-307`) of a discrete gradient plus a discrete
  curl: the MAC divergence of a discrete gradient is the discrete Laplacian and that
  of a curl (a stream function at the nodes) vanishes identically, so the projection
  returns the curl and the potential (zero mean).  Periodic and walled (Neumann
  correction) boxes.  (A pure curl alone has a right-hand side of rounding noise, and
  the reference's true-residual test, relative to |b|, rejects it: Projection.jl:261-284.)
"""
import ctypes as C

import numpy as np
import pytest

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import _abi, workloads
from eulerianfsi_b200.imex import ConfigBlock, Handle
from oracle.oracle import load as load_oracle
from tests.helpers import dp, fz, periodic_problem

MU = 0.01


def _handle(kind, metrics, bcs, models, numerics):
    if kind == "oracle":
        return Handle(load_oracle(), "oracle_", ConfigBlock(metrics, bcs, models, numerics), metrics)
    return Handle(_abi.load_library(), "efsi_", ConfigBlock(metrics, bcs, models, numerics), metrics)


def _quadratic_velocity(N):
    h = 1.0 / N
    xf, xc = np.arange(N) * h, (np.arange(N) + 0.5) * h
    X, Y = np.meshgrid(xf, xc, indexing="ij")
    U = X ** 2 + 2 * X * Y + 3 * Y ** 2          # u_xx = 2, u_yy = 6, u_xy = 2
    X, Y = np.meshgrid(xc, xf, indexing="ij")
    V = 2 * X ** 2 - X * Y + Y ** 2              # v_xx = 4, v_yy = 2, v_xy = -1
    return U, V, 2 * MU * 2 + MU * 6 + MU * (-1), MU * 4 + 2 * MU * 2 + MU * 2


def _check_viscous(kind, periodic):
    N = 32
    if periodic:
        grid, metrics, bcs, models = periodic_problem(N, None, viscosity=ef.ConstantViscosity(MU))
        numerics = ef.IMEXNumerics()
    else:
        w = workloads.cavity_disk(N=N)
        metrics, bcs, numerics = w.metrics, w.bcs, w.numerics
        models = ef.FSIModels(viscosity=ef.ConstantViscosity(MU))
    h = _handle(kind, metrics, bcs, models, numerics)
    U, V, au_exact, av_exact = _quadratic_velocity(N)
    uv = np.concatenate([U.ravel(order="F"), V.ravel(order="F")])
    out = np.zeros(2 * N * N)
    h.call("apply_viscous_operator", dp(fz(N, N)), dp(uv), dp(out))
    au = out[:N * N].reshape((N, N), order="F")[2:-2, 2:-2]
    av = out[N * N:].reshape((N, N), order="F")[2:-2, 2:-2]
    assert np.abs(au - au_exact).max() <= 1e-9 * abs(au_exact), np.abs(au - au_exact).max()
    assert np.abs(av - av_exact).max() <= 1e-9 * abs(av_exact), np.abs(av - av_exact).max()


def _box(periodic, N):
    if periodic:
        grid, metrics, bcs, models = periodic_problem(N, None)
        return metrics, bcs, models
    w = workloads.cavity_disk(N=N)
    return w.metrics, w.bcs, ef.FSIModels()


def _gradient_field(N, periodic):
    """(U, V, phi): the MAC gradient of a smooth cell field, normal wall faces zero."""
    h = 1.0 / N
    xc = (np.arange(N) + 0.5) * h
    X, Y = np.meshgrid(xc, xc, indexing="ij")
    if periodic:
        phi = np.cos(2 * np.pi * X) * np.sin(4 * np.pi * Y) + 0.3 * np.sin(2 * np.pi * (X + Y))
    else:
        phi = np.cos(np.pi * X) * np.cos(2 * np.pi * Y) + 0.5 * X * Y
    U, V = np.zeros((N + 1, N), order="F"), np.zeros((N, N + 1), order="F")
    if periodic:
        U[:N, :] = (phi - np.roll(phi, 1, axis=0)) / h
        U[N, :] = U[0, :]
        V[:, :N] = (phi - np.roll(phi, 1, axis=1)) / h
        V[:, N] = V[:, 0]
    else:
        U[1:N, :] = (phi[1:, :] - phi[:-1, :]) / h
        V[:, 1:N] = (phi[:, 1:] - phi[:, :-1]) / h
    return U, V, phi


def _curl_field(N, periodic):
    """(U, V): the MAC curl of a stream function at the nodes (zero on walls)."""
    h = 1.0 / N
    xn = np.arange(N + 1) * h
    X, Y = np.meshgrid(xn, xn, indexing="ij")
    if periodic:
        psi = np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) + 0.2 * np.cos(4 * np.pi * X)
    else:
        psi = np.sin(np.pi * X) ** 2 * np.sin(np.pi * Y) ** 2 * (1 + X)
    U = np.asfortranarray((psi[:, 1:] - psi[:, :-1]) / h)   # (N+1) x N
    V = np.asfortranarray(-(psi[1:, :] - psi[:-1, :]) / h)  # N x (N+1)
    return U, V


def _project(h, U, V, N):
    U, V = U.copy(order="F"), V.copy(order="F")
    h.set_correction(fz(N, N))
    r = _abi.ProjectionResultC()
    h.call("project", dp(U), dp(V), dp(fz(N, N)), C.byref(r))
    return U, V, h.get_correction()


def _check_projection(kind, periodic, N, solver="auto"):
    metrics, bcs, models = _box(periodic, N)
    h = _handle(kind, metrics, bcs, models, ef.IMEXNumerics(projection_reltol=1e-13, projection_solver=solver))
    Ug, Vg, phi = _gradient_field(N, periodic)
    Uc, Vc = _curl_field(N, periodic)
    scale = max(np.abs(Ug).max(), np.abs(Vg).max(), np.abs(Uc).max(), np.abs(Vc).max())
    Up, Vp, q = _project(h, Ug + Uc, Vg + Vc, N)
    assert max(np.abs(Up - Uc).max(), np.abs(Vp - Vc).max()) <= 1e-11 * scale
    assert np.abs(q - (phi - phi.mean())).max() <= 1e-11 * np.abs(phi).max()


@pytest.mark.parametrize("periodic", [False, True])
def test_oracle_viscous_operator_on_quadratics(periodic):
    _check_viscous("oracle", periodic)


@pytest.mark.parametrize("periodic", [False, True])
def test_oracle_projection_of_gradient_and_curl(periodic):
    _check_projection("oracle", periodic, 32)


@pytest.mark.gpu
@pytest.mark.parametrize("periodic", [False, True])
def test_gpu_viscous_operator_on_quadratics(periodic):
    _check_viscous("gpu", periodic)


@pytest.mark.gpu
@pytest.mark.parametrize("N,solver", [(64, "auto"), (64, "multigrid"), (48, "auto")])
@pytest.mark.parametrize("periodic", [False, True])
def test_gpu_projection_of_gradient_and_curl(periodic, N, solver):
    """Direct solve (64, auto), multigrid CG (64 forced, and 48, which the direct solve
    does not take)."""
    _check_projection("gpu", periodic, N, solver)
