"""Edge cases of the CUDA path against the FP64 CPU oracle: periodic grids smaller
than one kernel tile, anisotropic spacing (hx != hy) on a grid that is not a power
of two, MixedBoundary sides, and the configurations the device step rejects."""
import dataclasses

import numpy as np
import pytest

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import workloads
from tests.gpu_util import pair, random_inputs, rel_err
from tests.helpers import dp, fz, periodic_problem
from tests.test_gpu_parity import OP_TOL, PF, STEP_TOL, _assert_states, _run_steps

pytestmark = pytest.mark.gpu


def _periodic_inputs(metrics, seed):
    inp = random_inputs(metrics, seed=seed)
    inp["U"][-1, :] = inp["U"][0, :]
    inp["V"][:, -1] = inp["V"][:, 0]
    return inp


@pytest.mark.parametrize("N", [5, 8])
@pytest.mark.parametrize("name", list(PF))
def test_phase_field_rhs_tiny_periodic(N, name):
    """Grids narrower than the 32x8 tile plus its 3-cell halo: the staged halo
    wraps around the period several times."""
    grid, metrics, bcs, models = periodic_problem(N, PF[name])
    gpu, ora = pair(metrics, bcs, models, ef.IMEXNumerics())
    inp = _periodic_inputs(metrics, 17)
    outs = []
    for h in (gpu, ora):
        r = fz(N, N)
        h.call("phase_field_rhs", dp(inp["U"]), dp(inp["V"]), dp(inp["phi"]), dp(inp["G"]), dp(r))
        outs.append(r)
    assert rel_err(outs[0], outs[1]) <= OP_TOL, rel_err(outs[0], outs[1])


@pytest.mark.parametrize("normals", ["standard", "youngs", "smoothed9"])
def test_uwcdi_strang_step_tiny_periodic(normals):
    method = ef.PirozzoliUWCDIPhaseField(1.0, normal_reconstruction=normals)
    grid, metrics, bcs, models = periodic_problem(6, method)
    gpu, ora = pair(metrics, bcs, models, ef.IMEXNumerics())
    inp = _periodic_inputs(metrics, 19)
    outs = []
    for h in (gpu, ora):
        out = fz(6, 6)
        h.call("uwcdi_strang_step", dp(inp["U"]), dp(inp["V"]), dp(inp["phi"]), 0.002, 1, dp(out))
        outs.append(out)
    assert rel_err(outs[0], outs[1]) <= OP_TOL


def _tiny_periodic_workload(N):
    method = ef.PirozzoliUWCDIPhaseField(1.0, delta_normal=1e-14)
    grid, metrics, bcs, models = periodic_problem(N, method, viscosity=ef.ConstantViscosity(0.05),
                                                  elastic_stress=ef.LinearInternalTensorStress(0.2),
                                                  body_force=ef.KolmogorovBodyForce(0.5, 2.0 * np.pi))
    phi = workloads.initialize_circle(grid, (0.5, 0.5), 0.3, 1.5 / N)
    state = workloads._rest_state(N, N, phi)
    numerics = workloads._numerics(1e-13, 1e-13, "fp64", extension=False)
    return workloads.Workload("tiny_periodic", grid, metrics, bcs, models, numerics, state, 0.2 / N, 3)


@pytest.mark.parametrize("N", [6, 8])
def test_tiny_periodic_steps(N):
    w = _tiny_periodic_workload(N)
    (g, o), _, _ = _run_steps(w, 3)
    _assert_states(g, o, STEP_TOL * 10)


def _anisotropic_cavity(Nx=48, Ny=40):
    grid = ef.generate_grid(1.0, 1.0, Nx, Ny)
    metrics = ef.build_mesh_metrics(grid)
    h = 1.0 / Nx
    phi = workloads.initialize_circle(grid, (0.55, 0.45), 0.22, 1.5 / Ny)
    return workloads.Workload("cavity_disk_48x40", grid, metrics, workloads._cavity_bcs(),
                              workloads._cavity_models(h), workloads._numerics(1e-13, 1e-13, "fp64"),
                              workloads._rest_state(Nx, Ny, phi), 0.2 * h, 4)


def test_anisotropic_rectangular_cavity_steps():
    """48x40 cells on the unit square: hx != hy in every stencil and in the
    multigrid coefficients, and tiles that end inside the grid."""
    w = _anisotropic_cavity()
    (g, o), (rg, ro), _ = _run_steps(w, 4)
    _assert_states(g, o, STEP_TOL * 10)
    assert abs(rg[-1].minimum_phi - ro[-1].minimum_phi) <= 1e-12


def _mixed_boundary_cavity(N=40):
    """Lid-driven cavity (UWCDI phase field: the ACDI psi geometry takes no
    MixedBoundary) whose phase field is held at 1 on the lower half of the left wall and whose stress tensors are held at their rest values on every third
    bottom cell (no flux elsewhere)."""
    w = workloads.cavity_disk(N=N)
    half = np.arange(N) < N // 2
    n0 = ef.Neumann(0.0)
    phi_left = ef.MixedBoundary(half.astype(np.uint8), 1.0, 0.0)
    bc_phi = ef.BoundaryConditionSetup(phi_left, n0, n0, n0)
    part = (np.arange(N) % 3 == 0).astype(np.uint8)
    s1 = ef.BoundaryConditionSetup(n0, n0, ef.MixedBoundary(part, 1.0, 0.0), n0)
    s0 = ef.BoundaryConditionSetup(n0, n0, ef.MixedBoundary(part, 0.0, 0.0), n0)
    noflux = ef.BoundaryConditionSetup(n0, n0, n0, n0)
    bcs = ef.FSIBoundaryConditions(w.bcs.U, w.bcs.V, noflux, bc_phi, {"xx": s1, "yy": s1, "xy": s0})
    models = dataclasses.replace(w.models, phase_field_method=ef.PirozzoliUWCDIPhaseField(1.0, delta_normal=1e-14))
    return workloads.Workload("cavity_disk_mixed", w.grid, w.metrics, bcs, models,
                              workloads._numerics(1e-13, 1e-13, "fp64"), w.state, w.dt, 3)


def test_mixed_boundary_steps():
    w = _mixed_boundary_cavity()
    (g, o), _, _ = _run_steps(w, 3)
    _assert_states(g, o, STEP_TOL * 10)


def test_mixed_velocity_boundary_is_rejected():
    """The compact viscous operator takes Dirichlet or Periodic velocity sides only
    (the reference's ArgumentError)."""
    w = workloads.cavity_disk(N=16)
    wall = ef.Dirichlet(0.0)
    lid = ef.MixedBoundary((np.arange(17) < 8).astype(np.uint8), 1.0, 0.0)
    bcs = ef.FSIBoundaryConditions(ef.BoundaryConditionSetup(wall, wall, wall, lid), w.bcs.V, w.bcs.correction,
                                   w.bcs.phi, w.bcs.sigma)
    with pytest.raises(ef.ArgumentError, match="compact viscous operator"):
        ef.build_imex_context(w.metrics, bcs, w.models, numerics=w.numerics)


def test_stretched_mesh_is_rejected():
    """The device step needs uniform spacing; stretched meshes raise
    UnsupportedError when the context is built."""
    w = workloads.cavity_disk(N=32)
    grid = ef.generate_grid(1.0, 1.0, 32, 32, stretch_x="tanh_edges", gamma_x=1.5)
    metrics = ef.build_mesh_metrics(grid)
    with pytest.raises(ef.UnsupportedError):
        ef.build_imex_context(metrics, w.bcs, w.models, numerics=w.numerics)


def test_grid_without_small_coarse_level_is_rejected():
    """33x33 cells cannot be halved and exceed the 1024-cell dense coarse level."""
    w = workloads.cavity_disk(N=33)
    with pytest.raises(ef.UnsupportedError):
        ef.build_imex_context(w.metrics, w.bcs, w.models, numerics=w.numerics)
