"""Finite-difference sensitivities (eulerianfsi_b200.sensitivity) on the CPU: the
difference formulas on an analytic function, the objective's guards, a gradient
check through the oracle on a small cavity, and the replica ensemble on two gloo
ranks, which must return exactly the serial results."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import sensitivity as sens, workloads
from tests.gpu_util import oracle_final_state

N_SMALL, STEPS_SMALL = 16, 3
T_SMALL = STEPS_SMALL * 0.2 / N_SMALL


def _quadratic(p):
    p = np.asarray(p)
    return float(1.5 * p[0] ** 2 - p[1] * p[2] + 0.25 * p[3] + 2.0)


def _quadratic_grad(p):
    return np.array([3.0 * p[0], -p[2], -p[1], 0.25])


def test_central_differences_are_exact_on_a_quadratic():
    p = np.array(sens.DEFAULT_PARAMETERS)
    res = sens.gradient_check(_quadratic, p, seed=3, rel_h=1e-3)
    np.testing.assert_allclose(res["gradient"], _quadratic_grad(p), rtol=1e-9, atol=1e-12)
    d = sens.seeded_direction(3)
    assert abs(res["directional"] - _quadratic_grad(p) @ d) <= 1e-9
    assert res["rel_diff"] <= 1e-9 and res["runs"] == 11


def test_seeded_direction_is_a_unit_vector_and_reproducible():
    a, b = sens.seeded_direction(7), sens.seeded_direction(7)
    np.testing.assert_array_equal(a, b)
    assert abs(np.linalg.norm(a) - 1.0) <= 1e-15 and a.shape == (4,)


def test_difference_points_reject_a_zero_step():
    with pytest.raises(ef.ArgumentError):
        sens.difference_points(np.zeros(4), np.eye(4), 1e-6)


def test_objective_guards():
    w = workloads.cavity_disk_sensitivity(N=8, T=0.025)
    st = w.state.copy()
    st.sigma_xy[2, 2] = 2.0  # det = 1 - 4 < 0
    with pytest.raises(ef.DomainError):
        sens.objective(st, w, 0.1)
    st = w.state.copy()
    st.phi[...] = 0.0
    with pytest.raises(ef.ArgumentError):
        sens.objective(st, w, 0.1)


def test_objective_of_the_initial_state_is_the_disk_centroid():
    """sigma = I: no elastic energy, and the centroid of the symmetric profile is the
    disk centre up to the wall truncation of its tail."""
    w = workloads.cavity_disk_sensitivity(N=64, params=(0.1, 1.0, 0.5, 0.45), T=0.0)
    assert w.steps == 0
    assert abs(sens.objective(w.state, w, 0.1) - 0.45) <= 1e-6


def test_oracle_gradient_check_small_cavity():
    """Gradient by per-parameter central differences against the directional
    difference along a seeded direction, through the FP64 oracle."""
    ev = sens.make_evaluator(N_SMALL, T_SMALL, run=oracle_final_state)
    res = sens.gradient_check(ev, seed=0)
    assert res["rel_diff"] <= 1e-5, res
    g = np.array(res["gradient"])
    assert np.all(np.isfinite(g)) and abs(g[3]) > 0.5  # the centroid follows the disk centre


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ev = sens.make_evaluator(N_SMALL, T_SMALL, run=oracle_final_state)
        dirs = np.vstack([np.eye(4), sens.seeded_direction(1)[None, :]])
        J, D = sens.central_differences(ev, sens.DEFAULT_PARAMETERS, dirs, 1e-6, group=dist.group.WORLD)
        out[rank] = (J, D.tolist())
    finally:
        dist.destroy_process_group()


def test_replica_ensemble_on_two_gloo_ranks_matches_serial():
    ev = sens.make_evaluator(N_SMALL, T_SMALL, run=oracle_final_state)
    dirs = np.vstack([np.eye(4), sens.seeded_direction(1)[None, :]])
    J, D = sens.central_differences(ev, sens.DEFAULT_PARAMETERS, dirs, 1e-6)
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        for r in range(world):
            assert out[r][0] == J and out[r][1] == D.tolist()


def test_objective_cotangent_matches_differences_of_the_objective():
    """The host half of the adjoint gradient: dJ/d(final state) and dJ/dG of the
    objective against central differences of sensitivity.objective."""
    w = workloads.cavity_disk_sensitivity(N=8, T=0.025)
    rng = np.random.default_rng(4)
    st = w.state.copy()
    st.phi[...] = 0.2 + 0.6 * rng.random(st.phi.shape)
    st.sigma_xx[...] = 1.0 + 0.3 * rng.random(st.phi.shape)
    st.sigma_yy[...] = 1.0 + 0.3 * rng.random(st.phi.shape)
    st.sigma_xy[...] = 0.1 * rng.standard_normal(st.phi.shape)
    G = 0.1
    J, cot, dJdG = sens.objective_cotangent(st, w, G)
    assert abs(J - sens.objective(st, w, G)) <= 1e-15
    eps = 1e-6
    for name in ("phi", "sigma_xx", "sigma_yy", "sigma_xy"):
        d = rng.standard_normal(st.phi.shape)
        a, b = st.copy(), st.copy()
        getattr(a, name)[...] += eps * d
        getattr(b, name)[...] -= eps * d
        fd = (sens.objective(a, w, G) - sens.objective(b, w, G)) / (2 * eps)
        assert abs(fd - float(np.sum(cot[name] * d))) <= 1e-8 * max(abs(fd), 1.0), name
    fdG = (sens.objective(st, w, G + eps) - sens.objective(st, w, G - eps)) / (2 * eps)
    assert abs(fdG - dJdG) <= 1e-9


def test_circle_center_derivative_matches_differences():
    from eulerianfsi_b200.init import initialize_circle
    w = workloads.cavity_disk_sensitivity(N=16, T=0.025)
    h = 1.0 / 16
    c = (0.6, 0.5)
    dcx, dcy = sens.circle_center_derivative(w.grid, c, 0.2, 1.5 * h)
    eps = 1e-7
    fx = (initialize_circle(w.grid, (c[0] + eps, c[1]), 0.2, 1.5 * h) -
          initialize_circle(w.grid, (c[0] - eps, c[1]), 0.2, 1.5 * h)) / (2 * eps)
    fy = (initialize_circle(w.grid, (c[0], c[1] + eps), 0.2, 1.5 * h) -
          initialize_circle(w.grid, (c[0], c[1] - eps), 0.2, 1.5 * h)) / (2 * eps)
    assert np.max(np.abs(fx - dcx)) <= 1e-6 and np.max(np.abs(fy - dcy)) <= 1e-6
