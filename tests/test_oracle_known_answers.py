"""The reference's own known-answer tests (test/runtests.jl, test/growth_tests.jl),
restated against the CPU oracle.  These pin the oracle before it is trusted as the
checker of the CUDA path."""
import ctypes as C
import math

import numpy as np
import pytest

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import _abi
from oracle.oracle import Oracle, load
from tests.helpers import dp, fz, periodic_problem

EPS = np.finfo(float).eps


# ---- test/runtests.jl:7-76 -------------------------------------------------------
def _ext(rate, exponent, sxx, syy, sxy, phi):
    lib = load()
    n = len(phi)
    arrs = [np.ascontiguousarray(a, dtype=float) for a in (sxx, syy, sxy, phi)]
    out = [np.zeros(n) for _ in range(3)]
    msg = C.create_string_buffer(256)
    st = lib.oracle_structure_extension_rhs(rate, exponent, n, *[dp(a) for a in arrs],
                                            *[dp(o) for o in out], msg, 256)
    return st, out


def test_extension_constructor_checks():
    m = ef.GeometricStructureExtension(20.0, 4.0, safety_cutoff=1e-6)
    assert (m.max_rate, m.exponent, m.safety_cutoff) == (20.0, 4.0, 1e-6)
    with pytest.raises(ef.ArgumentError):
        ef.GeometricStructureExtension(-1.0)
    with pytest.raises(ef.ArgumentError):
        ef.GeometricStructureExtension(1.0, 0.0)
    with pytest.raises(ef.ArgumentError):
        ef.GeometricStructureExtension(1.0, 4.0, safety_cutoff=1.0)


def test_extension_neutral_state_is_fixed_point():
    phi = [1.0, 0.2, 0.5, 0.0]  # column-major [1.0 0.5; 0.2 0.0]
    st, (rx, ry, rxy) = _ext(20.0, 4.0, np.ones(4), np.ones(4), np.zeros(4), phi)
    assert st == 0
    assert np.all(rx == 0.0) and np.all(ry == 0.0) and np.all(rxy == 0.0)


def test_extension_preserves_unimodular_determinant_and_dissipates():
    st, (rx, ry, rxy) = _ext(20.0, 4.0, np.full(4, 2.0), np.full(4, 0.5), np.zeros(4), np.full(4, 0.2))
    S = np.array([[2.0, 0.0], [0.0, 0.5]])
    R = np.array([[rx[0], rxy[0]], [rxy[0], ry[0]]])
    assert abs(np.trace(np.linalg.inv(S) @ R)) <= 1e-12
    energy_gradient = 0.5 * (np.eye(2) - np.linalg.inv(S))
    assert np.trace(energy_gradient.T @ R) <= 1e-12


def test_extension_rotated_spd_closed_form():
    theta = 0.37
    Q = np.array([[math.cos(theta), -math.sin(theta)], [math.sin(theta), math.cos(theta)]])
    lam = np.array([3.0, 1.0 / 3.0])
    S = Q @ np.diag(lam) @ Q.T
    expected = Q @ np.diag(lam * np.log(lam)) @ Q.T
    st, (rx, ry, rxy) = _ext(20.0, 4.0, [S[0, 0]], [S[1, 1]], [S[0, 1]], [0.3])
    kappa = 20.0 * (1.0 - 0.3) ** 4.0
    assert abs(rx[0] + kappa * expected[0, 0]) <= 1e-12
    assert abs(ry[0] + kappa * expected[1, 1]) <= 1e-12
    assert abs(rxy[0] + kappa * expected[0, 1]) <= 1e-12


def test_extension_non_spd_is_domain_error():
    st, _ = _ext(20.0, 4.0, [1.0], [1.0], [2.0], [0.3])
    assert st == _abi.DOMAIN


def test_extension_safety_reset():
    lib = load()
    sxx, syy, sxy = np.full(4, 2.0), np.full(4, 0.5), np.full(4, 0.1)
    phi = np.ones(4)
    phi[0] = 0.5e-6
    cnt = lib.oracle_apply_structure_extension(_abi.EXT_GEOMETRIC, 1e-6, 4, dp(sxx), dp(syy), dp(sxy), dp(phi))
    assert cnt == 1
    assert (sxx[0], syy[0], sxy[0]) == (1.0, 1.0, 0.0)
    assert sxx[1] == 2.0


# ---- test/runtests.jl:78-87 ----------------------------------------------------------
def test_maxwell_relaxation_exact():
    lib = load()
    out = [np.zeros(1) for _ in range(3)]
    lib.oracle_relaxation_rhs(0.5, 1, dp(np.array([2.0])), dp(np.array([0.5])), dp(np.array([0.1])),
                              *[dp(o) for o in out])
    assert out[0][0] == -0.5 and out[1][0] == 0.25 and out[2][0] == -0.05


# ---- test/runtests.jl:90-119 ---------------------------------------------------------
def test_kolmogorov_body_force_profile():
    grid = ef.generate_grid(6.0, 2.0, 24, 8)
    metrics = ef.build_mesh_metrics(grid, periodic_x=True, periodic_y=False)
    p, n0 = ef.Periodic(), ef.Neumann(0.0)
    bc = ef.BoundaryConditionSetup(p, p, n0, n0)
    wall = ef.BoundaryConditionSetup(p, p, ef.Dirichlet(0.0), ef.Dirichlet(0.0))
    bcs = ef.FSIBoundaryConditions(wall, wall, bc, bc, {"xx": bc, "yy": bc, "xy": bc})
    ky = 2 * math.pi * 4 / 2.0
    amp = ky ** 2 / 100.0
    models = ef.FSIModels(body_force=ef.KolmogorovBodyForce(amp, ky))
    o = Oracle(metrics, bcs, models, ef.IMEXNumerics())
    Fx, Fy = fz(25, 8), fz(24, 9)
    o.call("body_force", 0.0, dp(Fx), dp(Fy))
    assert np.all(Fy == 0.0) and np.all(np.isfinite(Fx))
    y = 0.0
    for j in range(8):
        y += 0.5 * metrics.dy_c[j]
        assert np.max(np.abs(Fx[:, j] - amp * math.sin(ky * y))) <= 1e-12
        y += 0.5 * metrics.dy_c[j]


# ---- test/runtests.jl:160-227 ----------------------------------------------------------
PF_METHODS = {
    "current_cdi": ef.CurrentCDIPhaseField(4.0, 2 / 16, delta_normal=1e-6),
    "acdi": ef.JainACDIPhaseField(0.2, 0.51 / 16),
    "uwcdi": ef.PirozzoliUWCDIPhaseField(1.0),
    "uwcdi_youngs": ef.PirozzoliUWCDIPhaseField(1.0, normal_reconstruction="youngs"),
    "uwcdi_smoothed9": ef.PirozzoliUWCDIPhaseField(1.0, normal_reconstruction="smoothed9"),
}


def _pf_setup(method):
    grid, metrics, bcs, models = periodic_problem(16, method)
    U = np.full((17, 16), 0.2, order="F")
    V = np.full((16, 17), -0.1, order="F")
    U[-1, :] = U[0, :]
    V[:, -1] = V[:, 0]
    return grid, metrics, Oracle(metrics, bcs, models, ef.IMEXNumerics()), U, V


def _phi_wave(grid):
    x, y = np.asarray(grid.x_p), np.asarray(grid.y_p)
    return np.asfortranarray(0.5 + 0.2 * np.sin(2 * np.pi * x)[:, None] * np.cos(2 * np.pi * y)[None, :])


def test_phase_field_labels():
    assert ef.phase_field_label(PF_METHODS["current_cdi"]) == "current_cdi"
    assert ef.phase_field_label(PF_METHODS["acdi"]) == "jain_acdi"
    assert ef.phase_field_label(PF_METHODS["uwcdi"]) == "pirozzoli_uwcdi"
    assert abs(ef.jain_equilibrium_initialization_epsilon(PF_METHODS["acdi"]) - 1.02 / 16) < 1e-15


@pytest.mark.parametrize("name", list(PF_METHODS))
def test_phase_field_constant_state_stays_constant(name):
    grid, metrics, o, U, V = _pf_setup(PF_METHODS[name])
    phi = np.full((16, 16), 0.37, order="F")
    rhs = fz(16, 16)
    o.call("phase_field_rhs", dp(U), dp(V), dp(phi), dp(fz(16, 16)), dp(rhs))
    assert np.max(np.abs(rhs)) <= 1e-11


@pytest.mark.parametrize("name", list(PF_METHODS))
def test_phase_field_periodic_integral_vanishes(name):
    grid, metrics, o, U, V = _pf_setup(PF_METHODS[name])
    phi = _phi_wave(grid)
    rhs = fz(16, 16)
    o.call("phase_field_rhs", dp(U), dp(V), dp(phi), dp(fz(16, 16)), dp(rhs))
    integral = sum(rhs[i, j] * metrics.dx_c[i] * metrics.dy_c[j] for j in range(16) for i in range(16))
    assert abs(integral) <= 1e-11


def test_dynamic_acdi_zero_velocity_gives_zero_rhs():
    grid, metrics, bcs, models = periodic_problem(16, ef.JainACDIPhaseField(1.0, 0.51 / 16, dynamic_gamma=True))
    o = Oracle(metrics, bcs, models, ef.IMEXNumerics())
    rhs = fz(16, 16)
    o.call("phase_field_rhs", dp(fz(17, 16)), dp(fz(16, 17)), dp(_phi_wave(grid)), dp(fz(16, 16)), dp(rhs))
    assert np.max(np.abs(rhs)) <= 1e-12


def test_uwcdi_strang_step_conserves_mass():
    grid, metrics, o, U, V = _pf_setup(PF_METHODS["uwcdi"])
    phi = _phi_wave(grid)
    out = fz(16, 16)
    o.call("uwcdi_strang_step", dp(U), dp(V), dp(phi), 0.01, 1, dp(out))
    area = np.outer(metrics.dx_c, metrics.dy_c)
    assert abs(np.sum(out * area) - np.sum(phi * area)) <= 1e-12


def test_phase_field_constructor_checks():
    with pytest.raises(ef.ArgumentError):
        ef.PirozzoliUWCDIPhaseField(0.9)
    with pytest.raises(ef.ArgumentError):
        ef.PirozzoliUWCDIPhaseField(1.0, normal_reconstruction="invalid")
    with pytest.raises(ef.ArgumentError):
        ef.JainACDIPhaseField(-1.0, 0.01)


# ---- test/growth_tests.jl:6-57 ------------------------------------------------------
def _fields(models, phi, c):
    grid = ef.generate_grid(1.0, 1.0, 2, 2)
    metrics = ef.build_mesh_metrics(grid, periodic_x=True, periodic_y=True)
    p = ef.Periodic()
    bc = ef.BoundaryConditionSetup(p, p, p, p)
    bcs = ef.FSIBoundaryConditions(bc, bc, bc, bc, {"xx": bc, "yy": bc, "xy": bc})
    o = Oracle(metrics, bcs, models, ef.IMEXNumerics())
    outs = [fz(2, 2) for _ in range(8)]
    te = np.zeros(1)
    o.call("constitutive_fields", dp(phi), dp(c), *[dp(a) for a in outs], dp(te))
    return outs, te[0]


def test_growth_closures():
    phi = np.asfortranarray([[0.0, 0.5], [0.25, 1.0]])
    c = np.full((2, 2), 0.25, order="F")
    (G, *_), _ = _fields(ef.FSIModels(growth_source=ef.NoGrowth()), phi, c)
    assert np.all(G == 0.0)
    (G, *_), _ = _fields(ef.FSIModels(growth_source=ef.ConstantIntrinsicGrowth(0.2)), phi, c)
    assert np.allclose(G, 0.2 * phi)
    (G, Kxx, Kxy, Kyx, Kyy, *_), te = _fields(
        ef.FSIModels(growth_source=ef.SaturatingResourceGrowth(0.6, 0.25)), phi, c)
    assert np.allclose(G, 0.3 * phi)
    assert np.allclose(Kxx, 0.5 * G) and np.allclose(Kyy, 0.5 * G) and te == 0.0
    with pytest.raises(ef.ArgumentError):
        ef.SaturatingResourceGrowth(0.6, 0.0)
    (G, Kxx, Kxy, Kyx, Kyy, *_), te = _fields(
        ef.FSIModels(growth_source=ef.SaturatingResourceGrowth(0.6, 0.25),
                     growth_tensor=ef.DirectionalGrowthTensor(3.0, 4.0)), phi, c)
    assert np.max(np.abs(Kxx + Kyy - G)) < 1e-14
    assert np.allclose(Kxy, Kyx) and np.allclose(Kxx, (9 / 25) * G)
    with pytest.raises(ef.ArgumentError):
        ef.DirectionalGrowthTensor(0.0, 0.0)


def test_resource_transport_and_consumption():
    grid = ef.generate_grid(1.0, 1.0, 8, 8)
    metrics = ef.build_mesh_metrics(grid, periodic_x=True, periodic_y=True)
    p = ef.Periodic()
    bc = ef.BoundaryConditionSetup(p, p, p, p)
    bcs = ef.FSIBoundaryConditions(bc, bc, bc, bc, {"xx": bc, "yy": bc, "xy": bc})
    models = ef.FSIModels(diffusivity=ef.ConstantDiffusivity(0.01),
                          resource_consumption=ef.SaturatingResourceConsumption(0.4, 0.5))
    o = Oracle(metrics, bcs, models, ef.IMEXNumerics())
    c = np.asfortranarray(0.5 + 0.1 * np.sin(2 * np.pi * np.asarray(grid.x_p))[:, None] * np.ones((1, 8)))
    U = np.full((9, 8), 0.2, order="F")
    V = fz(8, 9)
    rhs = fz(8, 8)
    o.call("resource_explicit_rhs", dp(U), dp(V), dp(c), dp(fz(8, 8)), dp(rhs))
    area = np.outer(metrics.dx_c, metrics.dy_c)
    assert abs(np.sum(rhs * area)) < 1e-12
    phi = np.full((8, 8), 0.5, order="F")
    outs = [fz(8, 8) for _ in range(8)]
    o.call("constitutive_fields", dp(phi), dp(c), *[dp(a) for a in outs], dp(np.zeros(1)))
    D, sink = outs[6], outs[7]
    assert np.all(D == 0.01)
    assert np.all(sink >= 0.0)
    with pytest.raises(ef.ArgumentError):
        ef.ConstantDiffusivity(0.0)


# ---- test/growth_tests.jl:59-71 (host constructors) --------------------------------------
def test_legacy_constructors():
    state = ef.FSIState(fz(9, 8), fz(8, 9), fz(8, 8), np.ones((8, 8)), np.ones((8, 8)), fz(8, 8))
    assert state.resource.shape == (8, 8) and np.all(state.resource == 0)
    p = ef.Periodic()
    bc = ef.BoundaryConditionSetup(p, p, p, p)
    b = ef.FSIBoundaryConditions(bc, bc, bc, bc, {"xx": bc, "yy": bc, "xy": bc})
    assert b.resource is bc
    assert isinstance(ef.FSIModels().growth_source, ef.NoGrowth)
    assert isinstance(ef.FSIModels().diffusivity, ef.NoDiffusion)


# ---- test/growth_tests.jl:73-94 ------------------------------------------------------------
def test_projection_rejects_incompatible_source_and_meets_dirichlet_constraint():
    grid = ef.generate_grid(1.0, 1.0, 8, 8)
    pm = ef.build_mesh_metrics(grid, periodic_x=True, periodic_y=True)
    p = ef.Periodic()
    per = ef.BoundaryConditionSetup(p, p, p, p)
    bcs = ef.FSIBoundaryConditions(per, per, per, per, {"xx": per, "yy": per, "xy": per})
    o = Oracle(pm, bcs, ef.FSIModels(), ef.IMEXNumerics())
    r = _abi.ProjectionResultC()
    with pytest.raises(ef.ArgumentError):
        o.call("project", dp(fz(9, 8)), dp(fz(8, 9)), dp(np.full((8, 8), 0.1, order="F")), C.byref(r))
    om = ef.build_mesh_metrics(grid)
    d0 = ef.Dirichlet(0.0)
    bq = ef.BoundaryConditionSetup(d0, d0, d0, d0)
    n0 = ef.Neumann(0.0)
    nb = ef.BoundaryConditionSetup(n0, n0, n0, n0)
    bcs = ef.FSIBoundaryConditions(nb, nb, bq, nb, {"xx": nb, "yy": nb, "xy": nb})
    o = Oracle(om, bcs, ef.FSIModels(), ef.IMEXNumerics(projection_reltol=1e-12, projection_maxiter=2000))
    U, V = fz(9, 8), fz(8, 9)
    src = np.full((8, 8), 0.05, order="F")
    o.call("project", dp(U), dp(V), dp(src), C.byref(r))
    assert r.constraint_linf < 1e-7
    div = fz(8, 8)
    o.call("divergence", dp(U), dp(V), dp(div))
    assert np.max(np.abs(div - src)) < 1e-7


# ---- test/growth_tests.jl:96-142 -----------------------------------------------------------
def growth_smoke_problem():
    grid = ef.generate_grid(1.0, 1.0, 8, 8)
    metrics = ef.build_mesh_metrics(grid, periodic_x=True, periodic_y=False)
    px = ef.Periodic()
    bc_neumann = ef.BoundaryConditionSetup(px, px, ef.Neumann(0.0), ef.Neumann(0.0))
    bc_v = ef.BoundaryConditionSetup(px, px, ef.Neumann(0.0), ef.Dirichlet(0.0))
    bc_q = ef.BoundaryConditionSetup(px, px, ef.Dirichlet(0.0), ef.Neumann(0.0))
    bc_c = ef.BoundaryConditionSetup(px, px, ef.Dirichlet(1.0), ef.Dirichlet(1.0))
    bcs = ef.FSIBoundaryConditions(bc_neumann, bc_v, bc_q, bc_neumann, bc_c,
                                   {"xx": bc_neumann, "yy": bc_neumann, "xy": bc_neumann})
    state = ef.FSIState(fz(9, 8), fz(8, 9), np.full((8, 8), 0.5), np.ones((8, 8)), np.ones((8, 8)),
                        np.ones((8, 8)), fz(8, 8))
    models = ef.FSIModels(growth_source=ef.SaturatingResourceGrowth(0.02, 0.5),
                          growth_tensor=ef.IsotropicGrowthTensor(), diffusivity=ef.ConstantDiffusivity(0.01),
                          resource_consumption=ef.SaturatingResourceConsumption(0.002, 0.5))
    return grid, metrics, bcs, models, state


def test_coupled_imex_growth_smoke():
    grid, metrics, bcs, models, state = growth_smoke_problem()
    o = Oracle(metrics, bcs, models, ef.IMEXNumerics())
    o.upload(state)
    res = o.make_velocity_compatible()
    o.download(state)
    assert res.constraint_linf < 1e-7
    assert np.max(np.abs(state.U)) > 0.0
    o.handle.set_correction(fz(8, 8))
    rep = o.step(0.0, 1e-4)
    o.download(state)
    assert rep.maximum_projection_constraint_linf < 1e-6
    assert np.max(np.abs(state.U[-1, :] - state.U[0, :])) < 1e-12
    assert np.max(np.abs(state.V[:, -1])) < 1e-12
    assert rep.maximum_growth_trace_error < 1e-12
    assert rep.minimum_resource > 0.0
    assert np.all(np.isfinite(state.phi)) and np.all(np.isfinite(state.sigma_xx))


# ---- test/growth_tests.jl:144-162 ---------------------------------------------------------
def test_no_growth_rest_state():
    grid, metrics, bcs, models = periodic_problem(8, None)
    state = ef.FSIState(fz(9, 8), fz(8, 9), np.full((8, 8), 0.5), np.ones((8, 8)), np.ones((8, 8)), fz(8, 8))
    o = Oracle(metrics, bcs, models, ef.IMEXNumerics())
    o.upload(state)
    o.make_velocity_compatible()
    rep = o.step(0.0, 1e-4)
    o.download(state)
    assert rep.maximum_growth_trace_error == 0.0
    assert np.all(state.resource == 0.0)
    assert np.max(np.abs(state.U)) < 1e-9 and np.max(np.abs(state.V)) < 1e-9
    assert np.max(np.abs(state.phi - 0.5)) < 1e-9


def test_tensor_cell_diagnostics_known_answer():
    """tensor_cell_diagnostics_2d (test/runtests.jl:140-145)."""
    from oracle.oracle import load
    out = (C.c_double * 5)()
    load().oracle_tensor_cell_diagnostics(2.0, 0.5, 0.0, 0.2, 10.0, out)
    det, err, lmin, lmax, stress = list(out)
    assert det == pytest.approx(1.0) and err == pytest.approx(0.0, abs=1e-15)
    assert lmin == pytest.approx(0.5) and lmax == pytest.approx(2.0) and stress > 0.0


def test_oracle_state_diagnostics_disk():
    """Oracle diagnostics of a sharp disk: centroid at the disk centre, a perimeter
    proxy near 2 pi r, and round covariance."""
    from eulerianfsi_b200 import diagnostics, workloads
    from eulerianfsi_b200.imex import ConfigBlock, Handle
    from oracle.oracle import load
    w = workloads.cavity_disk(N=64)
    h = Handle(load(), "oracle_", ConfigBlock(w.metrics, w.bcs, w.models, w.numerics), w.metrics)
    h.upload(w.state)
    d = diagnostics.state_diagnostics(h, diagnostics.DiagnosticsConfig(nmax=4))
    assert abs(d["x_centroid"] - 0.6) < 1e-3 and abs(d["y_centroid"] - 0.5) < 1e-3
    assert abs(d["perimeter_proxy"] - 2 * np.pi * 0.2) / (2 * np.pi * 0.2) < 0.05
    assert d["aspect_ratio"] < 1.01 and max(d["amplitudes"]) < 1e-2 * d["perimeter_proxy"]
    assert d["global_region"]["cells"] == 64 * 64 and d["global_region"]["non_spd_cells"] == 0
