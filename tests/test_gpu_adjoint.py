"""The discrete adjoint of the IMEX step through the C-ABI.

* Dot-product tests of the transposed pieces against the production forward entry
  points: for the explicit tendencies (momentum forcing, viscous operator, ACDI phase
  field, structure tensor) and for the projection, <T'(x) v, w> by central
  differences of T equals <v, T'(x)^T w> from the adjoint, on walled and on periodic
  grids, including the derivatives in the elastic coefficient G and the lid datum.
* One and three steps (two checkpoint segments): <d step^n / dx v, w> by central
  differences equals <v, adjoint(w)>.
* The gradient of the cavity-disk objective over (G, lid speed, disk centre x, y)
  equals the central-difference gradient of the CUDA forward runs and of the FP64
  oracle's forward runs (N=32, 40 steps) to 1e-5 relative.

Solves run to 1e-13 so that differences of the forward resolve the derivatives; the
random fields keep velocities away from zero and phi inside (0, 1), where the upwind
and clamp switches do not flip under the perturbation."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import _abi, adjoint, sensitivity as sens, workloads
from eulerianfsi_b200.imex import ConfigBlock, Handle
from tests.gpu_util import oracle_final_state
from tests.helpers import dp, fz

pytestmark = pytest.mark.gpu


def _tight(numerics, **kw):
    ls = dataclasses.replace(numerics.linear_solvers, velocity_method="direct")
    return dataclasses.replace(numerics, linear_solvers=ls, projection_reltol=1e-13, projection_maxiter=3000, **kw)


def _problem(kind, N=16, G=0.3, lid=0.8):
    """(metrics, bcs, models, numerics): the cavity (walls, moving lid) or a doubly
    periodic box, ACDI, constant viscosity, linear elastic stress, Maxwell relaxation
    and the geometric structure extension."""
    h = 1.0 / N
    models = ef.FSIModels(viscosity=ef.ConstantViscosity(0.01), elastic_stress=ef.LinearInternalTensorStress(G),
                          tensor_relaxation=ef.MaxwellRelaxation(0.5),
                          phase_field_method=ef.JainACDIPhaseField(1.0, 0.51 * h, delta_normal=1e-14,
                                                                   dynamic_gamma=False))
    if kind == "cavity":
        w = workloads.cavity_disk_sensitivity(N, (G, lid, 0.55, 0.5), 0.1)
        metrics, bcs = w.metrics, w.bcs
    else:
        grid = ef.generate_grid(1.0, 1.0, N, N)
        metrics = ef.build_mesh_metrics(grid, periodic_x=True, periodic_y=True)
        p = ef.Periodic()
        bc = ef.BoundaryConditionSetup(p, p, p, p)
        bcs = ef.FSIBoundaryConditions(bc, bc, bc, bc, {"xx": bc, "yy": bc, "xy": bc})
    ext = ef.GeometricStructureExtension(20.0, 4.0, safety_cutoff=1e-6)
    num = _tight(ef.IMEXNumerics(structure_extension=ext), check_stage1_constraint=False)
    return metrics, bcs, models, num


def _fields(metrics, seed, walls):
    rng = np.random.default_rng(seed)
    Nx, Ny = metrics.Nx, metrics.Ny
    x = (np.arange(Nx) + 0.5) / Nx
    y = (np.arange(Ny) + 0.5) / Ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    f = lambda a: np.asfortranarray(a, dtype=np.float64)
    U = 0.3 + 0.2 * rng.random((Nx + 1, Ny))
    V = -0.3 - 0.2 * rng.random((Nx, Ny + 1))
    if walls:
        U[0, :] = U[-1, :] = 0.0
        V[:, 0] = V[:, -1] = 0.0
    else:  # the periodic duplicate faces repeat faces 0
        U[-1, :] = U[0, :]
        V[:, -1] = V[:, 0]
    phi = 0.5 + 0.4 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) + 0.02 * rng.standard_normal((Nx, Ny))
    phi = np.clip(phi, 0.02, 0.98)
    return dict(U=f(U), V=f(V), phi=f(phi), sxx=f(1.0 + 0.3 * rng.random((Nx, Ny))),
                syy=f(1.0 + 0.3 * rng.random((Nx, Ny))), sxy=f(0.1 * rng.standard_normal((Nx, Ny))))


def _direction(metrics, seed, walls):
    rng = np.random.default_rng(seed)
    Nx, Ny = metrics.Nx, metrics.Ny
    d = {k: np.asfortranarray(rng.standard_normal(s)) for k, s in
         (("U", (Nx + 1, Ny)), ("V", (Nx, Ny + 1)), ("phi", (Nx, Ny)), ("sxx", (Nx, Ny)), ("syy", (Nx, Ny)),
          ("sxy", (Nx, Ny)))}
    if walls:  # boundary faces hold wall data in a state; keep them fixed
        d["U"][0, :] = d["U"][-1, :] = 0.0
        d["V"][:, 0] = d["V"][:, -1] = 0.0
    else:
        d["U"][-1, :] = d["U"][0, :]
        d["V"][:, -1] = d["V"][:, 0]
    return d


def _tendencies(h, fl):
    """Forward tendencies through the production entry points."""
    Nx, Ny = h.metrics.Nx, h.metrics.Ny
    N = Nx * Ny
    Fx, Fy = fz(Nx + 1, Ny), fz(Nx, Ny + 1)
    h.call("momentum_explicit_rhs", 0.0, dp(fl["U"]), dp(fl["V"]), dp(fl["phi"]), dp(fl["sxx"]), dp(fl["syy"]),
           dp(fl["sxy"]), None, dp(Fx), dp(Fy))
    uv = np.concatenate([np.ravel(fl["U"][:Nx, :], order="F"), np.ravel(fl["V"][:, :Ny], order="F")])
    I = np.zeros(2 * N)
    h.call("apply_viscous_operator", dp(fl["phi"]), dp(uv), dp(I))
    Ephi = fz(Nx, Ny)
    h.call("phase_field_rhs", dp(fl["U"]), dp(fl["V"]), dp(fl["phi"]), None, dp(Ephi))
    Exx, Eyy, Exy = fz(Nx, Ny), fz(Nx, Ny), fz(Nx, Ny)
    h.call("structure_tensor_rhs", dp(fl["sxx"]), dp(fl["syy"]), dp(fl["sxy"]), dp(fl["U"]), dp(fl["V"]),
           dp(fl["phi"]), None, dp(Exx), dp(Eyy), dp(Exy))
    return {"Eu": np.asfortranarray(Fx[:Nx, :]), "Ev": np.asfortranarray(Fy[:, :Ny]),
            "Iu": I[:N].reshape((Nx, Ny), order="F"), "Iv": I[N:].reshape((Nx, Ny), order="F"),
            "Ephi": Ephi, "Exx": Exx, "Eyy": Eyy, "Exy": Exy}


def _dot(a, b):
    return sum(float(np.sum(a[k] * b[k])) for k in a)


@pytest.mark.parametrize("kind", ["cavity", "periodic"])
def test_tendencies_transpose_dot_product(kind):
    metrics, bcs, models, num = _problem(kind)
    ctx = ef.build_imex_context(metrics, bcs, models, numerics=num)
    h = ctx.handle
    walls = kind == "cavity"
    x = _fields(metrics, 1, walls)
    v = _direction(metrics, 2, walls)
    rng = np.random.default_rng(3)
    w = {k: np.asfortranarray(rng.standard_normal((metrics.Nx, metrics.Ny)))
         for k in ("Eu", "Ev", "Iu", "Iv", "Ephi", "Exx", "Eyy", "Exy")}
    eps = 1e-6
    tp = _tendencies(h, {k: x[k] + eps * v[k] for k in x})
    tm = _tendencies(h, {k: x[k] - eps * v[k] for k in x})
    fd = sum(float(np.sum((tp[k] - tm[k]) * w[k])) for k in w) / (2.0 * eps)
    fields = ef.FSIState(x["U"], x["V"], x["phi"], fz(metrics.Nx, metrics.Ny), x["sxx"], x["syy"], x["sxy"])
    lam, pg = adjoint.tendencies_adjoint(ctx, fields, w)
    ad = _dot({"U": v["U"], "V": v["V"], "phi": v["phi"], "sigma_xx": v["sxx"], "sigma_yy": v["syy"],
               "sigma_xy": v["sxy"]}, lam)
    assert abs(fd - ad) <= 1e-7 * max(abs(fd), 1.0), (fd, ad)
    # the elastic coefficient: T is affine in G, so a difference at G0 +/- G0/2 is exact
    G0 = models.elastic_stress.coefficient
    vals = []
    for G in (G0 * 1.5, G0 * 0.5):
        m2 = dataclasses.replace(models, elastic_stress=ef.LinearInternalTensorStress(G))
        c2 = ef.build_imex_context(metrics, bcs, m2, numerics=num)
        vals.append(_dot(_tendencies(c2.handle, x), w))
        c2.handle.close()
    fdG = (vals[0] - vals[1]) / G0
    assert abs(fdG - pg.elastic_coefficient) <= 1e-9 * max(abs(fdG), 1.0), (fdG, pg.elastic_coefficient)
    if walls:  # the lid datum (uniform U-top data); T is affine in it as well
        vals = []
        for lid in (0.8 * 1.5, 0.8 * 0.5):
            wl = workloads.cavity_disk_sensitivity(metrics.Nx, (0.3, lid, 0.55, 0.5), 0.1)
            c2 = ef.build_imex_context(metrics, wl.bcs, models, numerics=num)
            vals.append(_dot(_tendencies(c2.handle, x), w))
            c2.handle.close()
        fdl = (vals[0] - vals[1]) / 0.8
        adl = float(np.sum(pg.U_top))
        assert abs(fdl - adl) <= 1e-9 * max(abs(fdl), 1.0), (fdl, adl)
    ctx.handle.close()


@pytest.mark.parametrize("kind", ["cavity", "periodic"])
def test_projection_transpose_dot_product(kind):
    metrics, bcs, models, num = _problem(kind)
    ctx = ef.build_imex_context(metrics, bcs, models, numerics=num)
    h = ctx.handle
    Nx, Ny = metrics.Nx, metrics.Ny
    rng = np.random.default_rng(5)
    U = np.asfortranarray(rng.standard_normal((Nx + 1, Ny)))
    V = np.asfortranarray(rng.standard_normal((Nx, Ny + 1)))
    if kind == "cavity":  # compatible data: no flux through the walls
        U[0, :] = U[-1, :] = 0.0
        V[:, 0] = V[:, -1] = 0.0
    else:  # periodic: the duplicate faces repeat faces 0
        U[-1, :] = U[0, :]
        V[:, -1] = V[:, 0]
    wU = np.asfortranarray(rng.standard_normal((Nx + 1, Ny)))
    wV = np.asfortranarray(rng.standard_normal((Nx, Ny + 1)))

    def P(u, v):
        u, v = u.copy(order="F"), v.copy(order="F")
        h.set_correction(fz(Nx, Ny))
        h.call("project", dp(u), dp(v), None, C.byref(_abi.ProjectionResultC()))
        return u, v

    pu, pv = P(U, V)  # the projection is linear here (zero target, zero data): <P U, w> = <U, P^T w>
    lhs = float(np.sum(pu * wU) + np.sum(pv * wV))
    lu, lv = adjoint.project_adjoint(ctx, wU, wV)
    rhs = float(np.sum(U * lu) + np.sum(V * lv))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1.0), (lhs, rhs)
    ctx.handle.close()


def _step_map(metrics, bcs, models, num, x, dts):
    """Final state after len(dts) steps from the fields x."""
    gpu = Handle(_abi.load_library(), "efsi_", ConfigBlock(metrics, bcs, models, num), metrics)
    st = ef.FSIState(x["U"].copy(order="F"), x["V"].copy(order="F"), x["phi"].copy(order="F"),
                     fz(metrics.Nx, metrics.Ny), x["sxx"].copy(order="F"), x["syy"].copy(order="F"),
                     x["sxy"].copy(order="F"))
    gpu.upload(st)
    gpu.set_correction(fz(metrics.Nx, metrics.Ny))
    arr = (C.c_double * len(dts))(*dts)
    gpu.call("step_n", 0.0, arr, len(dts), None)
    gpu.download(st)
    gpu.close()
    return {"U": st.U, "V": st.V, "phi": st.phi, "sxx": st.sigma_xx, "syy": st.sigma_yy, "sxy": st.sigma_xy}


@pytest.mark.parametrize("kind,steps,every", [("cavity", 1, 0), ("cavity", 3, 2), ("periodic", 2, 1)])
def test_step_adjoint_dot_product(kind, steps, every):
    metrics, bcs, models, num = _problem(kind)
    walls = kind == "cavity"
    x = _fields(metrics, 11, walls)
    x["U"] *= 0.2
    x["V"] *= 0.2
    v = _direction(metrics, 12, walls)
    rng = np.random.default_rng(13)
    w = _direction(metrics, 14, walls)
    dt = 0.2 / metrics.Nx
    dts = [dt] * steps
    eps = 1e-6
    fp = _step_map(metrics, bcs, models, num, {k: x[k] + eps * v[k] for k in x}, dts)
    fm = _step_map(metrics, bcs, models, num, {k: x[k] - eps * v[k] for k in x}, dts)
    fd = sum(float(np.sum((fp[k] - fm[k]) * w[k])) for k in w) / (2.0 * eps)
    ctx = ef.build_imex_context(metrics, bcs, models, numerics=num)
    st = ef.FSIState(x["U"].copy(order="F"), x["V"].copy(order="F"), x["phi"].copy(order="F"),
                     fz(metrics.Nx, metrics.Ny), x["sxx"].copy(order="F"), x["syy"].copy(order="F"),
                     x["sxy"].copy(order="F"))
    final, pullback = adjoint.rrule_integrate_steps(st, 0.0, dts, ctx, every)
    cot = {"U": w["U"], "V": w["V"], "phi": w["phi"], "sigma_xx": w["sxx"], "sigma_yy": w["syy"],
           "sigma_xy": w["sxy"]}
    g, _ = pullback(cot)
    ad = float(np.sum(g.U * v["U"]) + np.sum(g.V * v["V"]) + np.sum(g.phi * v["phi"]) +
               np.sum(g.sigma_xx * v["sxx"]) + np.sum(g.sigma_yy * v["syy"]) + np.sum(g.sigma_xy * v["sxy"]))
    assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1.0), (fd, ad)
    # the forward of the rrule is the plain stepping
    plain = _step_map(metrics, bcs, models, num, x, dts)
    np.testing.assert_array_equal(final.U, plain["U"])
    ctx.handle.close()


N, STEPS = 32, 40


def test_adjoint_gradient_matches_finite_differences():
    """C4 objective at N=32 over 40 steps: adjoint gradient vs central differences of
    the CUDA forward and of the FP64 oracle forward, 1e-5 relative."""
    T = STEPS * 0.2 / N
    res = sens.adjoint_gradient(N, T)
    gpu = sens.gradient_check(sens.make_evaluator(N, T), seed=0)
    ora = sens.gradient_check(sens.make_evaluator(N, T, run=oracle_final_state), seed=0)
    a, g, o = (np.array(r["gradient"]) for r in (res, gpu, ora))
    assert abs(res["J"] - gpu["J"]) <= 1e-12 * abs(gpu["J"])
    assert np.linalg.norm(a - g) <= 1e-5 * np.linalg.norm(g), (a, g)
    assert np.linalg.norm(a - o) <= 1e-5 * np.linalg.norm(o), (a, o)
    # the directional derivative along the seeded direction
    d = np.array(gpu["direction"])
    assert abs(a @ d - ora["directional"]) <= 1e-5 * abs(ora["directional"])


def test_adjoint_gradient_through_saturated_phase_layers():
    """N=128 over 640 steps: the disk interior saturates to phi = 1 - 1e-15, where the
    reverse sweep differentiates psi and the normals with the floors of the adjoint;
    the gradient stays finite and equals the central differences of the CUDA forward
    to 1e-4 relative."""
    N2, T2 = 128, 640 * 0.2 / 128
    res = sens.adjoint_gradient(N2, T2)
    fd = sens.gradient_check(sens.make_evaluator(N2, T2), seed=0)
    a, g = np.array(res["gradient"]), np.array(fd["gradient"])
    assert np.all(np.isfinite(a))
    assert np.linalg.norm(a - g) <= 1e-4 * np.linalg.norm(g), (a, g)
