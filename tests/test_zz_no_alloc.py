"""efsi_divergence_residual_noalloc: the entry point for callers that cannot let a
library allocate device memory (hosts whose pool allocator owns all GPU memory, or
loops that must not meet the synchronisation cudaMalloc/cudaFree may cause).

It works on caller-owned device arrays and keeps its reduction scratch in a fixed
static device array.  The test checks it against the projection entry point
(efsi_project reports max |div v - G| of the velocity it returns) on two calls in a
row, so the second call runs on scratch the first one left behind.  The file name
makes pytest collect it last."""
import ctypes as C

import numpy as np
import pytest

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import _abi, workloads
from eulerianfsi_b200.imex import ConfigBlock, Handle
from tests.gpu_util import random_inputs
from tests.helpers import dp, fz

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, as the operator parity tests


def _scale(metrics, U, V):
    """Size of the terms whose difference is the divergence (rounding reference)."""
    return np.max(np.abs(U)) * metrics.Nx / metrics.Lx + np.max(np.abs(V)) * metrics.Ny / metrics.Ly


def _projected(case):
    """Velocity returned by efsi_project and the constraint it reports."""
    if case == "cavity":
        w = workloads.cavity_disk(N=48)
        metrics, bcs, models, numerics = w.metrics, w.bcs, w.models, w.numerics
    else:
        grid = ef.generate_grid(1.0, 1.0, 40, 40)
        metrics = ef.build_mesh_metrics(grid)
        d0, n0 = ef.Dirichlet(0.0), ef.Neumann(0.0)
        bq = ef.BoundaryConditionSetup(d0, d0, d0, d0)
        nb = ef.BoundaryConditionSetup(n0, n0, n0, n0)
        bcs = ef.FSIBoundaryConditions(nb, nb, bq, nb, {"xx": nb, "yy": nb, "xy": nb})
        models, numerics = ef.FSIModels(), ef.IMEXNumerics(projection_reltol=1e-12)
    h = Handle(_abi.load_library(), "efsi_", ConfigBlock(metrics, bcs, models, numerics), metrics)
    inp = random_inputs(metrics, seed=7)
    Nx, Ny = metrics.Nx, metrics.Ny
    G = inp["G"] if case == "dirichlet" else None
    U, V = inp["U"].copy(order="F"), inp["V"].copy(order="F")
    if case == "cavity":  # compatible data: no boundary flux, zero target
        U[0, :] = U[-1, :] = 0.0
        V[:, 0] = V[:, -1] = 0.0
    h.set_correction(fz(Nx, Ny))
    r = _abi.ProjectionResultC()
    h.call("project", dp(U), dp(V), dp(G) if G is not None else None, C.byref(r))
    h.close()
    return metrics, U, V, G, r.constraint_linf


def _device(a, torch):
    return torch.from_numpy(np.ravel(a, order="F").copy()).to("cuda")


def _noalloc(lib, torch, metrics, U, V, G):
    dU, dV = _device(U, torch), _device(V, torch)
    dG = _device(G, torch) if G is not None else None
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.efsi_divergence_residual_noalloc(metrics.Nx, metrics.Ny, metrics.Lx, metrics.Ly, dU.data_ptr(),
                                              dV.data_ptr(), dG.data_ptr() if dG is not None else None,
                                              out.data_ptr(), stream)
    assert st == _abi.OK, lib.efsi_last_error(None)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_divergence_residual_matches_projection_report():
    torch = pytest.importorskip("torch")
    lib = _abi.load_library()
    for case in ("cavity", "dirichlet"):  # two calls in a row on the shared scratch
        metrics, U, V, G, reported = _projected(case)
        got = _noalloc(lib, torch, metrics, U, V, G)
        assert abs(got[0] - reported) <= TOL * _scale(metrics, U, V), (case, got[0], reported)
        gmax = float(np.max(np.abs(G))) if G is not None else 0.0
        assert got[1] == gmax
        # and a velocity that is far from the constraint: the unprojected field
        inp = random_inputs(metrics, seed=11)
        hx, hy = metrics.Lx / metrics.Nx, metrics.Ly / metrics.Ny
        div = (inp["U"][1:, :] - inp["U"][:-1, :]) * (1.0 / hx) + (inp["V"][:, 1:] - inp["V"][:, :-1]) * (1.0 / hy)
        want = float(np.max(np.abs(div - (G if G is not None else 0.0))))
        got2 = _noalloc(lib, torch, metrics, inp["U"], inp["V"], G)
        assert abs(got2[0] - want) <= TOL * _scale(metrics, inp["U"], inp["V"])


def test_noalloc_rejects_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = _abi.load_library()
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    st = lib.efsi_divergence_residual_noalloc(4096, 4096, 1.0, 1.0, buf.data_ptr(), buf.data_ptr(), None,
                                              buf.data_ptr(), None)
    assert st == _abi.ARG
    assert b"fixed scratch" in lib.efsi_last_error(None)


def test_noalloc_reports_non_finite_fields():
    """A NaN or Inf in the velocity or the target never yields a finite residual (a
    plain max reduction would drop a NaN and report the rest of the grid)."""
    torch = pytest.importorskip("torch")
    lib = _abi.load_library()
    metrics, U, V, G, _ = _projected("dirichlet")
    bad_U = U.copy(order="F")
    bad_U[5, 7] = np.nan
    got = _noalloc(lib, torch, metrics, bad_U, V, G)
    assert not np.isfinite(got[0]) and np.isfinite(got[1])
    bad_G = G.copy(order="F")
    bad_G[3, 2] = np.inf
    got = _noalloc(lib, torch, metrics, U, V, bad_G)
    assert not np.isfinite(got[0]) and not np.isfinite(got[1])
    # the same shared scratch still gives the finite answer afterwards
    got = _noalloc(lib, torch, metrics, U, V, G)
    assert np.isfinite(got[0]) and got[1] == float(np.max(np.abs(G)))
