"""Helpers of the GPU parity tests: one CUDA handle and one oracle handle built
from the same configuration, and random inputs consistent with the boundaries."""
import ctypes as C

import numpy as np

import eulerianfsi_b200 as ef
from eulerianfsi_b200 import _abi
from eulerianfsi_b200.imex import ConfigBlock, Handle
from oracle.oracle import Oracle, load as load_oracle


def pair(metrics, bcs, models, numerics):
    """(gpu_handle, oracle_handle) for one configuration."""
    block = ConfigBlock(metrics, bcs, models, numerics)
    gpu = Handle(_abi.load_library(), "efsi_", block, metrics)
    ora = Handle(load_oracle(), "oracle_", ConfigBlock(metrics, bcs, models, numerics), metrics)
    return gpu, ora


def rel_err(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / den if den > 1e-300 else np.linalg.norm(a - b)


def random_inputs(metrics, seed=0, amp=0.3):
    rng = np.random.default_rng(seed)
    Nx, Ny = metrics.Nx, metrics.Ny
    x = (np.arange(Nx) + 0.5) / Nx
    y = (np.arange(Ny) + 0.5) / Ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    phi = 0.5 + 0.45 * np.tanh(4 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)) + 0.01 * rng.standard_normal((Nx, Ny))
    U = amp * rng.standard_normal((Nx + 1, Ny))
    V = amp * rng.standard_normal((Nx, Ny + 1))
    sxx = 1.0 + 0.2 * rng.random((Nx, Ny))
    syy = 1.0 + 0.2 * rng.random((Nx, Ny))
    sxy = 0.05 * rng.standard_normal((Nx, Ny))
    G = 0.1 * rng.standard_normal((Nx, Ny))
    c = 0.5 + 0.4 * rng.random((Nx, Ny))
    f = lambda a: np.asfortranarray(a, dtype=np.float64)
    return {k: f(v) for k, v in dict(U=U, V=V, phi=phi, sxx=sxx, syy=syy, sxy=sxy, G=G, c=c).items()}


def call_both(gpu, ora, name, *args_factory):
    """Run entry `name` on both handles; args_factory returns fresh argument tuples."""
    outs = []
    for h in (gpu, ora):
        args, keep = args_factory()
        h.call(name, *args)
        outs.append(keep)
    return outs


def oracle_final_state(w):
    """Run workload `w` for w.steps oracle steps from its initial state; the final state."""
    from tests.helpers import fz
    h = Handle(load_oracle(), "oracle_", ConfigBlock(w.metrics, w.bcs, w.models, w.numerics), w.metrics)
    state = w.state.copy()
    h.upload(state)
    h.set_correction(fz(w.metrics.Nx, w.metrics.Ny))
    t = 0.0
    for _ in range(w.steps):
        rep = _abi.StepReportC()
        h.call("integrate_step", t, w.dt, C.byref(rep))
        t += w.dt
    h.download(state)
    h.close()
    return state
