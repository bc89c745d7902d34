"""Golden fixtures (tests/golden/make_golden.py): the oracle reproduces them on the
CPU, and the CUDA path matches them on the GPU."""
import ctypes as C
import os

import numpy as np
import pytest

from tests.golden.make_golden import CASES, FIELDS, build_case, run_oracle

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(HERE, name + ".npz"))


def rel(a, b):
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / d if d > 0 else np.linalg.norm(a - b)


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_golden(name):
    g = load(name)
    _, st = run_oracle(name)
    for f in FIELDS:
        assert rel(getattr(st, f), g[f]) <= 1e-12, f


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_matches_golden(name):
    import eulerianfsi_b200 as ef
    g = load(name)
    w, steps, compatible = build_case(name)
    ctx = ef.build_imex_context(w.metrics, w.bcs, w.models, numerics=w.numerics)
    work = ef.allocate_imex_workspace(w.metrics)
    st = w.state.copy()
    if compatible:
        ef.make_velocity_compatible(st, ctx, work)
    t = 0.0
    for _ in range(steps):
        ef.integrate_step(st, t, w.dt, ctx, work)
        t += w.dt
    for f in FIELDS:
        assert rel(getattr(st, f), g[f]) <= 1e-10, (f, rel(getattr(st, f), g[f]))
