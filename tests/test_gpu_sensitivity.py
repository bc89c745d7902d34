"""Finite-difference sensitivities of the cavity-disk objective through the CUDA
library against the same differences through the FP64 oracle (N=32, 40 steps):
the gradient over (G, lid speed, disk centre x, y) and the directional derivative
along a seeded direction agree to 1e-5 relative."""
import numpy as np
import pytest

from eulerianfsi_b200 import sensitivity as sens
from tests.gpu_util import oracle_final_state

pytestmark = pytest.mark.gpu

N, STEPS = 32, 40
TOL = 1e-5


def test_gpu_finite_differences_match_oracle():
    T = STEPS * 0.2 / N
    gpu = sens.gradient_check(sens.make_evaluator(N, T), seed=0)
    ora = sens.gradient_check(sens.make_evaluator(N, T, run=oracle_final_state), seed=0)
    assert abs(gpu["J"] - ora["J"]) <= 1e-10 * abs(ora["J"])
    g, o = np.array(gpu["gradient"]), np.array(ora["gradient"])
    assert np.linalg.norm(g - o) <= TOL * np.linalg.norm(o), (g, o)
    assert abs(gpu["directional"] - ora["directional"]) <= TOL * abs(ora["directional"])
    assert gpu["rel_diff"] <= TOL
