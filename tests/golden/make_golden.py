"""Regenerate the golden fixtures of tests/golden/ with the FP64 CPU oracle.

    python tests/golden/make_golden.py

Each fixture holds the final state of a few IMEX steps of one small workload
(linear solves converged to 1e-13), produced by the oracle — the CPU restatement
of the reference step.  They pin the oracle against regressions (CPU test) and
give the GPU tests a reference that needs no oracle at run time.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = {
    # name: (workload factory, kwargs, steps, compatible start)
    "cavity_disk_N16_s3": ("cavity_disk", {"N": 16}, 3, False),
    "filament_N16_s2": ("filament_kolmogorov", {"N": 16}, 2, False),
    "channel_growth_N8_s2": ("channel_growth", {"N": 8}, 2, True),
}
FIELDS = ("U", "V", "phi", "resource", "sigma_xx", "sigma_yy", "sigma_xy")


def tight(numerics):
    import dataclasses
    ls = dataclasses.replace(numerics.linear_solvers, velocity_method="gmres", reltol=1e-13, maxiter=2000)
    return dataclasses.replace(numerics, linear_solvers=ls, projection_reltol=1e-13, projection_maxiter=3000)


def build_case(name):
    from eulerianfsi_b200 import workloads
    factory, kw, steps, compatible = CASES[name]
    w = getattr(workloads, factory)(**kw)
    w.numerics = tight(w.numerics)
    return w, steps, compatible


def run_oracle(name):
    from oracle.oracle import Oracle
    w, steps, compatible = build_case(name)
    o = Oracle(w.metrics, w.bcs, w.models, w.numerics)
    st = w.state.copy()
    o.upload(st)
    if compatible:
        o.make_velocity_compatible()
    t = 0.0
    for _ in range(steps):
        o.step(t, w.dt)
        t += w.dt
    o.download(st)
    return w, st


def main():
    for name in CASES:
        w, st = run_oracle(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **{f: getattr(st, f) for f in FIELDS})
        print("wrote", name)


if __name__ == "__main__":
    main()
