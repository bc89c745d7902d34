"""Generate the full-length oracle fixture of the filament configuration:

    python tests/golden/make_fulllength.py            # about 10 minutes on one core

The wall-supported filament in Kolmogorov flow at 256 x 256 (UWCDI phase field,
run_wall_supported_filament_kolmogorov_flow.jl's benchmark configuration) run for its
full 1000 steps by the FP64 CPU oracle with every linear solve converged to 1e-13; the
final state is stored (compressed) as filament_N256_s1000.npz.  The GPU test
tests/test_gpu_fulllength.py compares the CUDA step against it at 1e-8 relative L2.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NAME = "filament_N256_s1000"
FIELDS = ("U", "V", "phi", "resource", "sigma_xx", "sigma_yy", "sigma_xy")


def workload():
    from eulerianfsi_b200 import workloads
    from tests.golden.make_golden import tight
    w = workloads.filament_kolmogorov(N=256, steps=1000)
    w.numerics = tight(w.numerics)
    return w


def main(steps=None):
    from oracle.oracle import Oracle
    w = workload()
    steps = w.steps if steps is None else steps
    o = Oracle(w.metrics, w.bcs, w.models, w.numerics)
    st = w.state.copy()
    o.upload(st)
    o.handle.set_correction(np.zeros((w.metrics.Nx, w.metrics.Ny), order="F"))
    t0 = time.perf_counter()
    for k in range(steps):
        o.step(k * w.dt, w.dt)
        if k % 100 == 0:
            print(f"step {k} {time.perf_counter() - t0:.1f} s", flush=True)
    o.download(st)
    if steps == w.steps:
        np.savez_compressed(os.path.join(HERE, NAME + ".npz"), steps=steps, dt=w.dt,
                            **{f: getattr(st, f) for f in FIELDS})
    return st


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else None)
