"""The multi-GPU path of bench.py on CPU: world_size-2 gloo ranks.  The step does
not shard (replicas only), so the only cross-rank operations are the barrier and the
max-over-ranks of the device times; the reference arm runs on rank 0 alone."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        local = [3.5, 7.25][rank]
        out[rank] = bench.max_over_ranks(local, dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        assert dict(out) == {0: 7.25, 1: 7.25}


def test_max_over_ranks_without_group_is_identity():
    assert bench.max_over_ranks(4.0, None, "cpu") == 4.0


def test_reference_arm_runs_on_rank_zero_only(capsys):
    class A:  # any attribute access would fail: rank 1 must return before reading args
        def __getattr__(self, name):
            raise AssertionError(name)
    bench.run_reference(A(), rank=1)
    assert capsys.readouterr().out == ""


def test_clock_summary_reports_median_under_load_and_reasons():
    s = bench.ClockSampler(0)
    s.max_mhz = 1965.0
    s.samples = [(345.0, ()), (1965.0, ()), (1950.0, ("sw_power_cap",)), (1965.0, ())]
    out = s.summary()
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"] and out["samples"] == 4


def test_cpu_baseline_replicas_aggregate_over_processes():
    """The CPU baseline runs one single-thread oracle replica per process and sums
    their throughput."""
    import argparse
    a = argparse.Namespace(N=128, projection_reltol=1e-10, velocity_reltol=1e-8, steps=1)
    v, done, el, n = bench.cpu_replicas(a, budget_s=2.0, max_steps=2, nproc=2)
    assert n == 2 and done == 4 and v > 0.0 and el > 0.0
