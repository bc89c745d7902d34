"""Benchmark of the B200 IMEX fractional step (grid-cell-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 20-disk lid-driven cavity at 1024x1024 (ACDI, dt = 0.2 h), seeded
synthetic initial fields.  A step is one integrate_step! of that grid.  The headline
is the precision form (FP32 solver bulk, FP64 state, residuals, inner products and
refinement); the FP64 step is timed beside it from the same initial state and the
per-field relative L2 difference of the two after W+K steps is reported
(`vs_other_precision`).  `value` is timed with CUDA events on the library's stream
around K device-resident steps (inputs already in HBM); `e2e` repeats the
measurement through the public API: wall-clock time (time.perf_counter, after a
device synchronisation) around every `integrate_step` call with pinned host arrays,
so the host-side validation, the ctypes call and the host<->device copies of the
state are inside the timed region; the device-event time of the same calls is
reported beside it.  The working set (~0.5 GB) exceeds the 126 MB L2 on every step, so no
extra L2 flush is inserted.  Multi-GPU runs are independent replicas (the step is a
global elliptic solve and does not shard); rank 0 prints the aggregate.

`--impl reference` times the FP64 CPU restatement of the reference step (the
oracle; the Julia reference cannot run here) on the host cores for a bounded
sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-cell-steps/s"
UNIT = "cell-steps/s"
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from the ncu
# capture summarised in the named profile; None where no capture exists.
MEASURED_TRAFFIC = {
    ("visc_cg", "fp64"): (147.9e6, "profiles/k_visc_cg_cavity_disks20_N1024.md"),
    ("visc_cg", "mixed"): (26.1e6, "profiles/k_vcheb_cavity_disks20_N1024_mixed.md"),
}


# The kernel behind a timed site per precision form (the 1024^2 cavity has a constant
# viscosity, so the precision form's viscous solve is the Chebyshev kernel).
SITE_KERNELS = {("visc_cg", "fp64"): "k_visc_cg", ("visc_cg", "mixed"): "k_vcheb"}
SITE_NOTES = {("visc_cg", "mixed"): "temporally blocked: an iteration launch performs 4 Chebyshev steps on the "
                                    "tile, so its equivalent per-step rate is 4x `achieved`; issue-bound by design"}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Clock and throttle-reason sampling during the timed region: NVML polled every
    5 ms from a thread of this process (nvidia-smi -lms 200 when NVML is missing).
    Sampling only reads the GPU's state."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm_mhz, reason names) from NVML
        self.max_mhz = 0.0
        self.stop = threading.Event()

    def _open_nvml(self):
        import pynvml as nv
        nv.nvmlInit()
        visible = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v for v in visible.split(",") if v.strip()]
        idx = int(ids[self.gpu]) if ids and ids[self.gpu].strip().isdigit() else self.gpu
        h = nv.nvmlDeviceGetHandleByIndex(idx)
        self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        return nv, h, bits

    def _poll(self, nv, h, bits):
        while not self.stop.is_set():
            try:
                clk = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((clk, tuple(n for n, b in zip(self.NAMES, bits) if r & b)))
            except Exception:
                pass
            self.stop.wait(0.005)

    def __enter__(self):
        try:
            nv, h, bits = self._open_nvml()
            self.nvml = nv
            self.thread = threading.Thread(target=self._poll, args=(nv, h, bits), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], self.max_mhz, set()
        for clk, names in self.samples:
            sm.append(clk)
            reasons.update(names)
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                clk = float(parts[1])
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            sm.append(clk)
            for name, val in zip(self.NAMES, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        busy = [s for s in sm if s > 600] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml, 5 ms" if self.samples else "nvidia-smi, 200 ms"}


def max_over_ranks(value: float, dist, device: str) -> float:
    """The largest `value` over all ranks (every rank gets it); identity without
    a process group.  Device times of replicas are combined this way."""
    if dist is None:
        return value
    import torch
    tt = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def build_workload(args, precision):
    import dataclasses

    from eulerianfsi_b200 import workloads
    w = workloads.cavity_disks20(N=args.N, steps=args.steps, projection_reltol=args.projection_reltol,
                                 velocity_reltol=args.velocity_reltol, precision=precision)
    w.numerics = dataclasses.replace(w.numerics, projection_solver=getattr(args, "projection_solver", "auto"))
    return w


def cpu_sample(args, budget_s, max_steps):
    """Time the FP64 CPU oracle (single thread) on the same workload."""
    from oracle.oracle import Oracle
    w = build_workload(args, "fp64")
    o = Oracle(w.metrics, w.bcs, w.models, w.numerics)
    o.upload(w.state)
    done, t = 0, 0.0
    start = time.perf_counter()
    while done < max_steps:
        o.step(t, w.dt)
        t += w.dt
        done += 1
        if time.perf_counter() - start > budget_s:
            break
    elapsed = time.perf_counter() - start
    return w.cells * done / elapsed, done, elapsed


def _cpu_worker(argv, budget_s, max_steps, out):
    """One single-thread oracle replica (runs in a spawned process)."""
    out.put(cpu_sample(argparse.Namespace(**argv), budget_s, max_steps))


def cpu_replicas(args, budget_s, max_steps, nproc=None):
    """The oracle on every host core: independent single-thread replicas of the same
    sample in spawned processes (the oracle, like the reference, is serial).  Returns
    (aggregate cell-steps/s = sum over replicas, steps done by all, longest replica's
    seconds, replicas)."""
    import multiprocessing as mp
    nproc = nproc or len(os.sched_getaffinity(0))
    if nproc <= 1:
        v, done, el = cpu_sample(args, budget_s, max_steps)
        return v, done, el, 1
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_cpu_worker, args=(vars(args), budget_s, max_steps, q)) for _ in range(nproc)]
    for p_ in procs:
        p_.start()
    import queue
    res = []
    try:
        while len(res) < nproc:
            try:
                res.append(q.get(timeout=5.0))
            except queue.Empty:
                if all(not p_.is_alive() for p_ in procs) and q.empty():
                    raise RuntimeError("an oracle replica of the CPU baseline exited without a result")
    finally:
        for p_ in procs:
            p_.join(timeout=60)
            if p_.is_alive():
                p_.terminate()
    return sum(r[0] for r in res), sum(r[1] for r in res), max(r[2] for r in res), nproc


def run_reference(args, rank):
    if rank != 0:
        return
    max_steps = max(1, args.steps)
    value, done, elapsed, nproc = cpu_replicas(args, budget_s=args.reference_budget, max_steps=max_steps,
                                               nproc=args.cpu_procs)
    sample = (f"{done} IMEX step(s) of the {args.N}x{args.N} 20-disk cavity over {nproc} single-thread "
              f"oracle replicas (one per host thread) in {elapsed:.1f} s")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": done, "warmup": 0, "ms_per_step": 1e3 * elapsed / done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(args, "fp64"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_block(args, precision):
    return {"workload": "cavity_disks20", "Nx": args.N, "Ny": args.N, "disks": 20, "phase_field": "acdi",
            "precision": precision, "projection_reltol": args.projection_reltol,
            "projection_solver": getattr(args, "projection_solver", "auto"),
            "velocity_reltol": args.velocity_reltol,
            "l2": "working set exceeds the 126 MB L2 every step; no extra flush",
            "parallelism": f"replicas{args.gpus}"}


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    import eulerianfsi_b200 as ef
    from eulerianfsi_b200 import _abi

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    nd = max(args.warmup, args.steps, 1)

    def timed(precision, sample_clocks):
        """W untimed then K timed device-resident steps of one precision form."""
        w = build_workload(args, precision)
        ctx = ef.build_imex_context(w.metrics, w.bcs, w.models, numerics=w.numerics)
        h = ctx.handle
        if args.host_driven:
            h.call("set_step_mode", _abi.STEP_HOST)
        h.upload(w.state)
        h.set_correction(np.zeros((args.N, args.N), order="F"))
        dts = (C.c_double * nd)(*([w.dt] * nd))
        t = 0.0
        if args.warmup:
            h.call("step_n", t, dts, int(args.warmup), None)
            t += args.warmup * w.dt
        h.call("set_timed_site", -1)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local_rank) if sample_clocks else None
        if clocks:
            clocks.__enter__()
        h.call("step_n", t, dts, int(args.steps), None)
        torch.cuda.synchronize()
        if clocks:
            clocks.__exit__(None, None, None)
        if dist:
            dist.barrier()
        st = h.stats()
        ms = max_over_ranks(st["device_ms"], dist, "cuda")
        return dict(w=w, ctx=ctx, h=h, dts=dts, t=t + args.steps * w.dt, ms=ms, st=st, clocks=clocks)

    other = "fp64" if args.precision == "mixed" else "mixed"
    ref = None if args.no_compare else timed(other, False)
    run = timed(args.precision, True)
    w, ctx, h, dts, t, ms, st, clocks = (run[k] for k in ("w", "ctx", "h", "dts", "t", "ms", "st", "clocks"))
    launches = st["kernel_launches"]
    value = world * w.cells * args.steps / (ms / 1e3)
    compare = None
    if ref is not None:
        sa, sb = w.state.copy(), ref["w"].state.copy()
        h.download(sa)
        ref["h"].download(sb)
        errs = {}
        for name in ("U", "V", "phi", "sigma_xx", "sigma_yy", "sigma_xy"):
            a, b = getattr(sa, name), getattr(sb, name)
            errs[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
        ref_value = world * w.cells * args.steps / (ref["ms"] / 1e3)
        compare = {"precision": other, "value": ref_value, "ms_per_step": ref["ms"] / args.steps,
                   "speedup": (value / ref_value) if args.precision == "mixed" else (ref_value / value),
                   "rel_l2_after_steps": args.warmup + args.steps, "rel_l2": errs,
                   "max_rel_l2": max(errs.values())}
        ref["ctx"].handle.close()

    # ---- roofline of one kernel: the same steps enqueued from the host with CUDA events
    # around every launch of the site (per-launch events cannot sit inside graph loops)
    peak, peak_kind = _peaks()
    site_steps = max(1, min(args.site_steps, args.steps))
    h.call("set_timed_site", _abi.SITES.index(args.site))
    h.call("step_n", t, dts, site_steps, None)
    t += site_steps * w.dt
    sst = h.stats()
    h.call("set_timed_site", -1)
    site_ms = sst["site_ms"] / max(sst["site_launches"], 1)
    site_bytes = sst["site_bytes"] / max(sst["site_launches"], 1)
    achieved = site_bytes / (site_ms / 1e3) / 1e9 if site_ms > 0 else None
    # step-level roofline: algorithmic bytes of every launch site of one (host-driven,
    # same kernels and iterations) step over the device-timed step
    step_bytes = sst["step_bytes"] / site_steps
    step_achieved = step_bytes / (ms / args.steps / 1e3) / 1e9

    # ---- end to end through the public API with pinned host arrays ----
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, args.e2e_steps))
    pinned = []
    for a in w.state.arrays():
        t_ = torch.empty(a.shape[::-1], dtype=torch.float64).pin_memory()
        arr = t_.numpy().T  # Fortran-ordered view of pinned memory
        arr[...] = a
        pinned.append(arr)
    state = ef.FSIState(*pinned)
    work = ef.allocate_imex_workspace(w.metrics)
    qpin = torch.zeros((args.N, args.N), dtype=torch.float64).pin_memory().numpy().T
    work.correction = qpin  # the warm start travels with the state through integrate_step
    if e2e_steps:
        ef.integrate_step(state, 0.0, w.dt, ctx, work)  # warm the path
    e2e_ms = e2e_dev_ms = 0.0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(e2e_steps):
        t0 = time.perf_counter()
        ef.integrate_step(state, (k + 1) * w.dt, w.dt, ctx, work)  # returns with the state on the host
        e2e_ms += 1e3 * (time.perf_counter() - t0)
        e2e_dev_ms += h.stats()["device_ms"]
    e2e_ms = max_over_ranks(e2e_ms, dist, "cuda")
    e2e_dev_ms = max_over_ranks(e2e_dev_ms, dist, "cuda")
    field_bytes = sum(a.nbytes for a in state.arrays())
    h2d = field_bytes + qpin.nbytes
    d2h = field_bytes + qpin.nbytes
    e2e_value = world * w.cells * e2e_steps / (e2e_ms / 1e3) if e2e_steps else None
    e2e_dev_value = world * w.cells * e2e_steps / (e2e_dev_ms / 1e3) if e2e_steps else None

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-solver-bulk/f64-state-refinement", "data": "synthetic",
        "config": config_block(args, args.precision),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps, "timing": "wall clock around each integrate_step call",
                "ms_per_step": e2e_ms / e2e_steps if e2e_steps else None,
                "device_events": {"value": e2e_dev_value,
                                  "ms_per_step": e2e_dev_ms / e2e_steps if e2e_steps else None}},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": SITE_KERNELS.get((args.site, args.precision), args.site),
                     "site": args.site, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": args.traffic if args.traffic is not None else
                     (MEASURED_TRAFFIC[(args.site, args.precision)][0]
                      if (args.site, args.precision) in MEASURED_TRAFFIC and args.N == 1024 else None),
                     "avg_launch_us": site_ms * 1e3, "algorithmic_bytes_per_launch": site_bytes,
                     "note": SITE_NOTES.get((args.site, args.precision)),
                     "launches_timed": sst["site_launches"], "site_steps": site_steps},
        "step_roofline": {"bound": "hbm", "algorithmic_bytes_per_step": step_bytes,
                          "achieved": step_achieved, "peak": peak, "unit": "GB/s",
                          "frac": step_achieved / peak},
        "clocks": clocks.summary(),
        "vs_other_precision": compare,
        "solver": {"projection_iterations": st["projection_iterations"],
                   "velocity_iterations": st["velocity_iterations"]},
    }
    if world == 1 and not args.no_cpu_baseline:
        v, done, el, nproc = cpu_replicas(args, budget_s=args.cpu_budget, max_steps=args.cpu_steps,
                                          nproc=args.cpu_procs)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nproc, "kind": "port",
                                "sample": f"{done} IMEX step(s) of the {args.N}x{args.N} workload over {nproc} "
                                          f"single-thread oracle replicas (one per host thread), {el:.1f} s"}
    print(json.dumps(line), flush=True)


CONFIGS = {  # the four benchmark configurations: workload builder and steps timed
    "c0_cavity_disk_64": (lambda prec: _wl().cavity_disk(N=64, precision=prec), 50),
    "c1_filament_256": (lambda prec: _wl().filament_kolmogorov(N=256, precision=prec), 50),
    "c2_cavity_disks20_1024": (lambda prec: _wl().cavity_disks20(N=1024, precision=prec), 20),
    "c3_channel_growth_1024x512": (lambda prec: _wl().channel_growth(N=512, precision=prec), 20),
}


def _wl():
    from eulerianfsi_b200 import workloads
    return workloads


def run_configs(args):
    """Per configuration: FP64 and precision-form step time and the per-field
    relative L2 difference of the two after the same steps (one JSON line each)."""
    import numpy as np
    import torch

    import eulerianfsi_b200 as ef
    torch.cuda.set_device(0)
    for name, (make, steps) in CONFIGS.items():
        res = {}
        for prec in ("fp64", "mixed"):
            w = make(prec)
            ctx = ef.build_imex_context(w.metrics, w.bcs, w.models, numerics=w.numerics)
            h = ctx.handle
            st = w.state.copy()
            h.upload(st)
            h.set_correction(np.zeros((w.metrics.Nx, w.metrics.Ny), order="F"))
            if w.needs_compatible_start:
                ef.make_velocity_compatible(st, ctx, ef.allocate_imex_workspace(w.metrics))
                h.upload(st)
            dts = (C.c_double * steps)(*([w.dt] * steps))
            h.call("step_n", 0.0, dts, 3, None)  # warm-up (graph capture, first touches)
            h.call("step_n", 3 * w.dt, dts, steps, None)
            ms = h.stats()["device_ms"] / steps
            out = st.copy()
            h.download(out)
            res[prec] = (ms, out, w.cells)
        errs = {f: float(np.linalg.norm(getattr(res["mixed"][1], f) - getattr(res["fp64"][1], f))
                         / max(np.linalg.norm(getattr(res["fp64"][1], f)), 1e-300))
                for f in ("U", "V", "phi", "resource", "sigma_xx", "sigma_yy", "sigma_xy")}
        cells = res["fp64"][2]
        print(json.dumps({"config": name, "steps": steps, "warmup": 3, "fp64_ms_per_step": res["fp64"][0],
                          "mixed_ms_per_step": res["mixed"][0],
                          "fp64_cell_steps_per_s": cells / (res["fp64"][0] / 1e3),
                          "mixed_cell_steps_per_s": cells / (res["mixed"][0] / 1e3),
                          "speedup": res["fp64"][0] / res["mixed"][0], "rel_l2_mixed_vs_fp64": errs}),
              flush=True)


def run_sensitivity(args, rank, world, dist):
    """Finite-difference sensitivities of the cavity-disk objective (N=256 to T=2 by
    default): one ensemble of forward runs (base, +/- h per parameter, +/- h along a
    seeded direction) spread over the ranks, and the FD gradient's cost in forward
    runs.  Rank 0 prints one JSON line."""
    import time

    import torch

    from eulerianfsi_b200 import sensitivity as sens
    times = []
    ev = sens.make_evaluator(args.sens_N, args.sens_T, timings=times)
    group = dist.group.WORLD if dist else None
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    res = sens.gradient_check(ev, seed=args.sens_seed, group=group)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    dev_ms = float(sum(times))
    if dist:
        wall = max_over_ranks(wall, dist, "cuda")
        dev_ms = max_over_ranks(dev_ms, dist, "cuda")
    if rank:
        return
    forward_ms = times[0]  # run 0 (the base point) always runs on rank 0
    steps = int(round(args.sens_T / (0.2 / args.sens_N)))
    res.update({"config": {"workload": "cavity_disk_sensitivity", "Nx": args.sens_N, "Ny": args.sens_N,
                           "T": args.sens_T, "steps": steps, "dt": 0.2 / args.sens_N, "precision": "fp64",
                           "solver_reltol": sens.FD_RELTOL, "parameters": list(sens.PARAMETERS),
                           "at": list(sens.DEFAULT_PARAMETERS), "seed": args.sens_seed, "rel_h": 1e-6},
                "n_gpus": world, "method": "central differences (discrete adjoint not built)",
                "forward_ms": forward_ms, "forward_cell_steps_per_s": args.sens_N ** 2 * steps / (forward_ms / 1e3),
                "gradient_cost_in_forward_runs": 2 * len(sens.PARAMETERS),
                "ensemble_device_ms_max_over_ranks": dev_ms, "ensemble_wall_s": wall})
    print(json.dumps(res), flush=True)


def run_adjoint(args):
    """Differentiation form on the cavity-disk objective (N=256 to T=2 by default): the
    gradient over (G, lid speed, disk centre x, y) from one checkpointed forward run and
    one reverse sweep, its cost in plain forward runs, and (unless --no-fd) its agreement
    with the central-difference gradient of the same forward (11 runs).  One JSON line."""
    import numpy as np
    import torch

    from eulerianfsi_b200 import sensitivity as sens
    torch.cuda.set_device(0)
    p = sens.DEFAULT_PARAMETERS
    plain = []
    ev = sens.make_evaluator(args.sens_N, args.sens_T, timings=plain)
    J_plain = ev(p)  # one plain forward run (device-resident steps, no checkpoints)
    res = sens.adjoint_gradient(args.sens_N, args.sens_T, p, every=args.adj_every)
    forward_ms = plain[0]
    line = {"metric": "adjoint/forward cost", "value": (res["forward_ms"] + res["backward_ms"]) / forward_ms,
            "unit": "forward runs per gradient", "higher_is_better": False,
            "config": {"workload": "cavity_disk_sensitivity", "Nx": args.sens_N, "Ny": args.sens_N,
                       "T": args.sens_T, "steps": res["steps"], "dt": 0.2 / args.sens_N, "precision": "fp64",
                       "solver_reltol": sens.FD_RELTOL, "parameters": list(sens.PARAMETERS), "at": list(p),
                       "checkpoint_every": args.adj_every or int(np.ceil(np.sqrt(res["steps"])))},
            "J": res["J"], "J_plain_forward": J_plain, "gradient": res["gradient"],
            "plain_forward_ms": forward_ms, "checkpointed_forward_ms": res["forward_ms"],
            "backward_ms": res["backward_ms"], "dtype": "f64", "data": "synthetic"}
    if not args.no_fd:
        fds = []
        for rel_h in args.fd_rel_h:
            fd = sens.gradient_check(ev, p, seed=args.sens_seed, rel_h=rel_h)
            g, a = np.array(fd["gradient"]), np.array(res["gradient"])
            d = np.array(fd["direction"])
            fds.append({
                "rel_h": rel_h, "gradient": fd["gradient"],
                "rel_l2_adjoint_vs_fd": float(np.linalg.norm(a - g) / np.linalg.norm(g)),
                "directional_fd": fd["directional"], "directional_adjoint": float(a @ d),
                "rel_diff_directional": abs(float(a @ d) - fd["directional"]) / abs(fd["directional"]),
                "fd_self_consistency": fd["rel_diff"], "runs": fd["runs"]})
        line["finite_differences"] = fds
    print(json.dumps(line), flush=True)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--N", type=int, default=1024)
    p.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                   help="headline precision form; the other form is timed beside it")
    p.add_argument("--no-compare", action="store_true", help="skip the other precision form")
    p.add_argument("--projection-reltol", type=float, default=1e-10)
    p.add_argument("--velocity-reltol", type=float, default=1e-8)
    p.add_argument("--projection-solver", default="auto", choices=["auto", "multigrid"],
                   help="auto: direct fast-diagonalisation solve where the grid allows it")
    p.add_argument("--site", default="visc_cg")
    p.add_argument("--traffic", type=float, default=None, help="ncu dram bytes per launch of the site")
    p.add_argument("--site-steps", type=int, default=3)
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--cpu-steps", type=int, default=1)
    p.add_argument("--cpu-budget", type=float, default=60.0)
    p.add_argument("--reference-budget", type=float, default=150.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-procs", type=int, default=None,
                   help="oracle replicas for the CPU baseline and the reference arm (default: one per host thread)")
    p.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    p.add_argument("--host-driven", action="store_true",
                   help="enqueue every kernel from the host instead of the captured step graph (launch lists)")
    p.add_argument("--configs", action="store_true",
                   help="FP64 vs precision form on the four benchmark configurations (1 GPU)")
    p.add_argument("--sensitivity", action="store_true",
                   help="finite-difference sensitivities of the cavity-disk objective, runs spread over ranks")
    p.add_argument("--sens-N", type=int, default=256)
    p.add_argument("--sens-T", type=float, default=2.0)
    p.add_argument("--sens-seed", type=int, default=0)
    p.add_argument("--adjoint", action="store_true",
                   help="discrete-adjoint gradient of the cavity-disk objective and its cost in forward runs")
    p.add_argument("--adj-every", type=int, default=0, help="checkpoint spacing (0: ceil(sqrt(steps)))")
    p.add_argument("--no-fd", action="store_true", help="skip the finite-difference comparison of --adjoint")
    p.add_argument("--fd-rel-h", type=float, nargs="+", default=[1e-6],
                   help="relative steps of the finite differences --adjoint compares against")
    args = p.parse_args()
    if args.configs:
        run_configs(args)
        return
    if args.adjoint:
        run_adjoint(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            run_reference(args, rank)
        elif args.sensitivity:
            import torch
            torch.cuda.set_device(local_rank)
            import torch.distributed as dist
            run_sensitivity(args, rank, world, dist if world > 1 else None)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
