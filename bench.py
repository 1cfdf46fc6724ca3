# SPDX-License-Identifier: 0BSD
"""Benchmark of the FP64 z-averaged heat step on B200.

Workload (one GPU): 8192 x 8192 nodes, dx = 5 um, k = 20 W/m/K, rho = 7900,
cp = 500, 50 um layer, absorptivity 0.4, 200 W, r0 = 50 um, dt = 0.2 dx^2/alpha,
bidirectional raster (100 um hatch, 1 m/s, 10 tracks over 20000 steps), mirror
edges, reference loss terms, uniform 300 K start.  One bench step = 1000 time
steps of the plan (the plan continues across bench steps; 20 bench steps = the
full 20000-step run).  Metric: GCell-updates/s (cells x time steps / second).

Arms:
  --impl b200       (default) liblpbf_b200 through its C-ABI; `value` is timed
                    with the fields resident in HBM, `e2e` through the public
                    call on pinned host buffers (field in, field + per-step
                    Partials out, every bench step).
  --impl reference  the reference's own CPU step task (StepTileTask, compiled
                    from the reference sources into oracle/_ref and driven by
                    the hh-compat graph over ny/64 row strips on all host
                    threads), on a bounded prefix of the same workload.

Multi-GPU (torchrun): every rank advances its own independent 8192^2 field
(raster angle differs by rank); no data-path collective; weak scaling.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SIDE = 8192                  # grid side (--side for a smaller profiling case)
N_STEPS_TOTAL = 20000
STEPS_PER_ITER = 1000          # time steps per bench step (--iter-steps)
BYTES_PER_UPDATE = 16          # read T (8 B) + write T (8 B) per cell-update


def workload(rank: int = 0):
    from hedgehog_lpbf_b200 import params as P
    from hedgehog_lpbf_b200 import plan as PL
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(N_SIDE)
    dt = P.dt_fraction(mat, dom)
    k = P.make_const(mat, pr, dom, dt)
    angle = np.deg2rad(15.0 * rank)
    plan = PL.raster_for_steps(dom, dt, N_STEPS_TOTAL, V=1.0, hatch=100e-6, n_tracks=10,
                               angle=angle)
    return mat, pr, dom, k, plan


def plan_slice(plan, i):
    idx = (np.arange(STEPS_PER_ITER) + i * STEPS_PER_ITER) % len(plan)
    return plan[idx]


def config(depth, n_gpus):
    return {"workload": f"{N_SIDE}x{N_SIDE} FP64 z-averaged heat step, bidirectional raster "
                        "(100 um hatch, 1 m/s, 10 tracks / 20000 steps), dx 5 um, mirror edges",
            "grid": [N_SIDE, N_SIDE], "time_steps_per_bench_step": STEPS_PER_ITER,
            "temporal_depth": depth, "parallelism": f"independent fields x{n_gpus}",
            "l2": "inputs larger than L2 (two 537 MB f64 fields per GPU)"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (no MEASURED_PEAKS.json: earlier copy-bandwidth measurement on B200)"


# ncu counters of the dominant kernel, summarised with the commands that
# produced them in profiles/advance_kernel_8192.md: DRAM bytes read +
# written per full-size launch (8192^2, depth 3, two consecutive launches of
# the bench's own command with --cache-control none, so a launch also pays
# the write-back of the previous launch's dirty lines: the steady state),
# and the FP64 pipe's share of active cycles (4096^2 --set full capture of
# the same kernel).
ADVANCE_PROFILE = {
    3: {"dram_bytes": 1.13944e9, "dram_read_bytes": 0.60274e9, "dram_write_bytes": 0.53670e9,
        "fp64_pipe": 0.539, "issue_active": 0.495, "limiter": "fp64_pipe_latency",
        "source": "profiles/advance_kernel_8192.md"},
}


class ClockSampler:
    """Samples SM clocks and clock-event reasons through NVML every 100 ms."""

    REASONS = {
        "gpu_idle": 0x1, "applications_clocks_setting": 0x2, "sw_power_cap": 0x4,
        "hw_slowdown": 0x8, "sync_boost": 0x10, "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80,
        "display_clock_setting": 0x100,
    }

    def __init__(self, index: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None
        self.t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(0.1)

    def __enter__(self):
        if self.nv:
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.nv and self.t.is_alive():
            self.t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons - {"gpu_idle"}), "samples": len(self.samples)}


def cpu_reference_rate(mat, pr, dom, k, plan, budget_s: float, threads: int | None = None):
    """GCell-updates/s of the reference CPU path on a bounded prefix."""
    from oracle import oracle as O
    from hedgehog_lpbf_b200 import plan as PL
    las = PL.laser_array(plan)
    n_threads = threads or os.cpu_count() or 1
    T = np.full(dom.nx * dom.ny, pr.Tamb)
    if O.have_reference():
        kind = "reference"
        _, w1, _ = O.ref_hh_run(T, mat, pr, dom, k.dt, las[:1], n_threads, dom.ny // 64, Tm=mat.Tm)
        n = int(max(1, min(len(las) - 1, budget_s / max(w1, 1e-3))))
        T, wall, _ = O.ref_hh_run(T, mat, pr, dom, k.dt, las[1:1 + n], n_threads, dom.ny // 64,
                                  Tm=mat.Tm)
        cores = n_threads
        desc = (f"reference StepTileTask (hh-compat graph, {dom.ny // 64} row strips, "
                f"{n_threads} threads) + its per-step driver work, {n} steps of {dom.nx}x{dom.ny}")
    else:
        kind = "port"
        t0 = time.perf_counter()
        O.run(T, k, las[:1], Tm=mat.Tm, with_ring=False)
        w1 = time.perf_counter() - t0
        n = int(max(1, min(len(las) - 1, budget_s / max(w1, 1e-3))))
        t0 = time.perf_counter()
        O.run(T, k, las[1:1 + n], Tm=mat.Tm)
        wall = time.perf_counter() - t0
        cores = 1
        desc = f"oracle C port (single thread), {n} steps of {dom.nx}x{dom.ny}"
    rate = dom.nx * dom.ny * n / wall / 1e9
    return {"value": rate, "unit": "GCell-updates/s", "cores": cores, "kind": kind,
            "sample": desc, "wall_s": wall}


def cpu_single_thread_rate(mat, pr, dom, k, budget_s: float):
    """The reference's single-thread CPU solver, run_cpu (src/gpu/lpbf_cuda.cu:
    423-448: cpu_step plus measure_host every step), on the same grid and
    constants.  It follows its built-in single-track law rather than the
    raster; its per-step work does not depend on the laser's path (the
    source is evaluated at every cell)."""
    from oracle import oracle as O
    if not O.have_reference():
        return None
    w1 = O.ref_run_cpu(mat, pr, dom, k.dt, 1)["wall_ms"] * 1e-3
    n = int(max(1, budget_s / max(w1, 1e-3)))
    wall = O.ref_run_cpu(mat, pr, dom, k.dt, n)["wall_ms"] * 1e-3
    return {"value": dom.nx * dom.ny * n / wall / 1e9, "unit": "GCell-updates/s", "cores": 1,
            "kind": "reference", "wall_s": wall,
            "sample": f"reference run_cpu (single thread, its single-track law), {n} steps of "
                      f"{dom.nx}x{dom.ny}"}


def reference_gpu_rate(timeout_s: float = 600.0):
    """reference_gpu_child() in a child process on the same GPU: the
    reference's task aborts its process on a CUDA error, which must not end
    the bench.  Returns its result, or a record of why there is none."""
    import subprocess
    try:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-gpu-child",
                            "--side", str(N_SIDE)], capture_output=True, text=True,
                           timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"reference GPU task graph exceeded {timeout_s:.0f} s"}
    for ln in r.stdout.splitlines()[::-1]:
        if ln.startswith("{"):
            return json.loads(ln)
    tail = (r.stderr or r.stdout).strip().splitlines()[-1:] or [""]
    return {"unavailable": f"reference GPU task graph exited {r.returncode}: {tail[0][:200]}"}


def reference_gpu_child():
    """The reference's own GPU path on this GPU: its GpuStepTask graph
    (include/gpu_step_task.hpp, run as run_one_row does, hh_gpu_main.cpp:171-
    207) with its kernels (src/gpu/kernels.cu built for sm_100a), default
    options (mode 2, batch 64, unfused, pageable staging) and with the fused
    step+reduce kernel, over the bench's raster plan.  Steady-state rate from
    two run lengths (the task's device set-up cancels in the difference);
    the fused form finalizes 262,144 per-block partials on one thread per
    step (34 ms), so it is sampled over fewer steps."""
    from oracle import oracle as O
    mat, pr, dom, k, plan = workload(0)
    if not O.have_reference():
        return {"unavailable": "oracle/_ref (the reference built from its sources) is absent"}
    out = {"unit": "GCell-updates/s", "kind": "reference",
           "what": "reference GpuStepTask graph (mode 2, batch 64) with its own kernels "
                   f"(kernels.cu built for sm_100a), wall clock, {dom.nx}x{dom.ny} on the "
                   "bench's raster"}
    with ClockSampler(0) as clk:
        for name, fused, n1, n2 in (("unfused", False, 192, 1216), ("fused", True, 64, 192)):
            O.ref_gpu_task_run(k, dom, plan[:64], mat.Tm, pr.Tamb, fused=fused)     # warm-up
            t1, _ = O.ref_gpu_task_run(k, dom, plan[:n1], mat.Tm, pr.Tamb, fused=fused)
            t2, pk = O.ref_gpu_task_run(k, dom, plan[:n2], mat.Tm, pr.Tamb, fused=fused)
            out[name] = {"value": dom.nx * dom.ny * (n2 - n1) / ((t2 - t1) * 1e-3) / 1e9,
                         "ms_per_step": (t2 - t1) / (n2 - n1), "peak_T_K": pk,
                         "steps": f"{n2} - {n1}"}
    out["value"] = max(out["unfused"]["value"], out["fused"]["value"])
    out["clocks"] = clk.summary()
    return out


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    mat, pr, dom, k, plan = workload(0)
    per_step = []
    for _ in range(args.warmup):
        cpu_reference_rate(mat, pr, dom, k, plan, budget_s=1.0)
    for _ in range(args.steps):
        per_step.append(cpu_reference_rate(mat, pr, dom, k, plan, budget_s=args.ref_budget))
    rate = statistics.median(r["value"] for r in per_step)
    cb = dict(per_step[-1])
    cb["value"] = rate
    wall = sum(r["wall_s"] for r in per_step)
    line = {"metric": "GCell-updates/s", "value": rate, "unit": "GCell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * wall / max(1, len(per_step)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": config(None, args.gpus), "cpu_baseline": cb,
            "e2e": {"value": rate, "unit": "GCell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    st = cpu_single_thread_rate(mat, pr, dom, k, budget_s=args.ref_budget)
    if st:
        cb["single_thread_run_cpu"] = st
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu and N_SIDE == 8192 and not args.no_ref_gpu:
        # beside the CPU figure: the reference's own GPU task graph on this GPU
        line["ref_gpu"] = reference_gpu_rate()
    print(json.dumps(line), flush=True)


def process_map_leg(args, dev, rank=0, world=1):
    """The batched process map: seeded scenarios (grid side 256..2048, power,
    speed, spot radius, raster angle and hatch drawn per scenario) advanced
    together through one CUDA graph of the persistent batch kernel, with
    autotuned tiles; one scenario per size class is checked bit for bit
    against its own single-field run, which is also timed (serial).  With
    several ranks the scenarios are dealt round-robin (no data exchange);
    the value is all scenarios' updates over the slowest rank's time."""
    import torch
    from hedgehog_lpbf_b200 import process_map as PM
    from hedgehog_lpbf_b200.batch import Batch, autotune, opts_dict
    from hedgehog_lpbf_b200.ranks import shard, throughput
    from hedgehog_lpbf_b200.solver import Solver, ring_to_numpy
    torch.cuda.empty_cache()
    n_scen, n_steps = args.pm_scenarios, args.pm_steps
    mine = shard(n_scen, rank, world)
    scs = [PM.process_map(1, n_steps, first_index=i)[0] for i in mine]
    t0 = time.time()
    opts = autotune(scs, n_steps, cache=args.tune_cache, trial_steps=12, device=dev)
    tune_s = time.time() - t0
    b = Batch(scs, n_steps, opts=opts, device=dev)
    b.capture(0, n_steps)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record()
        b.run(0, n_steps, use_graph=True)
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cells = b.cells()
    err = b.read_error()
    rate, ms_max = throughput(cells * n_steps, ms, device=dev)
    checks, serial_ms, serial_cells = [], 0.0, 0
    for cls in range(4):
        idx = [i for i, sc in enumerate(scs)
               if b.lib.lpbf_b200_batch_size_class(sc.k.nx, sc.k.ny) == cls]
        if not idx:
            continue
        i = idx[0]
        sc = scs[i]
        s = Solver(sc.k, bc=sc.bc, T_edge=sc.T_edge, Tm=sc.Tm, device=dev, T0=sc.k.Tamb)
        ring = s.new_ring(n_steps)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record()
        s.advance(sc.plan, ring)
        f1.record()
        torch.cuda.synchronize()
        serial_ms += f0.elapsed_time(f1)
        serial_cells += sc.k.nx * sc.k.ny
        same = (torch.equal(s.field.view(torch.int64), b.field(i).view(torch.int64)) and
                ring_to_numpy(ring).tobytes() == b.ring(i)[:n_steps].tobytes())
        checks.append({"scenario": mine[i], "side": sc.k.nx, "bit_identical": bool(same)})
        del s, ring
    out = {"value": rate / 1e9, "unit": "GCell-updates/s", "ranks": world,
           "scaling": "strong (scenarios dealt across ranks)",
           "workload": f"{n_scen} seeded scenarios (side 256/512/1024/2048, P 100-400 W, "
                       f"V 0.5-2 m/s, r0 35-70 um, raster angle 0-pi, hatch 80-120 um), "
                       f"{n_steps} steps each, FP64, uniform 300 K start",
           "scenarios": n_scen, "steps": n_steps, "cells_rank0": cells, "ms": ms_max,
           "launches": b.launches(n_steps), "tasks_per_launch": b.tasks(),
           "tuned": opts_dict(opts), "tune_s": tune_s, "graph": True,
           "bit_identical_to_single_runs": checks,
           "serial_single_field": {"value": serial_cells * n_steps / (serial_ms * 1e-3) / 1e9,
                                   "unit": "GCell-updates/s",
                                   "scenarios": [c["scenario"] for c in checks]},
           "clocks": clk.summary(), "error_word": err}
    b.close()
    return out


def dropin_leg(args, dev):
    """The reference's per-step call sequence (its GpuStepTask batch loop:
    step, reduce, finalize, hot-column extract, one ring copy and one sync
    per 64 steps) over this library's drop-in C-ABI, on the bench field and
    raster: what a reference build gets by linking this library in place of
    its kernels.  Unfused and fused forms, 64 warm-up steps, then the timed
    ones."""
    import torch
    from hedgehog_lpbf_b200 import dropin
    mat, pr, dom, k, plan = workload(0)
    n = args.dropin_steps
    out = {"unit": "GCell-updates/s",
           "what": "reference GpuStepTask call sequence (mode 2, batch 64) over this "
                   "library's lpbf_launch_* entry points, CUDA events"}
    for name, fused in (("unfused", False), ("fused", True)):
        dropin.run(k, dom, plan[:64], mat.Tm, fused=fused, device=dev)
        r = dropin.run(k, dom, plan[64:64 + n], mat.Tm, fused=fused, device=dev)
        out[name] = {"value": r["gcell_updates_per_s"], "ms_per_step": r["ms_per_step"],
                     "steps": n, "extract_col": r["extract_col"]}
        del r
        torch.cuda.empty_cache()
    out["value"] = max(out["unfused"]["value"], out["fused"]["value"])
    return out


def ext_leg(args, dev):
    """Extended physics (phys = 1: Mills k(T), cp(T) with latent heat, the
    reference's StepTileTask extended branch) on the 8192^2 field: the
    bench's raster at dt = 0.1 dx^2/alpha (half the baseline step: the
    conductivity reaches 1.5x the baseline's), one step per launch,
    per-step Partials, fields resident in HBM."""
    import torch
    from hedgehog_lpbf_b200 import params as P
    from hedgehog_lpbf_b200 import plan as PL
    from hedgehog_lpbf_b200.solver import Solver
    torch.cuda.empty_cache()
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(N_SIDE)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom, 0.1))
    n = args.ext_steps
    plan = PL.raster_for_steps(dom, k.dt, 2 * N_STEPS_TOTAL, V=1.0, hatch=100e-6, n_tracks=10)
    s = Solver(k, phys=1, device=dev, Tm=mat.Tm)
    ring = s.new_ring(n)
    s.advance(plan[:n], ring)                       # warm-up: the laser's first n steps
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record()
        s.advance(plan[n:2 * n], ring)
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    peak, _ = measured_peaks()
    cells = dom.nx * dom.ny
    out = {"value": cells * n / (ms * 1e-3) / 1e9, "unit": "GCell-updates/s",
           "time_steps": n, "launches": s.launches(n), "ms": ms, "kmult": k.kmult,
           "dt_s": k.dt, "kernel": "ext_step_kernel (one step per launch, fused reduction)",
           "roofline": {"bound": "hbm", "achieved": BYTES_PER_UPDATE * cells * n / (ms * 1e-3) / 1e9,
                        "peak": peak, "unit": "GB/s"},
           "clocks": clk.summary(), "error_word": s.read_error()}
    out["roofline"]["frac"] = out["roofline"]["achieved"] / peak
    del s, ring
    return out


FLOP_PER_PIXEL = 2 * 9 * (4 * 32 + 3 * 32 * 32 + 32 * 1)   # one forward of the super-stepper


def superstep_leg(args, dev):
    """The learned super-stepper (committed weights trained by this library's
    own tcgen05 kernels): forward throughput on the 4096^2 field, training
    step throughput (batch 32 of 256^2 patches), and the hybrid run with the
    FP64 judge and rollback on the 4096^2 raster (20 tracks, 100 um hatch,
    1 m/s) over a prefix of its 200,000 steps, against plain FP64 on the
    same prefix."""
    import torch
    from hedgehog_lpbf_b200 import params as P
    from hedgehog_lpbf_b200 import plan as PL
    from hedgehog_lpbf_b200.solver import Solver
    from hedgehog_lpbf_b200.superstep import WEIGHTS, load, run_hybrid
    from hedgehog_lpbf_b200.surrogate import STEPS, Net, features, init_params
    torch.cuda.empty_cache()
    if os.path.exists(WEIGHTS):
        net, rec = load(WEIGHTS, device=dev)
    else:
        net, rec = Net(init_params(0), device=dev), None
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(4096)
    dt = P.dt_fraction(mat, dom)
    k = P.make_const(mat, pr, dom, dt)
    plan = PL.raster_for_steps(dom, dt, 200000, V=1.0, hatch=100e-6, n_tracks=20)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            fn()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / reps

    T = torch.full((4096, 4096), 300.0, dtype=torch.float64, device=dev)
    x4 = features(T, k, plan[:STEPS])[None]
    y = torch.empty((1, 4096, 4096), dtype=torch.float32, device=dev)
    fwd_ms = timed(lambda: net.forward(x4, y), 5)
    px = 4096 * 4096
    del x4, y
    tnet = Net(init_params(1), device=dev)
    xb = torch.randn((32, 256, 256, 4), device=dev).to(torch.bfloat16)
    tb = torch.randn((32, 256, 256), dtype=torch.float32, device=dev)
    tr_ms = timed(lambda: tnet.train_step(xb, tb), 10)
    del tnet, xb, tb
    torch.cuda.empty_cache()
    # hybrid vs plain FP64 on a prefix of the 4096^2 raster
    n = args.ss_steps
    T0 = np.full(px, 300.0)
    Th, hyb = run_hybrid(net, k, plan, T0, n, judge_every=8, tol_K=5.0, area_tol=0.02,
                         Tm=mat.Tm, device=dev)
    s = Solver(k, Tm=mat.Tm, device=dev, depth=3)
    s.set_field(300.0)
    torch.cuda.synchronize()
    ev[0].record()
    s.advance(plan[:hyb["steps"]])
    ev[1].record()
    torch.cuda.synchronize()
    plain_ms = ev[0].elapsed_time(ev[1])
    Tp = s.field
    melt_p = int((Tp > mat.Tm).sum().item())
    melt_h = int((Th > mat.Tm).sum().item())
    out = {
        "network": "5 x conv3x3 (4-32-32-32-32-1), GELU, bf16 on tcgen05, fp32 accumulation",
        "weights": "committed" if rec else "untrained (no weights file)",
        "forward_4096sq": {"ms": fwd_ms,
                           "gcell_updates_equiv": px * STEPS / (fwd_ms * 1e-3) / 1e9,
                           "tflops": FLOP_PER_PIXEL * px / (fwd_ms * 1e-3) / 1e12},
        "train_step_32x256sq": {"ms": tr_ms,
                                "tflops": 3 * FLOP_PER_PIXEL * 32 * 256 * 256 / (tr_ms * 1e-3) / 1e12},
        "hybrid_4096sq": {"steps": hyb["steps"], "hybrid_ms": hyb["gpu_ms"], "plain_fp64_ms": plain_ms,
                          "speedup_vs_plain": plain_ms / hyb["gpu_ms"],
                          "max_abs_err_vs_fp64_K": _finite((Th - Tp).abs().max().item()),
                          "melt_area_err": abs(melt_h - melt_p) / max(melt_p, 1),
                          "judged": hyb["judged"], "rolled_back": hyb["rolled_back"],
                          "worst_window_K": _finite(hyb["worst_K"]),
                          "full_fp64_blocks": hyb.get("full_fp64_blocks", 0)},
        "heldout": rec.get("heldout_trained") if rec else None,
    }
    del s, Tp, Th
    if args.ss_scenarios > 0:
        out["hybrid_process_map"] = hybrid_scenarios(net, args.ss_scenarios, args.ss_pm_steps,
                                                     dev)
    peak = None
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as f:
            peak = json.load(f).get("bf16_tflops")
    if peak:
        out["forward_4096sq"]["frac_of_measured_bf16"] = out["forward_4096sq"]["tflops"] / peak
    else:   # earlier cuBLAS bf16 burst measurement on B200
        out["forward_4096sq"]["frac_of_fallback_bf16_1590"] = out["forward_4096sq"]["tflops"] / 1590.0
    # 32-channel 3x3 layers do about 111 FLOP per byte they must move, below
    # the B200's ridge (bf16 peak / HBM bandwidth, about 256): the forward is
    # bound by HBM.  Bytes per pixel: features in (8), four 32-channel bf16
    # activations written (4 x 64) and read by the next layer (4 x 64), y
    # out (4).
    fwd_bytes = px * (8 + 4 * 64 + 4 * 64 + 4)
    hbm = measured_peaks()
    gbs = fwd_bytes / (fwd_ms * 1e-3) / 1e9
    out["forward_4096sq"]["roofline"] = {
        "bound": "hbm", "algorithmic_bytes": fwd_bytes, "achieved": gbs, "unit": "GB/s",
        "peak": hbm[0], "peak_source": hbm[1], "frac": gbs / hbm[0]}
    return out


def _finite(v):
    """A float for the JSON line, or None when it is not finite (strict JSON
    has no NaN)."""
    v = float(v)
    return v if math.isfinite(v) else None


def hybrid_scenarios(net, n_scen: int, n_steps: int, dev):
    """The batched part of the surrogate-in-the-loop workload: n_scen seeded
    process-map scenarios (grid side 256..2048, power, speed, spot, raster
    angle and hatch drawn per scenario), each advanced n_steps by super-steps
    of the network with the FP64 judge every 8 super-steps (one scenario
    after another), against the same scenarios advanced together by the
    batched FP64 kernel (one launch sequence): time-to-solution, max |dT|
    and melt-area error against the FP64 fields."""
    import torch
    from hedgehog_lpbf_b200 import process_map as PM
    from hedgehog_lpbf_b200.batch import Batch, batch_opts
    from hedgehog_lpbf_b200.superstep import run_hybrid
    torch.cuda.empty_cache()
    scs = PM.process_map(n_scen, n_steps)
    b = Batch(scs, n_steps, opts=batch_opts(depth=2), device=dev, rings=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.run(0, n_steps)
    e1.record()
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    hyb_ms, worst, area_worst, judged, rolled, full = 0.0, 0.0, 0.0, 0, 0, 0
    for i, sc in enumerate(scs):
        Th, r = run_hybrid(net, sc.k, sc.plan, np.full(sc.k.nx * sc.k.ny, sc.k.Tamb), n_steps,
                           judge_every=8, tol_K=5.0, area_tol=0.02, Tm=sc.Tm, device=dev)
        hyb_ms += r["gpu_ms"]
        judged += r["judged"]
        rolled += r["rolled_back"]
        full += r["full_fp64_blocks"]
        Tp = b.field(i)
        d = float((Th - Tp).abs().max().item())
        worst = d if not math.isfinite(d) else max(worst, d)
        mp, mh = int((Tp > sc.Tm).sum().item()), int((Th > sc.Tm).sum().item())
        area_worst = max(area_worst, abs(mh - mp) / max(mp, 1) if (mp or mh) else 0.0)
        del Th
    b.close()
    return {"scenarios": n_scen, "steps_each": n_steps, "hybrid_ms": hyb_ms,
            "plain_fp64_batched_ms": plain_ms, "speedup_vs_plain": plain_ms / hyb_ms,
            "max_abs_err_vs_fp64_K": _finite(worst), "worst_melt_area_err": area_worst,
            "judged": judged, "rolled_back": rolled, "full_fp64_blocks": full,
            "note": "hybrid scenarios run one after another; the FP64 reference is the "
                    "batched kernel over all scenarios"}


def sharded_leg(args, dev, rank=0, world=1, single_value=None):
    """One 8192^2 field cut into row strips: across the ranks (one strip
    each, halo rows exchanged over NCCL after every launch; strong scaling),
    or, on one GPU, into 4 strips exchanged by device copies (the cost of
    the cut and of the exchange).  On one GPU the result is checked bit for
    bit against the single-field solver."""
    import torch
    from hedgehog_lpbf_b200.sharded import ShardedField
    from hedgehog_lpbf_b200.solver import Solver
    mat, pr, dom, k, plan = workload(0)
    depth = 3
    n_warm, n = 30, args.sh_steps
    kw = dict(depth=depth, device=dev, T0=300.0, Tm=mat.Tm)
    if world > 1:
        f = ShardedField.distributed(k, rank, world, **kw)
        parts, kind = world, "NCCL send/recv between ranks"
    else:
        f = ShardedField.local(k, 4, **kw)
        parts, kind = 4, "device copies within one GPU"
    f.advance(plan[:n_warm], rings=False)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rings = f.advance(plan[n_warm:n_warm + n])
    e1.record()
    torch.cuda.synchronize()
    from hedgehog_lpbf_b200.ranks import max_over_ranks
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    out = {"value": dom.nx * dom.ny * n / (ms * 1e-3) / 1e9, "unit": "GCell-updates/s",
           "strips": parts, "halo_rows": depth, "exchange": kind, "time_steps": n, "ms": ms,
           "launches": "one stream per strip" if world == 1 else "one strip per rank",
           "scaling": "strong (one field)" if world > 1 else "one GPU",
           "error_word": f.read_error()}
    parts_ring = f.partials(rings)
    if world == 1:
        s = Solver(k, device=dev, Tm=mat.Tm, depth=depth, T0=300.0)
        s.advance(plan[:n_warm])
        r = s.new_ring(n)
        s.advance(plan[n_warm:n_warm + n], r)
        same = torch.equal(f.field(), s.field)
        out["bit_identical_to_single_field"] = bool(
            same and parts_ring.tobytes() == r.cpu().numpy().tobytes())
        if single_value:
            out["vs_single_field"] = out["value"] / single_value
        del s
    return out


def run_b200_arm(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from hedgehog_lpbf_b200.solver import Solver

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    mat, pr, dom, k, plan = workload(rank)
    s = Solver(k, device=dev, Tm=mat.Tm, depth=args.depth)
    depth = min(4, args.depth) if args.depth > 0 else (3 if N_SIDE * N_SIDE >= (1 << 22) else 2)
    launches = s.launches(STEPS_PER_ITER)
    ring = s.new_ring(STEPS_PER_ITER)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up
    for i in range(args.warmup):
        s.advance(plan_slice(plan, i), ring)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        step_ev[0].record(stream)
        for i in range(args.steps):
            s.advance(plan_slice(plan, args.warmup + i), ring)
            step_ev[i + 1].record(stream)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    step_ms = [step_ev[i].elapsed_time(step_ev[i + 1]) for i in range(args.steps)]
    T64 = s.field.clone() if args.f32k else None
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    err = s.read_error()

    cells = dom.nx * dom.ny
    updates = cells * STEPS_PER_ITER * args.steps * world
    value = updates / (ms_max * 1e-3) / 1e9

    # ---- end-to-end through the public call, host buffers -----------------
    host_in = torch.full((dom.ny, dom.nx), 300.0, dtype=torch.float64).pin_memory()
    host_out = torch.empty((dom.ny, dom.nx), dtype=torch.float64).pin_memory()
    host_ring = torch.empty(STEPS_PER_ITER * 24, dtype=torch.uint8).pin_memory()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    # independent runs streamed through the public call: every run's field
    # is copied in from pinned host memory and its field and Partials copied
    # out, on a copy stream that overlaps the neighbouring runs' compute
    s.run_many([host_in] * e2e_steps, [plan_slice(plan, i) for i in range(e2e_steps)],
               [host_out] * e2e_steps, [host_ring] * e2e_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    t2 = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_value = cells * STEPS_PER_ITER * e2e_steps * world / (float(t2.item()) * 1e-3) / 1e9

    # ---- FP32 compensated variant on the same plan, against the FP64 field --
    f32k = None
    if args.f32k:
        from hedgehog_lpbf_b200.solver import SolverF32K
        del host_in, host_out
        sk = SolverF32K(k, device=dev, Tm=mat.Tm, depth=args.depth)
        for i in range(args.warmup):
            sk.advance(plan_slice(plan, i), ring)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for i in range(args.steps):
            sk.advance(plan_slice(plan, args.warmup + i), ring)
        f1.record(stream)
        torch.cuda.synchronize()
        fms = f0.elapsed_time(f1)
        err32 = float((sk.field64() - T64).abs().max().item())
        f32k = {"value": cells * STEPS_PER_ITER * args.steps / (fms * 1e-3) / 1e9,
                "unit": "GCell-updates/s", "ms_per_step": fms / args.steps,
                "time_steps": STEPS_PER_ITER * (args.warmup + args.steps),
                "max_abs_err_vs_fp64_K": err32, "target_K": 0.05,
                "bytes_per_update": 16}
        del sk
        # the plain FP32 field (one f32 array, 8 B per update), same plan
        from hedgehog_lpbf_b200.solver import SolverF32
        sp = SolverF32(k, device=dev, Tm=mat.Tm, depth=args.depth)
        for i in range(args.warmup):
            sp.advance(plan_slice(plan, i), ring)
        torch.cuda.synchronize()
        f0.record(stream)
        for i in range(args.steps):
            sp.advance(plan_slice(plan, args.warmup + i), ring)
        f1.record(stream)
        torch.cuda.synchronize()
        pms = f0.elapsed_time(f1)
        errp = float((sp.field64() - T64).abs().max().item())
        pval = cells * STEPS_PER_ITER * args.steps / (pms * 1e-3) / 1e9
        hbm = measured_peaks()
        f32k["plain_f32"] = {
            "value": pval, "unit": "GCell-updates/s", "ms_per_step": pms / args.steps,
            "vs_fp64": pval / (value / world), "max_abs_err_vs_fp64_K": errp,
            "target_K": 0.05, "bytes_per_update": 8,
            "algorithmic_GBs": pval * 8, "frac_of_hbm": pval * 8 / hbm[0],
            "hbm_source": hbm[1], "error_word": sp.read_error()}
        del sp, T64

    del s
    # across ranks only on request: that path (NCCL halo exchange) is
    # exercised by the tests with gloo ranks on CPU, not on several GPUs
    run_sh = args.sharded and (world == 1 or args.shard_ranks)
    sh = sharded_leg(args, dev, rank, world, value / world) if run_sh else None
    ext = ext_leg(args, dev) if args.ext else None
    di = dropin_leg(args, dev) if args.dropin else None
    pm = None
    if args.process_map:
        pm = process_map_leg(args, dev, rank, world)
    ss = None
    if args.superstep and world == 1:
        ss = superstep_leg(args, dev)

    if rank != 0:
        return
    peak, peak_src = measured_peaks()
    launch_ms = statistics.median(step_ms) / launches
    steps_per_launch = STEPS_PER_ITER / launches
    achieved = BYTES_PER_UPDATE * cells * steps_per_launch / (launch_ms * 1e-3) / 1e9
    prof = ADVANCE_PROFILE.get(depth, {}) if N_SIDE == 8192 else {}
    traffic = prof.get("dram_bytes")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                "kernel": f"advance_kernel<{depth},TMA,reduce>",
                "algorithmic_bytes": f"{BYTES_PER_UPDATE} B per cell-update x {cells} cells"
                                     f" x {steps_per_launch:g} steps per launch",
                "frac_meaning": "algorithmic bytes of the time steps one launch advances "
                                "(temporal blocking: effective, may exceed 1)",
                "launch_ms": launch_ms}
    if traffic:
        # the DRAM bytes ncu counted for one launch over this run's launch time
        roofline["dram_gbs"] = traffic / (launch_ms * 1e-3) / 1e9
        roofline["dram_frac"] = roofline["dram_gbs"] / peak
    if prof.get("fp64_pipe") is not None:
        roofline["fp64_pipe"] = prof["fp64_pipe"]
        roofline["limiter"] = prof.get("limiter")
    if prof:
        roofline["profile"] = prof["source"]
    line = {
        "metric": "GCell-updates/s", "value": value, "unit": "GCell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (uniform 300 K start, seeded raster plan per rank)",
        "config": config(depth, world),
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": "GCell-updates/s",
                "h2d_bytes_per_step": cells * 8,
                "d2h_bytes_per_step": cells * 8 + STEPS_PER_ITER * 24,
                "steps": e2e_steps,
                "call": "Solver.run_many: independent runs, host copies overlapped with "
                        "the neighbouring runs' compute"},
        "gpu_launches": launches * args.steps,
        "f32k": f32k,
        "ext_physics": ext,
        "dropin_abi": di,
        "process_map": pm,
        "sharded": sh,
        "superstep": ss,
        "clocks": clk.summary(),
        "error_word": err,
    }
    if world == 1 and not args.no_cpu_baseline:
        # the reference's own implementations of the step, timed here as the
        # baselines: its multi-threaded CPU task, its single-thread run_cpu
        # and its GPU task graph on this GPU
        cb = cpu_reference_rate(mat, pr, dom, k, plan, budget_s=args.ref_budget)
        st = cpu_single_thread_rate(mat, pr, dom, k, budget_s=args.ref_budget)
        if st:
            cb["single_thread_run_cpu"] = st
        line["cpu_baseline"] = cb
        if N_SIDE == 8192 and not args.no_ref_gpu:
            torch.cuda.empty_cache()
            rg = reference_gpu_rate()
            line["ref_gpu"] = rg
            if rg.get("value"):
                line["speedup_vs_ref_gpu"] = value / rg["value"]
                line["e2e_speedup_vs_ref_gpu"] = e2e_value / rg["value"]
                if di:
                    # the same host call sequence: this library's kernels
                    # against the reference's
                    di["vs_ref_gpu_same_calls"] = di["value"] / rg["value"]
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--depth", type=int, default=0, help="time steps per launch (0 = auto)")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--ref-budget", type=float, default=15.0,
                    help="seconds of CPU work per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the reference baselines (CPU and GPU)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the reference GPU task graph baseline")
    ap.add_argument("--no-f32k", dest="f32k", action="store_false",
                    help="skip the FP32 compensated leg")
    ap.add_argument("--no-dropin", dest="dropin", action="store_false",
                    help="skip the reference call-sequence leg over the drop-in C-ABI")
    ap.add_argument("--dropin-steps", type=int, default=448)
    ap.add_argument("--no-ext", dest="ext", action="store_false",
                    help="skip the extended-physics leg")
    ap.add_argument("--ext-steps", type=int, default=300)
    ap.add_argument("--no-process-map", dest="process_map", action="store_false",
                    help="skip the batched process-map leg")
    ap.add_argument("--no-sharded", dest="sharded", action="store_false",
                    help="skip the row-strip sharded leg")
    ap.add_argument("--sh-steps", type=int, default=300)
    ap.add_argument("--shard-ranks", action="store_true",
                    help="with --gpus > 1: also shard one field across the ranks")
    ap.add_argument("--pm-scenarios", type=int, default=256)
    ap.add_argument("--pm-steps", type=int, default=5000)
    ap.add_argument("--no-superstep", dest="superstep", action="store_false",
                    help="skip the learned super-stepper leg")
    ap.add_argument("--ss-steps", type=int, default=20480,
                    help="steps of the 4096^2 raster run by the hybrid (multiple of 128)")
    ap.add_argument("--ss-scenarios", type=int, default=64,
                    help="process-map scenarios of the batched hybrid part (0 = skip)")
    ap.add_argument("--ss-pm-steps", type=int, default=1024,
                    help="steps of each scenario in the batched hybrid part")
    ap.add_argument("--tune-cache", default=None,
                    help="JSON cache of the batch autotuner (default: tune every run)")
    ap.add_argument("--side", type=int, default=N_SIDE,
                    help="grid side (smaller sides are for profiling only)")
    ap.add_argument("--iter-steps", type=int, default=STEPS_PER_ITER,
                    help="time steps per bench step")
    ap.add_argument("--ref-gpu-child", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    globals()["N_SIDE"] = args.side
    globals()["STEPS_PER_ITER"] = args.iter_steps
    if args.ref_gpu_child:
        print(json.dumps(reference_gpu_child()), flush=True)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_b200_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
