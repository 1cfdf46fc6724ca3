# SPDX-License-Identifier: 0BSD
"""The reference-compatible C-ABI (include/lpbf_kernels.hpp) driven one time
step at a time, in the call sequence of the reference's GpuStepTask batch
loop (include/gpu_step_task.hpp:145-197 of hedgehog_lpbf).  Per step:
lpbf_launch_step, lpbf_launch_reduce over min(256, ceil(N / 256)) blocks and
lpbf_launch_reduce_finalize into that step's ring slot (unfused), or
lpbf_launch_step_reduce and a finalize over the ceil(nx/16) x ceil(ny/16)
block Partials (fused).  On cruise steps (not wrapped, laser between 0.45
and 0.85 of the domain's width) lpbf_launch_extract_col copies the hot
column.  Once per batch: one copy of the batch's ring to the host and one
synchronization.

This is what a reference build gets by linking liblpbf_b200.so in place of
its kernels: the same host loop, this library's kernels.  The multi-step
entry point (lpbf_b200_advance) is the faster route; this module measures
the drop-in one.

    python -m hedgehog_lpbf_b200.dropin --side 8192 --steps 512 [--fused]
"""
from __future__ import annotations

import ctypes
import json
import time

import numpy as np
import torch

from . import _lib
from . import params as P
from . import plan as PL
from .params import StepConst
from .solver import PARTIAL_DTYPE, _stream_handle


def run(k: StepConst, dom, plan: np.ndarray, Tm: float, *, fused: bool = False,
        batch: int = 64, T0: float = 300.0, device=None) -> dict:
    """Advance a field of k.nx x k.ny cells from a uniform T0 along `plan`
    through the five reference-compatible entry points; returns the timing,
    the per-step Partials (host) and the final field (device)."""
    lib = _lib.lib()
    dev = torch.device(device) if device is not None else torch.device("cuda")
    nx, ny = k.nx, k.ny
    n_cells = nx * ny
    nblocks = int(min(256, (n_cells + 255) // 256))
    nblocks_fused = ((nx + 15) // 16) * ((ny + 15) // 16)
    cur = torch.full((ny, nx), float(T0), dtype=torch.float64, device=dev)
    nxt = torch.empty_like(cur)
    parts = torch.empty(24 * max(nblocks, nblocks_fused), dtype=torch.uint8, device=dev)
    ring = torch.empty(24 * batch, dtype=torch.uint8, device=dev)
    cols = torch.empty((batch, ny), dtype=torch.float64, device=dev)
    host_ring = torch.empty(24 * batch, dtype=torch.uint8, pin_memory=True)
    kk = StepConst.from_buffer_copy(bytes(k))
    out = np.zeros(len(plan), dtype=PARTIAL_DTYPE)
    n_cols = 0
    with torch.cuda.device(dev):
        s = _stream_handle(None)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        for b0 in range(0, len(plan), batch):
            bn = min(batch, len(plan) - b0)
            for i in range(bn):
                tk = plan[b0 + i]
                kk.x_l, kk.y_l, kk.q_scale = float(tk["x_l"]), float(tk["y_l"]), float(tk["q_scale"])
                slot = ring.data_ptr() + 24 * i
                if fused:
                    lib.lpbf_launch_step_reduce(cur.data_ptr(), nxt.data_ptr(), ctypes.byref(kk),
                                                0, Tm, parts.data_ptr(), s)
                    cur, nxt = nxt, cur
                    lib.lpbf_launch_reduce_finalize(parts.data_ptr(), nblocks_fused, nx, ny,
                                                    slot, s)
                else:
                    lib.lpbf_launch_step(cur.data_ptr(), nxt.data_ptr(), ctypes.byref(kk), 0, s)
                    cur, nxt = nxt, cur
                    lib.lpbf_launch_reduce(cur.data_ptr(), nx, ny, Tm, parts.data_ptr(),
                                           nblocks, s)
                    lib.lpbf_launch_reduce_finalize(parts.data_ptr(), nblocks, nx, ny, slot, s)
                xl = float(tk["x_laser_csv"])
                if not bool(tk["wrapped"]) and 0.45 * dom.Lx <= xl <= 0.85 * dom.Lx:
                    lib.lpbf_launch_extract_col(cur.data_ptr(), nx, ny, slot,
                                                cols[i].data_ptr(), s)
                    n_cols += 1
            host_ring[:24 * bn].copy_(ring[:24 * bn], non_blocking=True)
            torch.cuda.current_stream(dev).synchronize()
            out[b0:b0 + bn] = host_ring[:24 * bn].numpy().view(PARTIAL_DTYPE)
        e1.record()
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
        ms = e0.elapsed_time(e1)
    n = len(plan)
    return {"steps": n, "ms": ms, "wall_s": wall, "fused": fused, "batch": batch,
            "extract_col": n_cols, "gcell_updates_per_s": n_cells * n / (ms * 1e-3) / 1e9,
            "ms_per_step": ms / max(n, 1), "partials": out, "field": cur}


def _cli():
    import argparse
    ap = argparse.ArgumentParser(prog="python -m hedgehog_lpbf_b200.dropin")
    ap.add_argument("--side", type=int, default=8192)
    ap.add_argument("--steps", type=int, default=512)
    ap.add_argument("--warmup", type=int, default=64)
    ap.add_argument("--fused", action="store_true")
    a = ap.parse_args()
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(a.side)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    plan = PL.raster_for_steps(dom, k.dt, a.warmup + a.steps, V=1.0, hatch=100e-6, n_tracks=10)
    run(k, dom, plan[:a.warmup], mat.Tm, fused=a.fused)
    r = run(k, dom, plan[a.warmup:], mat.Tm, fused=a.fused)
    r.pop("partials")
    r.pop("field")
    r["side"] = a.side
    print(json.dumps(r))


if __name__ == "__main__":
    _cli()
