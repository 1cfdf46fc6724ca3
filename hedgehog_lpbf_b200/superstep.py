# SPDX-License-Identifier: 0BSD
"""Training and in-loop use of the learned super-stepper.

* ``make_dataset``: seeded process-map trajectories (grid side, laser power,
  speed, spot radius, raster angle and hatch drawn per trajectory) advanced
  by the batched FP64 solver; every 16 steps the network inputs of the field
  and the field's change over the next 16 steps are kept (bf16 features,
  fp32 targets, on the device).
* ``train``: AdamW on 256 x 256 patches (batch 32), most centred near the
  laser, through the tcgen05 training step of liblpbf_b200.
* ``evaluate``: error of the network against the FP64 solver on held-out
  trajectories, in kelvin, beside the error of predicting no change.
* ``run_hybrid``: advance a field by super-steps of the network; every
  ``judge_every`` super-steps the FP64 solver re-advances the laser window
  (with a halo) from the block's start, and where the network's field there
  differs by more than ``tol_K`` or its melt-pool area (T > T_melt) by more
  than ``area_tol``, the window is rolled back to the FP64 result.

CLI: ``python -m hedgehog_lpbf_b200.superstep train --out FILE`` trains and
stores the weights (npz) with the training record.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np
import torch

from . import params as P
from . import plan as PL
from . import process_map as PM
from .batch import Batch, batch_opts
from .solver import Solver
from .surrogate import (DT_SCALE, STEPS, Net, apply, features, flatten, init_params, target,
                        unflatten)

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "superstepper.npz")


class Dataset:
    """Per snapshot pair: inputs x4 (bf16 [side, side, 4]), target (fp32
    [side, side]) and the laser's grid position at the pair's middle step."""

    def __init__(self, x4, tgt, centre, meta):
        self.x4, self.tgt, self.centre, self.meta = x4, tgt, centre, meta

    def __len__(self):
        return self.x4.shape[0]


def make_dataset(n_traj: int, n_steps: int, side: int = 1024, first_index: int = 0,
                 device="cuda:0") -> Dataset:
    n_pairs = n_steps // STEPS
    n_steps = n_pairs * STEPS
    scs = PM.process_map(n_traj, n_steps, first_index=first_index, side=side)
    dev = torch.device(device)
    b = Batch(scs, n_steps, opts=batch_opts(depth=2, rows=(24, 48, 48, 96)), device=dev,
              rings=False)
    N = n_traj * n_pairs
    x4 = torch.empty((N, side, side, 4), dtype=torch.bfloat16, device=dev)
    tgt = torch.empty((N, side, side), dtype=torch.float32, device=dev)
    centre = np.zeros((N, 2), dtype=np.int64)
    T0 = [torch.empty((side, side), dtype=torch.float64, device=dev) for _ in range(n_traj)]
    for q in range(n_pairs):
        s0 = q * STEPS
        for i, sc in enumerate(scs):
            j = i * n_pairs + q
            features(b.field(i), sc.k, sc.plan[s0:s0 + STEPS], out=x4[j])
            T0[i].copy_(b.field(i))
            mid = sc.plan[s0 + STEPS // 2]
            centre[j] = (int(round(mid["y_l"] / sc.k.dy)), int(round(mid["x_l"] / sc.k.dx)))
        b.run(s0, STEPS)
        for i in range(n_traj):
            target(T0[i], b.field(i), out=tgt[i * n_pairs + q])
    torch.cuda.synchronize(dev)
    b.close()
    meta = {"trajectories": n_traj, "steps": n_steps, "side": side, "first_index": first_index,
            "pairs": N}
    return Dataset(x4, tgt, centre, meta)


def sample(ds: Dataset, rng: np.random.Generator, batch: int, patch: int, near: float = 0.8):
    side = ds.x4.shape[1]
    idx = rng.integers(0, len(ds), size=batch)
    xs, ts = [], []
    for j in idx:
        if rng.random() < near:
            cy, cx = ds.centre[j] + rng.integers(-patch // 4, patch // 4 + 1, size=2)
            y0, x0 = cy - patch // 2, cx - patch // 2
        else:
            y0, x0 = rng.integers(0, side - patch + 1, size=2)
        y0 = int(np.clip(y0, 0, side - patch))
        x0 = int(np.clip(x0, 0, side - patch))
        xs.append(ds.x4[j, y0:y0 + patch, x0:x0 + patch])
        ts.append(ds.tgt[j, y0:y0 + patch, x0:x0 + patch])
    return torch.stack(xs).contiguous(), torch.stack(ts).contiguous()


def train(net: Net, ds: Dataset, iters: int, batch: int = 32, patch: int = 256,
          lr: float = 1e-3, weight_decay: float = 0.01, seed: int = 0, log_every: int = 200):
    """AdamW with cosine decay from lr to lr/100; returns the loss record."""
    rng = np.random.default_rng(seed)
    hist = []
    t0 = time.time()
    for it in range(iters):
        x, t = sample(ds, rng, batch, patch)
        cur = lr * (0.01 + 0.99 * 0.5 * (1.0 + math.cos(math.pi * it / max(1, iters))))
        loss = net.train_step(x, t, lr=cur, weight_decay=weight_decay)
        if (it + 1) % log_every == 0 or it == iters - 1:
            hist.append({"iter": it + 1, "loss": float(loss.item()), "lr": cur,
                         "seconds": time.time() - t0})
    torch.cuda.synchronize(net.device)
    if net.error_word() != 0:
        raise RuntimeError("tensor-core wait timed out during training")
    return hist


def evaluate(net: Net, ds: Dataset, patch: int = 256, n: int = 64, seed: int = 1):
    """Errors (K) of the network's 16-step change on laser-centred patches,
    beside those of predicting no change."""
    rng = np.random.default_rng(seed)
    err, base, sq, sqb, cnt = 0.0, 0.0, 0.0, 0.0, 0
    for _ in range(max(1, n // 16)):
        x, t = sample(ds, rng, 16, patch, near=1.0)
        y = net.forward(x)
        d = (y - t) * DT_SCALE
        err = max(err, float(d.abs().max().item()))
        base = max(base, float((t * DT_SCALE).abs().max().item()))
        sq += float((d.double() ** 2).sum().item())
        sqb += float(((t * DT_SCALE).double() ** 2).sum().item())
        cnt += t.numel()
    return {"max_abs_K": err, "rms_K": math.sqrt(sq / cnt),
            "no_change_max_abs_K": base, "no_change_rms_K": math.sqrt(sqb / cnt)}


def save(net: Net, path: str, record: dict) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=net.params_vector(), record=json.dumps(record))


def load(path: str = WEIGHTS, device="cuda:0") -> tuple[Net, dict]:
    z = np.load(path, allow_pickle=False)
    net = Net(z["params"], device=device)
    return net, json.loads(str(z["record"]))


# ---- in-loop use -----------------------------------------------------------------

def _window(plan, s0, s1, k, margin, nx, ny):
    xs, ys = plan["x_l"][s0:s1], plan["y_l"][s0:s1]
    x0 = int(math.floor(xs.min() / k.dx)) - margin
    x1 = int(math.ceil(xs.max() / k.dx)) + margin
    y0 = int(math.floor(ys.min() / k.dy)) - margin
    y1 = int(math.ceil(ys.max() / k.dy)) + margin
    return max(0, y0), min(ny, y1 + 1), max(0, x0), min(nx, x1 + 1)


def judge(got: torch.Tensor, ref: torch.Tensor, tol_K: float, area_tol: float, Tm: float):
    """The FP64 judge's verdict on one window: (max |got - ref| in K, melt-pool
    area error, roll back?).  Roll back where the field misses by more than
    tol_K or the area of T > Tm differs by more than area_tol (relative)."""
    diff, area, back = judge_device(got, ref, tol_K, area_tol, Tm)
    return float(diff.item()), float(area.item()), bool(back.item())


def judge_device(got: torch.Tensor, ref: torch.Tensor, tol_K: float, area_tol: float,
                 Tm: float):
    """``judge`` as 0-d device tensors, with no host synchronization: the
    loop below acts on the verdict on the device (torch.where) and reads the
    records once at the end."""
    diff = (got - ref).abs().max()
    a_ref = (ref > Tm).sum()
    a_got = (got > Tm).sum()
    area = (a_got - a_ref).abs().double() / a_ref.clamp(min=1).double()
    back = (diff > tol_K) | (area > area_tol) | ~torch.isfinite(diff)
    return diff, area, back


def _windows(plan, blocks: int, per_block: int, k, margin: int, halo: int):
    """Per judged block: the laser window (rows y0:y1, columns x0:x1, the
    cells the judge compares) and the origin of a fixed-size FP64 solve box
    that holds it with `halo` cells of surroundings (fewer at the field's
    edges, which are the field's own boundary).  Returns (windows, box
    height, box width)."""
    win = [_window(plan, b * per_block, (b + 1) * per_block, k, margin, k.nx, k.ny)
           for b in range(blocks)]
    bh = min(k.ny, max(w[1] - w[0] for w in win) + 2 * halo)
    bw = min(k.nx, max(w[3] - w[2] for w in win) + 2 * halo)
    out = []
    for wy0, wy1, wx0, wx1 in win:
        oy = min(max(wy0 - halo, 0), k.ny - bh)
        ox = min(max(wx0 - halo, 0), k.nx - bw)
        out.append((wy0, wy1, wx0, wx1, oy, ox))
    return out, bh, bw


def run_hybrid(net: Net, k, plan, T0, n_steps: int, judge_every: int = 8, tol_K: float = 5.0,
               area_tol: float = 0.02, Tm: float = 1700.0, margin: int | None = None,
               halo: int = 32, device="cuda:0", guard: bool = True):
    """Super-steps of the network with the FP64 judge and rollback.  Returns
    (field, record).

    Every ``judge_every`` super-steps the FP64 solver re-advances, from the
    block's start, a fixed-size box around the block's laser window (one
    solver for the whole run, so no buffers, workspace or tensor map are
    made per window); the verdict and the rollback (torch.where over the
    window) stay on the device, and the per-window records are read once at
    the end.

    Outside the windows the network's errors accumulate unjudged, so every
    block is also held to the discrete maximum principle: the laser heats
    only inside the judged box, and the explicit step with its losses towards
    Tamb/Tsub moves no cell above the largest or below the smallest of its
    neighbourhood and those temperatures.  So after a block every cell lies
    within [min(block-start field, Tamb, Tsub) - tol_K, max(block-start
    field, FP64 box field, Tamb, Tsub) + tol_K].  A block whose field leaves
    that range or is not finite is redone from its start with the FP64
    solver over the whole field (counted in "full_fp64_blocks"); this keeps
    the field inside the range in which the explicit step (whose radiation
    term is unstable for very large T) stays finite.  The check reads one
    flag per block on the host; ``guard=False`` leaves it out (the network's
    own error outside the windows then shows in the field)."""
    dev = torch.device(device)
    if isinstance(T0, torch.Tensor):
        T = T0.to(dev, torch.float64).reshape(k.ny, k.nx).clone()
    else:
        T = torch.as_tensor(np.asarray(T0, dtype=np.float64)).to(dev).reshape(k.ny, k.nx).clone()
    if margin is None:
        margin = int(math.ceil(6.0 / math.sqrt(k.inv_r0_sq) / k.dx)) + 8
    per_block = STEPS * judge_every
    blocks = n_steps // per_block
    wins, bh, bw = _windows(plan, blocks, per_block, k, margin, halo) if blocks else ([], 1, 2)
    ks = P.StepConst.from_buffer_copy(bytes(k))
    ks.nx, ks.ny = bw, bh
    fp64 = Solver(ks, Tm=Tm, device=dev, T0=k.Tamb) if blocks else None
    diffs = torch.zeros(max(blocks, 1), dtype=torch.float64, device=dev)
    areas = torch.zeros(max(blocks, 1), dtype=torch.float64, device=dev)
    backs = torch.zeros(max(blocks, 1), dtype=torch.bool, device=dev)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    x4 = torch.empty((k.ny, k.nx, 4), dtype=torch.bfloat16, device=dev)
    T_start = torch.empty_like(T)
    full = None                  # FP64 solver over the whole field, made on first need
    n_full = 0
    t_lo, t_hi = min(k.Tamb, k.Tsub), max(k.Tamb, k.Tsub)
    for blk, (wy0, wy1, wx0, wx1, oy, ox) in enumerate(wins):
        s_blk = blk * per_block
        T_start.copy_(T)
        mn0, mx0 = torch.aminmax(T_start)
        fp64.set_field(T[oy:oy + bh, ox:ox + bw])
        for j in range(judge_every):
            s = s_blk + j * STEPS
            features(T, k, plan[s:s + STEPS], out=x4)
            y = net.forward(x4[None])
            apply(T, y[0])
        # FP64 judge on the window (the box's other cells give it the surroundings)
        sub_plan = plan[s_blk:s_blk + per_block].copy()
        sub_plan["x_l"] -= ox * k.dx
        sub_plan["y_l"] -= oy * k.dy
        fp64.advance(sub_plan)
        mn1, mx1 = torch.aminmax(T)
        lo = torch.clamp(mn0, max=t_lo) - tol_K
        hi = torch.maximum(mx0, fp64.field.max()).clamp(min=t_hi) + tol_K
        ok = torch.isfinite(mn1) & torch.isfinite(mx1) & (mn1 >= lo) & (mx1 <= hi)
        if guard and not bool(ok):
            if full is None:
                full = Solver(k, Tm=Tm, device=dev, T0=k.Tamb)
            full.set_field(T_start)
            full.advance(plan[s_blk:s_blk + per_block])
            T.copy_(full.field)
            n_full += 1
        ref = fp64.field[wy0 - oy:wy1 - oy, wx0 - ox:wx1 - ox]
        got = T[wy0:wy1, wx0:wx1]
        d, a, back = judge_device(got, ref, tol_K, area_tol, Tm)
        diffs[blk], areas[blk], backs[blk] = d, a, back
        got.copy_(torch.where(back, ref, got))
    e1.record()
    torch.cuda.synchronize(dev)
    rb = backs[:blocks].cpu().numpy()
    rec = {"super_steps": blocks * judge_every, "judged": blocks,
           "rolled_back": int(rb.sum()),
           "worst_K": float(diffs[:blocks].max().item()) if blocks else 0.0,
           "worst_area": float(areas[:blocks].max().item()) if blocks else 0.0,
           "fp64_window_cells": blocks * bh * bw, "judge_box": [bh, bw],
           "full_fp64_blocks": n_full,
           "gpu_ms": e0.elapsed_time(e1), "steps": blocks * per_block}
    return T, rec


def _cli():
    ap = argparse.ArgumentParser(prog="python -m hedgehog_lpbf_b200.superstep")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--trajectories", type=int, default=64)
    t.add_argument("--steps", type=int, default=512)
    t.add_argument("--side", type=int, default=1024)
    t.add_argument("--iters", type=int, default=20000)
    t.add_argument("--batch", type=int, default=32)
    t.add_argument("--patch", type=int, default=256)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--heldout", type=int, default=8)
    t.add_argument("--seed", type=int, default=0)
    f = sub.add_parser("forward", help="time the network's forward pass on a side x side field")
    f.add_argument("--side", type=int, default=4096)
    f.add_argument("--reps", type=int, default=5)
    f.add_argument("--form", type=int, default=0,
                   help="layer kernel form (lpbf_b200_sg_set_form: 0 rows, 1 tap tiles, 2 plain)")
    a = ap.parse_args()
    if a.cmd == "forward":
        from . import _lib
        _lib.check(_lib.lib().lpbf_b200_sg_set_form(a.form), "sg_set_form")
        net = load()[0] if os.path.exists(WEIGHTS) else Net(init_params(0))
        mat, pr = P.benchmark_material_process()
        dom = P.square_domain(a.side)
        k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
        plan = PL.raster_for_steps(dom, k.dt, 64, V=1.0, hatch=100e-6, n_tracks=2)
        T = torch.full((a.side, a.side), 300.0, dtype=torch.float64, device="cuda")
        x4 = features(T, k, plan)[None]
        y = net.forward(x4)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.reps):
            net.forward(x4, y)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
        flop = 2 * 9 * (4 * 32 + 3 * 32 * 32 + 32) * a.side * a.side
        print(json.dumps({"side": a.side, "form": a.form, "ms": ms,
                          "tflops": flop / (ms * 1e-3) / 1e12, "error_word": net.error_word()}))
        return
    t0 = time.time()
    ds = make_dataset(a.trajectories, a.steps, side=a.side, first_index=0)
    held = make_dataset(a.heldout, a.steps, side=a.side, first_index=100000)
    t_data = time.time() - t0
    net = Net(init_params(a.seed))
    before = evaluate(net, held, patch=a.patch)
    hist = train(net, ds, a.iters, batch=a.batch, patch=a.patch, lr=a.lr, seed=a.seed)
    after = evaluate(net, held, patch=a.patch)
    rec = {"dataset": ds.meta, "heldout": held.meta, "iters": a.iters, "batch": a.batch,
           "patch": a.patch, "lr": a.lr, "optimizer": "AdamW, cosine decay to lr/100, wd 0.01",
           "data_seconds": t_data, "train_seconds": hist[-1]["seconds"],
           "loss": hist, "heldout_untrained": before, "heldout_trained": after}
    save(net, a.out, rec)
    print(json.dumps({k: v for k, v in rec.items() if k != "loss"} |
                     {"final_loss": hist[-1]["loss"]}))


if __name__ == "__main__":
    _cli()
