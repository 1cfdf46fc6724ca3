# SPDX-License-Identifier: 0BSD
"""Seeded process-map scenarios: grid side, laser power, speed, spot radius,
raster angle and hatch drawn per scenario.

Scenario i draws from a 64-bit Mersenne Twister (the std::mt19937_64 engine
of the C++ standard, restated here from its published definition: Matsumoto
and Nishimura's MT19937-64) seeded with i, in this order:

    side  = (256, 512, 1024, 2048)[x >> 62]
    P     = 100 + 300 u   [W]        u = (x >> 11) * 2^-53 of the next draw
    V     = 0.5 + 1.5 u   [m/s]
    r0    = 35e-6 + 35e-6 u [m]
    angle = pi u          [rad]
    hatch = 80e-6 + 40e-6 u [m]

so a C++ front end built on std::mt19937_64 draws the same scenarios.  The
scan is a serpentine raster of tracks of length 0.6 L spaced `hatch` apart,
covering a 0.6 L square centred in the L x L domain and rotated by `angle`
(it stays inside the domain for every angle).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import params as P
from . import plan as PL

_MASK = (1 << 64) - 1


class MT19937_64:
    """The 64-bit Mersenne Twister (w=64, n=312, m=156, r=31)."""
    N, M = 312, 156
    A = 0xB5026F5AA96619E9
    UPPER, LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF

    def __init__(self, seed: int):
        mt = [0] * self.N
        mt[0] = seed & _MASK
        for i in range(1, self.N):
            mt[i] = (6364136223846793005 * (mt[i - 1] ^ (mt[i - 1] >> 62)) + i) & _MASK
        self.mt = mt
        self.i = self.N

    def _twist(self) -> None:
        mt = self.mt
        for k in range(self.N):
            y = (mt[k] & self.UPPER) | (mt[(k + 1) % self.N] & self.LOWER)
            v = mt[(k + self.M) % self.N] ^ (y >> 1)
            if y & 1:
                v ^= self.A
            mt[k] = v
        self.i = 0

    def __call__(self) -> int:
        if self.i >= self.N:
            self._twist()
        x = self.mt[self.i]
        self.i += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x ^= x >> 43
        return x & _MASK


def u01(x: int) -> float:
    """Top 53 bits of a 64-bit draw as a double in [0, 1)."""
    return (x >> 11) * (1.0 / 9007199254740992.0)


SIDES = (256, 512, 1024, 2048)


@dataclass
class Draw:
    index: int
    side: int
    P: float
    V: float
    r0: float
    angle: float
    hatch: float


def draw(index: int) -> Draw:
    g = MT19937_64(index)
    side = SIDES[g() >> 62]
    Pw = 100.0 + 300.0 * u01(g())
    V = 0.5 + 1.5 * u01(g())
    r0 = 35e-6 + 35e-6 * u01(g())
    angle = math.pi * u01(g())
    hatch = 80e-6 + 40e-6 * u01(g())
    return Draw(index, side, Pw, V, r0, angle, hatch)


def scenario_inputs(d: Draw, n_steps: int, dx: float = 5e-6, side: int | None = None):
    """(StepConst, plan, Material) of a drawn scenario; `side` overrides the
    drawn grid side (smaller test grids with the same laser draws)."""
    n = d.side if side is None else side
    mat, pr = P.benchmark_material_process(P=d.P, V=d.V, r0=d.r0)
    dom = P.square_domain(n, dx)
    dt = P.dt_fraction(mat, dom)
    k = P.make_const(mat, pr, dom, dt)
    span = 0.6 * dom.Lx
    n_tracks = max(1, int(math.floor(span / d.hatch)) + 1)
    plan = PL.raster(dom, dt, n_steps, V=d.V, hatch=d.hatch, track_len=span,
                     n_tracks=n_tracks, angle=d.angle)
    return k, plan, mat


def process_map(n_scen: int, n_steps: int, first_index: int = 0, side: int | None = None):
    """Scenarios first_index .. first_index + n_scen - 1 as batch Scenarios
    (uniform T_amb start, mirror edges)."""
    from .batch import Scenario
    out = []
    for i in range(first_index, first_index + n_scen):
        d = draw(i)
        k, plan, mat = scenario_inputs(d, n_steps, side=side)
        out.append(Scenario(k=k, plan=plan, bc=0, T_edge=300.0, Tm=mat.Tm, T0=None,
                            tag={"draw": d}))
    return out


def cells(n_scen: int, first_index: int = 0) -> int:
    return sum(draw(i).side ** 2 for i in range(first_index, first_index + n_scen))


def summarize(ring: np.ndarray, dy: float) -> dict:
    """Per-scenario results of a run from its per-step Partials: the peak
    temperature and its step, the first molten step and the widest molten
    band (rows from ymin to ymax, as the reference's Partial records them)."""
    tmax = ring["tmax"]
    molten = ring["ymax"] >= 0
    rows = np.where(molten, ring["ymax"] - ring["ymin"] + 1, 0)
    return {"peak_T_K": float(tmax.max()) if len(tmax) else float("nan"),
            "peak_step": int(tmax.argmax()) if len(tmax) else -1,
            "first_melt_step": int(np.argmax(molten)) if molten.any() else -1,
            "molten_steps": int(molten.sum()),
            "max_melt_rows": int(rows.max()) if len(rows) else 0,
            "max_melt_extent_um": float(rows.max() * dy * 1e6) if len(rows) else 0.0}


COLUMNS = ("index", "side", "P_W", "V_mps", "r0_um", "angle_rad", "hatch_um", "steps",
           "peak_T_K", "peak_step", "first_melt_step", "molten_steps", "max_melt_rows",
           "max_melt_extent_um")


def main(argv=None) -> int:
    """Run seeded process-map scenarios as one batch on one GPU and print one
    CSV row per scenario (draw parameters and melt results)."""
    import argparse
    import sys
    import torch
    from .batch import Batch, autotune, batch_opts, opts_dict

    ap = argparse.ArgumentParser(prog="python -m hedgehog_lpbf_b200.process_map")
    ap.add_argument("--scenarios", type=int, default=16)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--first", type=int, default=0, help="index of the first scenario")
    ap.add_argument("--side", type=int, default=None, help="override every drawn grid side")
    ap.add_argument("--depth", type=int, default=None,
                    help="fixed tiles (time steps per launch); default: autotune")
    ap.add_argument("--rows", default="0,0,0,0", help="rows per task per size class (fixed tiles)")
    ap.add_argument("--ctas", type=int, default=0, help="CTAs per SM (fixed tiles; 0 = max)")
    ap.add_argument("--staging", type=int, default=0,
                    help="1 bulk row copies, 2 tensor maps, 0 automatic (fixed tiles)")
    ap.add_argument("--tune-cache", default=None, help="JSON cache of autotuned tiles")
    ap.add_argument("--no-graph", dest="graph", action="store_false")
    ap.add_argument("--out", default="-", help="CSV file ('-' = standard output)")
    args = ap.parse_args(argv)
    if args.scenarios < 1 or args.steps < 1:
        ap.error("--scenarios and --steps must be positive")
    dev = torch.device("cuda:0")
    scs = process_map(args.scenarios, args.steps, args.first, side=args.side)
    if args.depth is not None:
        rows = [int(r) for r in args.rows.split(",")]
        if len(rows) != 4:
            ap.error("--rows takes four comma-separated values")
        opts = batch_opts(depth=args.depth, ctas_per_sm=args.ctas, rows=rows,
                          staging=args.staging)
    else:
        opts = autotune(scs, args.steps, cache=args.tune_cache, device=dev)
    b = Batch(scs, args.steps, opts=opts, device=dev)
    if args.graph:
        b.capture(0, args.steps)          # graph built outside the timed region
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    b.run(0, args.steps, use_graph=args.graph)
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    err = b.read_error()
    out = sys.stdout if args.out == "-" else open(args.out, "w")
    try:
        out.write(",".join(COLUMNS) + "\n")
        for i, sc in enumerate(scs):
            d = sc.tag["draw"]
            r = summarize(b.ring(i), sc.k.dy)
            row = [d.index, sc.k.nx, d.P, d.V, d.r0 * 1e6, d.angle, d.hatch * 1e6, args.steps,
                   r["peak_T_K"], r["peak_step"], r["first_melt_step"], r["molten_steps"],
                   r["max_melt_rows"], r["max_melt_extent_um"]]
            out.write(",".join(f"{v:.6g}" if isinstance(v, float) else str(v) for v in row)
                      + "\n")
    finally:
        if out is not sys.stdout:
            out.close()
    cells = b.cells()
    b.close()
    print(f"# {args.scenarios} scenarios x {args.steps} steps, {cells} cells, "
          f"tiles {opts_dict(opts)}: {ms:.1f} ms, "
          f"{cells * args.steps / (ms * 1e-3) / 1e9:.1f} GCell-updates/s, error word {err}",
          file=sys.stderr)
    return 1 if err else 0


__all__ = ["MT19937_64", "u01", "draw", "Draw", "scenario_inputs", "process_map", "cells", "SIDES",
           "summarize", "main"]

if __name__ == "__main__":
    raise SystemExit(main())
