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


__all__ = ["MT19937_64", "u01", "draw", "Draw", "scenario_inputs", "process_map", "cells", "SIDES"]
