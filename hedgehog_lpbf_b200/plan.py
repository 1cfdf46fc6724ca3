# SPDX-License-Identifier: 0BSD
"""Laser plans: one ``Tick`` per time step.

A plan is a numpy structured array with the byte layout of the reference's
``lpbf::Tick`` (include/gpu_messages.hpp:18-26), so it can be passed to the
C-ABI as ``const Tick*`` without conversion.  The step kernel uses
``x_l, y_l, q_scale`` of step s (the *pre*-advance laser position);
``x_laser_csv``/``wrapped`` are the *post*-advance state used by the metrics.

* ``single_track``  -- the reference's law, src/gpu/hh_gpu_main.cpp:141-157
  (start at 0.2 Lx on the centre line, advance V dt, wrap back to the start
  once past 0.9 Lx).
* ``raster``        -- new: a serpentine (bidirectional) or unidirectional
  hatch pattern at any angle, which the reference cannot express; it emits
  the same Tick fields, so every plan remains checkable against the
  reference's own step, which accepts any per-step (x_l, y_l, q_scale).
"""
from __future__ import annotations

import math

import numpy as np

from .params import Domain, Process

TICK_DTYPE = np.dtype({
    "names": ["step", "t", "x_l", "y_l", "q_scale", "x_laser_csv", "wrapped", "dump"],
    "formats": [np.int32, np.float64, np.float64, np.float64, np.float64, np.float64,
                np.bool_, np.bool_],
    "offsets": [0, 8, 16, 24, 32, 40, 48, 49],
    "itemsize": 56,
})


def _dump_flags(n_steps: int, snap_every: int) -> np.ndarray:
    s = np.arange(n_steps)
    dump = (s == n_steps - 1)
    if snap_every > 0:
        dump |= (s % snap_every == 0)
    return dump


def single_track(pr: Process, dom: Domain, dt: float, n_steps: int,
                 snap_every: int = 0) -> np.ndarray:
    """hh_gpu_main.cpp:141-157, step for step (the same double arithmetic)."""
    plan = np.zeros(n_steps, dtype=TICK_DTYPE)
    x = 0.20 * dom.Lx
    y = 0.50 * dom.Ly
    x_start = x
    wrapped = False
    xs = np.empty(n_steps)
    xcsv = np.empty(n_steps)
    wr = np.empty(n_steps, dtype=bool)
    for s in range(n_steps):
        xs[s] = x
        x += pr.V * dt
        if x > 0.90 * dom.Lx:
            x = x_start
            wrapped = True
        xcsv[s] = x
        wr[s] = wrapped
    plan["step"] = np.arange(n_steps, dtype=np.int32)
    plan["t"] = np.arange(n_steps, dtype=np.float64) * dt
    plan["x_l"] = xs
    plan["y_l"] = y
    plan["q_scale"] = 1.0
    plan["x_laser_csv"] = xcsv
    plan["wrapped"] = wr
    plan["dump"] = _dump_flags(n_steps, snap_every)
    return plan


def raster(dom: Domain, dt: float, n_steps: int, V: float, hatch: float,
           track_len: float, n_tracks: int, angle: float = 0.0,
           center: tuple[float, float] | None = None, bidirectional: bool = True,
           jump_time: float = 0.0, t0: float = 0.0, snap_every: int = 0) -> np.ndarray:
    """Hatch pattern of ``n_tracks`` parallel tracks of length ``track_len``
    spaced ``hatch`` apart, rotated by ``angle`` about ``center`` (default:
    the domain centre), scanned at speed ``V``.  Bidirectional scans alternate
    direction (serpentine).  Between tracks the beam is off (q_scale = 0) for
    ``jump_time`` seconds; with jump_time = 0 the beam moves on at once.  After
    the last track the pattern restarts and ``wrapped`` becomes true.  Step s
    uses the position at time t0 + s*dt."""
    if n_tracks < 1 or track_len <= 0 or V <= 0:
        raise ValueError("raster needs n_tracks >= 1, track_len > 0, V > 0")
    cx, cy = center if center is not None else (0.5 * dom.Lx, 0.5 * dom.Ly)
    d = np.array([math.cos(angle), math.sin(angle)])
    nrm = np.array([-math.sin(angle), math.cos(angle)])
    t_track = track_len / V
    t_unit = t_track + jump_time
    period = n_tracks * t_unit

    def pos(t: np.ndarray):
        tt = np.mod(t, period)
        i = np.minimum((tt // t_unit).astype(np.int64), n_tracks - 1)
        u = tt - i * t_unit                      # time since track start
        on = u < t_track
        frac = np.clip(u / t_track, 0.0, 1.0)
        off = (i - 0.5 * (n_tracks - 1)) * hatch
        sgn = np.where(bidirectional & (i % 2 == 1), -1.0, 1.0)
        along = sgn * (frac - 0.5) * track_len
        x = cx + off * nrm[0] + along * d[0]
        y = cy + off * nrm[1] + along * d[1]
        return x, y, on, t >= period

    s = np.arange(n_steps, dtype=np.float64)
    x, y, on, _ = pos(t0 + s * dt)
    xp, _, _, wrapped = pos(t0 + (s + 1.0) * dt)
    plan = np.zeros(n_steps, dtype=TICK_DTYPE)
    plan["step"] = np.arange(n_steps, dtype=np.int32)
    plan["t"] = s * dt
    plan["x_l"] = x
    plan["y_l"] = y
    plan["q_scale"] = np.where(on, 1.0, 0.0)
    plan["x_laser_csv"] = xp
    plan["wrapped"] = wrapped
    plan["dump"] = _dump_flags(n_steps, snap_every)
    return plan


def raster_for_steps(dom: Domain, dt: float, n_steps: int, V: float, hatch: float,
                     n_tracks: int, angle: float = 0.0, snap_every: int = 0) -> np.ndarray:
    """Raster whose tracks are long enough that ``n_tracks`` tracks take
    ``n_steps`` steps (track_len = V * n_steps * dt / n_tracks)."""
    track_len = V * n_steps * dt / n_tracks
    return raster(dom, dt, n_steps, V=V, hatch=hatch, track_len=track_len,
                  n_tracks=n_tracks, angle=angle, snap_every=snap_every)


def laser_array(plan: np.ndarray) -> np.ndarray:
    """(n_steps, 3) float64 array of (x_l, y_l, q_scale) per step."""
    out = np.empty((len(plan), 3), dtype=np.float64)
    out[:, 0] = plan["x_l"]
    out[:, 1] = plan["y_l"]
    out[:, 2] = plan["q_scale"]
    return out
