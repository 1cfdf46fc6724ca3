# SPDX-License-Identifier: 0BSD
"""Snapshots and resume.

A snapshot is the reference's file format (SnapshotWriterTask,
include/gpu_step_task.hpp:427-449; src/main.cpp:364-372): ``T_step_%06d.bin``,
the row-major nx x ny float64 field after that step, no header.  The laser
plan is a pure function of the step index, so (snapshot, step) is a full
checkpoint: ``resume`` loads the field into a Solver, and advancing it along
``plan[step + 1:]`` continues the run bit-identically.
"""
from __future__ import annotations

import os

import numpy as np


def path(directory: str, step: int) -> str:
    return os.path.join(directory, f"T_step_{step:06d}.bin")


def save(field, directory: str, step: int) -> str:
    """Write the field after `step` (torch tensor or array) as a snapshot."""
    os.makedirs(directory, exist_ok=True)
    a = field.detach().cpu().numpy() if hasattr(field, "detach") else np.asarray(field)
    p = path(directory, step)
    np.ascontiguousarray(a, dtype=np.float64).tofile(p)
    return p


def load(p: str, nx: int, ny: int) -> np.ndarray:
    a = np.fromfile(p, dtype=np.float64)
    if a.size != nx * ny:
        raise ValueError(f"{p}: {a.size} values, expected {nx} x {ny}")
    return a.reshape(ny, nx)


def resume(solver, directory: str, step: int):
    """Load the snapshot of `step` into `solver`; continue with plan[step+1:]."""
    solver.set_field(load(path(directory, step), solver.nx, solver.ny))
    return solver
