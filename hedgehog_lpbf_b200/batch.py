# SPDX-License-Identifier: 0BSD
"""Python host API of the batched process map (lpbf_b200_batch_* in
include/lpbf_b200.h).

A :class:`Batch` owns, for each scenario, a device ping-pong pair and a ring
of per-step Partials, plus one workspace; ``run`` advances every scenario
along its own plan in shared launches (optionally one CUDA graph).  The
reference runs the same ensemble serially, one GpuStepTask graph per manifest
row (src/gpu/hh_gpu_main.cpp:162-270).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .params import StepConst
from .plan import TICK_DTYPE
from .solver import PARTIAL_DTYPE, _stream_handle


@dataclass
class Scenario:
    """One field of a batch: its constants, its plan (one Tick per step of the
    batch) and its edge condition; T0 is a scalar or an (ny, nx) array."""
    k: StepConst
    plan: np.ndarray
    bc: int = 0
    T_edge: float = 300.0
    Tm: float = 1700.0
    T0: float | np.ndarray | None = None
    tag: dict = field(default_factory=dict)


def batch_opts(depth: int = 0, ctas_per_sm: int = 0, rows=(0, 0, 0, 0),
               staging: int = 0) -> _lib.BatchOpts:
    o = _lib.BatchOpts()
    o.depth = depth
    o.ctas_per_sm = ctas_per_sm
    o.staging = staging
    for i in range(4):
        o.rows[i] = int(rows[i])
    return o


def _host_array(scenarios, n_steps):
    """lpbf_b200_scenario array with the host fields only (k, plan, edges);
    returns it with the objects that must stay alive while it is used."""
    arr = (_lib.Scenario * len(scenarios))()
    keep = []
    for i, s in enumerate(scenarios):
        k = StepConst.from_buffer_copy(bytes(s.k))
        plan = np.ascontiguousarray(s.plan[:n_steps], dtype=TICK_DTYPE)
        if len(plan) < n_steps:
            raise ValueError(f"scenario {i}: plan has {len(plan)} < {n_steps} steps")
        keep += [k, plan]
        arr[i].k = ctypes.pointer(k)
        arr[i].plan = plan.ctypes.data
        arr[i].bc = s.bc
        arr[i].T_edge = s.T_edge
        arr[i].Tm = s.Tm
    return arr, keep


def tune_key(scenarios) -> str:
    """Cache key of a batch (GPU name, SM count, size-class histogram)."""
    arr, _keep = _host_array(scenarios, 0)
    buf = ctypes.create_string_buffer(512)
    _lib.check(_lib.lib().lpbf_b200_batch_tune_key(arr, len(scenarios), buf, 512), "tune_key")
    return buf.value.decode()


def autotune(scenarios, n_steps: int, cache: str | None = None, trial_steps: int = 12,
             device: torch.device | str | None = None) -> _lib.BatchOpts:
    """Rows per size class, depth, CTAs per SM and staging for this batch,
    from the JSON cache when it has the batch's key, else by timed trials
    (lpbf_b200_batch_autotune; stores the result when `cache` is given)."""
    arr, _keep = _host_array(scenarios, n_steps)
    out = _lib.BatchOpts()
    dev = torch.device(device) if device is not None else torch.device("cuda")
    with torch.cuda.device(dev):
        _lib.check(_lib.lib().lpbf_b200_batch_autotune(
            arr, len(scenarios), n_steps, cache.encode() if cache else None,
            min(trial_steps, n_steps), ctypes.byref(out)), "lpbf_b200_batch_autotune")
    return out


def opts_dict(o: _lib.BatchOpts) -> dict:
    return {"depth": o.depth, "ctas_per_sm": o.ctas_per_sm, "staging": o.staging,
            "rows": [o.rows[i] for i in range(4)]}


class Batch:
    """Device state and handle of one batched process map."""

    def __init__(self, scenarios: list[Scenario], n_steps: int | None = None, *,
                 opts: _lib.BatchOpts | None = None, device: torch.device | str | None = None,
                 rings: bool = True):
        if not scenarios:
            raise ValueError("empty batch")
        self.lib = _lib.lib()
        self.handle = None
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.n_steps = int(n_steps if n_steps is not None else len(scenarios[0].plan))
        self.scenarios = scenarios
        self.opts = opts if opts is not None else batch_opts()
        n = len(scenarios)
        self._k = [StepConst.from_buffer_copy(bytes(s.k)) for s in scenarios]
        self._plans = []
        self.fields = []
        self.rings = []
        arr = (_lib.Scenario * n)()
        for i, s in enumerate(scenarios):
            plan = np.ascontiguousarray(s.plan[: self.n_steps], dtype=TICK_DTYPE)
            if len(plan) < self.n_steps:
                raise ValueError(f"scenario {i}: plan has {len(plan)} < {self.n_steps} steps")
            self._plans.append(plan)
            k = self._k[i]
            shape = (k.ny, k.nx)
            pair = [torch.empty(shape, dtype=torch.float64, device=self.device) for _ in range(2)]
            self.fields.append(pair)
            ring = (torch.zeros(24 * max(self.n_steps, 1), dtype=torch.uint8, device=self.device)
                    if rings else None)
            self.rings.append(ring)
            arr[i].k = ctypes.pointer(k)
            arr[i].plan = plan.ctypes.data
            arr[i].T_a = pair[0].data_ptr()
            arr[i].T_b = pair[1].data_ptr()
            arr[i].ring = ring.data_ptr() if ring is not None else None
            arr[i].bc = s.bc
            arr[i].T_edge = s.T_edge
            arr[i].Tm = s.Tm
        self._arr = arr
        for i, s in enumerate(scenarios):
            self.set_field(i, s.T0 if s.T0 is not None else self._k[i].Tamb, which=0)
        nbytes = self.lib.lpbf_b200_batch_workspace_bytes(arr, n, self.n_steps,
                                                          ctypes.byref(self.opts))
        if nbytes == 0:
            raise ValueError("invalid batch (workspace size 0)")
        self.work = torch.empty(nbytes + 256, dtype=torch.uint8, device=self.device)
        self._work_ptr = (self.work.data_ptr() + 255) // 256 * 256
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_batch_create(
                arr, n, self.n_steps, ctypes.byref(self.opts), self._work_ptr, nbytes,
                _stream_handle(None), ctypes.byref(h)), "lpbf_b200_batch_create")
        self.handle = h

    # -- state ---------------------------------------------------------------
    @property
    def cur(self) -> int:
        """Buffer index (0: T_a, 1: T_b) holding the current fields."""
        if self.handle is None:
            return 0
        return self.lib.lpbf_b200_batch_result_in_b(self.handle)

    def set_field(self, i: int, T0, which: int | None = None) -> None:
        dst = self.fields[i][self.cur if which is None else which]
        if np.isscalar(T0):
            dst.fill_(float(T0))
        else:
            dst.copy_(torch.as_tensor(np.asarray(T0, dtype=np.float64).reshape(dst.shape)))

    def field(self, i: int) -> torch.Tensor:
        return self.fields[i][self.cur]

    def ring(self, i: int) -> np.ndarray:
        return self.rings[i].cpu().numpy().view(PARTIAL_DTYPE)

    def rows(self, i: int) -> int:
        return self.lib.lpbf_b200_batch_scenario_rows(self.handle, i)

    def tasks(self) -> int:
        return self.lib.lpbf_b200_batch_tasks(self.handle)

    def launches(self, n_steps: int) -> int:
        return self.lib.lpbf_b200_batch_launches(self.handle, n_steps)

    def cells(self) -> int:
        return sum(k.nx * k.ny for k in self._k)

    # -- execution -----------------------------------------------------------
    def run(self, first_step: int = 0, n_steps: int | None = None, use_graph: bool = False,
            stream: torch.cuda.Stream | None = None) -> None:
        n = self.n_steps - first_step if n_steps is None else n_steps
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_batch_run(self.handle, first_step, n, int(use_graph),
                                                    _stream_handle(stream)),
                       "lpbf_b200_batch_run")

    def capture(self, first_step: int = 0, n_steps: int | None = None) -> None:
        """Build the graph of these steps ahead of the first graph run."""
        n = self.n_steps - first_step if n_steps is None else n_steps
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_batch_capture(self.handle, first_step, n),
                       "lpbf_b200_batch_capture")

    def read_error(self) -> int:
        err = ctypes.c_uint(0)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_batch_read_error(self.handle, _stream_handle(None),
                                                           ctypes.byref(err)), "read_error")
        return err.value

    def close(self) -> None:
        if self.handle is not None:
            with torch.cuda.device(self.device):
                torch.cuda.synchronize()
                self.lib.lpbf_b200_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
