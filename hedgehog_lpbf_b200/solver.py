# SPDX-License-Identifier: 0BSD
"""Python host API over the C-ABI: a device-resident field that advances
along a laser plan.

PyTorch provides device memory and streams only; every kernel runs in
liblpbf_b200.so through ``lpbf_b200_advance``.  The per-step results are the
reference's ``Partial`` records (peak T, argmax flat index with smallest-index
ties, molten row extent), as produced by the reference's reduce + finalize
(src/gpu/kernels.cu:205-262).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .params import StepConst
from .plan import TICK_DTYPE

PARTIAL_DTYPE = np.dtype({"names": ["tmax", "arg", "ymin", "ymax"],
                          "formats": [np.float64, np.int64, np.int32, np.int32],
                          "offsets": [0, 8, 16, 20], "itemsize": 24})


def _stream_handle(stream: torch.cuda.Stream | None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def ring_to_numpy(ring: torch.Tensor) -> np.ndarray:
    """Device ring (uint8 tensor) -> numpy PARTIAL_DTYPE array."""
    return ring.cpu().numpy().view(PARTIAL_DTYPE)


class Solver:
    """Two device fields (ping-pong), the workspace and the metric ring of one
    simulation.  ``advance`` runs a plan slice; ``field`` is the current field.

    depth: time steps per launch (temporal blocking), 0 = automatic.
    bc: 0 zero-flux mirror edges (the reference's), 1 fixed edges at T_edge.
    """

    def __init__(self, k: StepConst, *, phys: int = 0, bc: int = 0, T_edge: float = 300.0,
                 Tm: float = 1609.0, depth: int = 0, rows: int = 0,
                 device: torch.device | str | None = None, T0: float | np.ndarray | None = None):
        self.lib = _lib.lib()
        self.k = StepConst.from_buffer_copy(bytes(k))
        self.nx, self.ny = k.nx, k.ny
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.opts = _lib.Opts(phys=phys, bc=bc, T_edge=T_edge, Tm=Tm, depth=depth, rows=rows)
        shape = (self.ny, self.nx)
        self.bufs = [torch.empty(shape, dtype=torch.float64, device=self.device),
                     torch.empty(shape, dtype=torch.float64, device=self.device)]
        self.cur = 0
        nbytes = self.lib.lpbf_b200_workspace_bytes()
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_workspace_init(
                self.work.data_ptr(), nbytes, _stream_handle(None)), "workspace_init")
        if T0 is None:
            T0 = k.Tamb
        self.set_field(T0)

    @property
    def field(self) -> torch.Tensor:
        return self.bufs[self.cur]

    def set_field(self, T0) -> None:
        """A scalar, a host array, or a tensor (a device tensor is copied on
        the device, stream-ordered, with no host synchronization)."""
        if np.isscalar(T0):
            self.bufs[self.cur].fill_(float(T0))
        elif isinstance(T0, torch.Tensor):
            self.bufs[self.cur].copy_(T0.reshape(self.ny, self.nx))
        else:
            src = torch.as_tensor(np.asarray(T0, dtype=np.float64).reshape(self.ny, self.nx))
            self.bufs[self.cur].copy_(src)

    def new_ring(self, n_steps: int) -> torch.Tensor:
        return torch.zeros(n_steps * 24, dtype=torch.uint8, device=self.device)

    def launches(self, n_steps: int) -> int:
        return self.lib.lpbf_b200_advance_launches(self.nx, self.ny, n_steps,
                                                   ctypes.byref(self.opts))

    def advance(self, plan: np.ndarray, ring: torch.Tensor | None = None,
                stream: torch.cuda.Stream | None = None) -> torch.Tensor:
        """Advance by len(plan) steps (plan: TICK_DTYPE array on the host).
        ring: uint8 device tensor of >= 24*len(plan) bytes, or None."""
        plan = np.ascontiguousarray(plan, dtype=TICK_DTYPE)
        n = len(plan)
        if ring is not None and ring.numel() < 24 * n:
            raise ValueError("ring too small")
        in_b = ctypes.c_int(0)
        a = self.bufs[self.cur]
        b = self.bufs[1 - self.cur]
        with torch.cuda.device(self.device):
            st = self.lib.lpbf_b200_advance(
                a.data_ptr(), b.data_ptr(), ctypes.byref(self.k),
                plan.ctypes.data if n else None, n, ctypes.byref(self.opts),
                ring.data_ptr() if ring is not None else None,
                self.work.data_ptr(), self.work.numel(), _stream_handle(stream),
                ctypes.byref(in_b))
        _lib.check(st, "lpbf_b200_advance")
        if in_b.value:
            self.cur = 1 - self.cur
        return self.field

    def read_error(self) -> int:
        err = ctypes.c_uint(0)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_read_error(self.work.data_ptr(), _stream_handle(None),
                                                     ctypes.byref(err)), "read_error")
        return err.value

    def run(self, T0_host: np.ndarray, plan: np.ndarray, pinned_out: np.ndarray | None = None):
        """End-to-end call on host data: copy T0 in, advance along the plan,
        copy the final field and the per-step Partials out."""
        self.set_field(T0_host)
        ring = self.new_ring(len(plan))
        self.advance(plan, ring)
        T = self.field.cpu().numpy()
        return T, ring_to_numpy(ring)

    def run_many(self, inputs, plans, outputs, rings_out=None) -> None:
        """Independent runs streamed through this solver: run i starts from
        inputs[i] (host (ny, nx) float64 tensors, pinned for overlap), follows
        plans[i] and leaves its final field in outputs[i] (and its per-step
        Partials in rings_out[i], host uint8 tensors of 24 bytes per step).

        The copies go on a copy stream through two device staging slots:
        run i+1's field is copied in, and run i-1's result copied out, while
        run i computes, so the host link is busy only at the ends of the
        sequence.  Returns when every output has arrived."""
        n = len(inputs)
        if len(plans) != n or len(outputs) != n or (rings_out is not None and len(rings_out) != n):
            raise ValueError("inputs, plans and outputs must have the same length")
        if n == 0:
            return
        dev = self.device
        comp = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(device=dev)
        shape = (self.ny, self.nx)
        s_in = [torch.empty(shape, dtype=torch.float64, device=dev) for _ in range(2)]
        s_out = [torch.empty(shape, dtype=torch.float64, device=dev) for _ in range(2)]
        rings = [self.new_ring(max(len(p) for p in plans) or 1) for _ in range(2)]
        ev = lambda: torch.cuda.Event()                               # noqa: E731
        in_ready = [ev() for _ in range(n)]      # staging slot filled (copy stream)
        in_free = [ev() for _ in range(n)]       # staging slot consumed (compute stream)
        out_ready = [ev() for _ in range(n)]     # result staged (compute stream)
        out_free = [ev() for _ in range(n)]      # result copied out (copy stream)

        def copy_in(i):
            with torch.cuda.stream(copy):
                if i >= 2:
                    copy.wait_event(in_free[i - 2])
                s_in[i % 2].copy_(torch.as_tensor(inputs[i]).reshape(shape), non_blocking=True)
                in_ready[i].record(copy)

        def copy_out(i):
            with torch.cuda.stream(copy):
                copy.wait_event(out_ready[i])
                outputs[i].copy_(s_out[i % 2], non_blocking=True)
                if rings_out is not None:
                    rings_out[i].copy_(rings[i % 2][:rings_out[i].numel()], non_blocking=True)
                out_free[i].record(copy)

        copy_in(0)
        for i in range(n):
            if i + 1 < n:
                copy_in(i + 1)
            comp.wait_event(in_ready[i])
            self.bufs[self.cur].copy_(s_in[i % 2])
            in_free[i].record(comp)
            if i >= 2:
                comp.wait_event(out_free[i - 2])
            self.advance(plans[i], rings[i % 2])
            s_out[i % 2].copy_(self.field)
            out_ready[i].record(comp)
            copy_out(i)
        torch.cuda.current_stream(dev).wait_stream(copy)
        torch.cuda.synchronize(dev)


class SolverF32K:
    """The FP32 compensated field (hi + lo f32 pairs) with the same plan API
    as Solver; ``field64()`` returns hi + lo in FP64."""

    def __init__(self, k: StepConst, *, bc: int = 0, T_edge: float = 300.0, Tm: float = 1609.0,
                 depth: int = 0, rows: int = 0, device: torch.device | str | None = None,
                 T0: float | np.ndarray | None = None):
        self.lib = _lib.lib()
        self.k = StepConst.from_buffer_copy(bytes(k))
        self.nx, self.ny = k.nx, k.ny
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.opts = _lib.Opts(phys=0, bc=bc, T_edge=T_edge, Tm=Tm, depth=depth, rows=rows)
        n = self.nx * self.ny
        self.hi = [torch.empty(n, dtype=torch.float32, device=self.device) for _ in range(2)]
        self.lo = [torch.empty(n, dtype=torch.float32, device=self.device) for _ in range(2)]
        self.cur = 0
        nbytes = self.lib.lpbf_b200_workspace_bytes()
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_workspace_init(self.work.data_ptr(), nbytes,
                                                         _stream_handle(None)), "workspace_init")
        self.set_field(k.Tamb if T0 is None else T0)

    def set_field(self, T0) -> None:
        n = self.nx * self.ny
        if np.isscalar(T0):
            src = torch.full((n,), float(T0), dtype=torch.float64, device=self.device)
        else:
            src = torch.as_tensor(np.asarray(T0, dtype=np.float64).ravel()).to(self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_f32k_split(src.data_ptr(), self.hi[self.cur].data_ptr(),
                                                     self.lo[self.cur].data_ptr(), n,
                                                     _stream_handle(None)), "f32k_split")

    def new_ring(self, n_steps: int) -> torch.Tensor:
        return torch.zeros(n_steps * 24, dtype=torch.uint8, device=self.device)

    def advance(self, plan: np.ndarray, ring: torch.Tensor | None = None,
                stream: torch.cuda.Stream | None = None) -> None:
        plan = np.ascontiguousarray(plan, dtype=TICK_DTYPE)
        n = len(plan)
        in_b = ctypes.c_int(0)
        a, b = self.cur, 1 - self.cur
        with torch.cuda.device(self.device):
            st = self.lib.lpbf_b200_advance_f32k(
                self.hi[a].data_ptr(), self.lo[a].data_ptr(), self.hi[b].data_ptr(),
                self.lo[b].data_ptr(), ctypes.byref(self.k), plan.ctypes.data if n else None, n,
                ctypes.byref(self.opts), ring.data_ptr() if ring is not None else None,
                self.work.data_ptr(), self.work.numel(), _stream_handle(stream),
                ctypes.byref(in_b))
        _lib.check(st, "lpbf_b200_advance_f32k")
        if in_b.value:
            self.cur = 1 - self.cur

    def field64(self) -> torch.Tensor:
        n = self.nx * self.ny
        out = torch.empty(n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_f32k_join(self.hi[self.cur].data_ptr(),
                                                    self.lo[self.cur].data_ptr(), out.data_ptr(),
                                                    n, _stream_handle(None)), "f32k_join")
        return out.view(self.ny, self.nx)


class SolverF32:
    """The plain FP32 field (one f32 array, each step's update rounded once)
    with the same plan API as Solver; ``field`` is the f32 field and
    ``field64()`` its FP64 copy."""

    def __init__(self, k: StepConst, *, bc: int = 0, T_edge: float = 300.0, Tm: float = 1609.0,
                 depth: int = 0, rows: int = 0, device: torch.device | str | None = None,
                 T0: float | np.ndarray | None = None):
        self.lib = _lib.lib()
        self.k = StepConst.from_buffer_copy(bytes(k))
        self.nx, self.ny = k.nx, k.ny
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.opts = _lib.Opts(phys=0, bc=bc, T_edge=T_edge, Tm=Tm, depth=depth, rows=rows)
        n = self.nx * self.ny
        self.bufs = [torch.empty(n, dtype=torch.float32, device=self.device) for _ in range(2)]
        self.cur = 0
        nbytes = self.lib.lpbf_b200_workspace_bytes()
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_workspace_init(self.work.data_ptr(), nbytes,
                                                         _stream_handle(None)), "workspace_init")
        self.set_field(k.Tamb if T0 is None else T0)

    def set_field(self, T0) -> None:
        if np.isscalar(T0):
            self.bufs[self.cur].fill_(float(T0))
        else:
            src = torch.as_tensor(np.asarray(T0, dtype=np.float64).ravel()).to(self.device)
            self.bufs[self.cur].copy_(src)        # rounded to nearest

    @property
    def field(self) -> torch.Tensor:
        return self.bufs[self.cur].view(self.ny, self.nx)

    def field64(self) -> torch.Tensor:
        return self.field.double()

    def new_ring(self, n_steps: int) -> torch.Tensor:
        return torch.zeros(n_steps * 24, dtype=torch.uint8, device=self.device)

    def read_error(self) -> int:
        err = ctypes.c_uint(0)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_read_error(self.work.data_ptr(), _stream_handle(None),
                                                     ctypes.byref(err)), "read_error")
        return err.value

    def advance(self, plan: np.ndarray, ring: torch.Tensor | None = None,
                stream: torch.cuda.Stream | None = None) -> None:
        plan = np.ascontiguousarray(plan, dtype=TICK_DTYPE)
        n = len(plan)
        in_b = ctypes.c_int(0)
        a, b = self.cur, 1 - self.cur
        with torch.cuda.device(self.device):
            st = self.lib.lpbf_b200_advance_f32(
                self.bufs[a].data_ptr(), self.bufs[b].data_ptr(), ctypes.byref(self.k),
                plan.ctypes.data if n else None, n, ctypes.byref(self.opts),
                ring.data_ptr() if ring is not None else None, self.work.data_ptr(),
                self.work.numel(), _stream_handle(stream), ctypes.byref(in_b))
        _lib.check(st, "lpbf_b200_advance_f32")
        if in_b.value:
            self.cur = 1 - self.cur
