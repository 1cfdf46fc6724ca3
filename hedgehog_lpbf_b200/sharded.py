# SPDX-License-Identifier: 0BSD
"""Row-strip sharding of one field: each strip (one per rank, or several in
one process) holds its owned rows plus `halo` rows of each neighbour, is
advanced `depth` steps per launch by ``lpbf_b200_advance_rows``, then trades
`halo` boundary rows with its neighbours.  The per-step Partials of the
strips combine by the reference's reduction rule (src/gpu/kernels.cu:205-262:
larger peak, equal peaks to the smaller flat index, NaN never wins, molten
rows min/max) into the whole field's; fields and Partials equal a
single-field ``Solver`` run bit for bit.

Transport: ``DistExchange`` sends and receives the boundary rows with
torch.distributed point-to-point operations (NCCL over NVLink between GPUs,
gloo between CPU processes); ``LocalExchange`` copies them between strips
that live in one process.  Halo rows are contiguous in the row-major
buffers, so each exchange is one message per neighbour and direction.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .params import StepConst
from .plan import TICK_DTYPE
from .solver import PARTIAL_DTYPE, _stream_handle


def split_rows(ny: int, parts: int) -> list[tuple[int, int]]:
    """Balanced contiguous row ranges [a, b) of `parts` strips (the first
    ny % parts strips one row longer)."""
    if parts < 1 or ny < parts:
        raise ValueError(f"cannot split {ny} rows into {parts} strips")
    q, r = divmod(ny, parts)
    out, a = [], 0
    for i in range(parts):
        b = a + q + (1 if i < r else 0)
        out.append((a, b))
        a = b
    return out


@dataclass(frozen=True)
class Strip:
    """Field rows [a, b) owned; `top`/`bot` halo rows held above/below (zero
    at the field's edges).  Buffer row 0 is field row a - top."""
    a: int
    b: int
    top: int
    bot: int

    @property
    def row0(self) -> int:
        return self.a - self.top

    @property
    def rows(self) -> int:
        return self.top + (self.b - self.a) + self.bot

    @property
    def lo(self) -> int:
        return self.top

    @property
    def hi(self) -> int:
        return self.top + (self.b - self.a)


def strip_layout(ny: int, parts: int, halo: int) -> list[Strip]:
    """Strips of a field of ny rows with `halo` rows from each neighbour."""
    ranges = split_rows(ny, parts)
    if parts > 1 and min(b - a for a, b in ranges) < halo:
        raise ValueError(f"strips of {ny // parts} rows cannot feed a halo of {halo}")
    return [Strip(a, b, halo if i > 0 else 0, halo if i < parts - 1 else 0)
            for i, (a, b) in enumerate(ranges)]


def combine_partials(rings, nx: int, ny: int) -> np.ndarray:
    """Per-step combination of strip Partials (PARTIAL_DTYPE arrays of equal
    length) into the field's, by the reduction's rule."""
    rings = [np.asarray(r).view(PARTIAL_DTYPE) for r in rings]
    n = len(rings[0])
    out = np.zeros(n, dtype=PARTIAL_DTYPE)
    out["tmax"] = -1.0
    out["arg"] = nx * ny
    out["ymin"] = ny
    out["ymax"] = -1
    for r in rings:
        t, a = r["tmax"], r["arg"]
        # t > best, or an equal peak at a smaller flat index (NaN compares false)
        take = (t > out["tmax"]) | ((t == out["tmax"]) & (a < out["arg"]))
        out["tmax"] = np.where(take, t, out["tmax"])
        out["arg"] = np.where(take, a, out["arg"])
        out["ymin"] = np.minimum(out["ymin"], r["ymin"])
        out["ymax"] = np.maximum(out["ymax"], r["ymax"])
    return out


def strip_const(k: StepConst, strip: Strip) -> StepConst:
    """The field's constants with ny = the strip buffer's rows."""
    ks = StepConst.from_buffer_copy(bytes(k))
    ks.ny = strip.rows
    return ks


class CudaStripStepper:
    """One launch of lpbf_b200_advance_rows per call, with its own workspace."""

    def __init__(self, device: torch.device, *, bc: int = 0, T_edge: float = 300.0,
                 Tm: float = 1609.0, rows: int = 0):
        self.lib = _lib.lib()
        self.device = device
        self.opts = _lib.Opts(phys=0, bc=bc, T_edge=T_edge, Tm=Tm, depth=0, rows=rows)
        nbytes = self.lib.lpbf_b200_workspace_bytes()
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=device)
        with torch.cuda.device(device):
            _lib.check(self.lib.lpbf_b200_workspace_init(self.work.data_ptr(), nbytes,
                                                         _stream_handle(None)), "workspace_init")

    def __call__(self, T_in: torch.Tensor, T_out: torch.Tensor, ks: StepConst, gny: int,
                 strip: Strip, plan: np.ndarray, ring: torch.Tensor | None) -> None:
        plan = np.ascontiguousarray(plan, dtype=TICK_DTYPE)
        rw = _lib.Rows(row0=strip.row0, global_ny=gny, lo=strip.lo, hi=strip.hi)
        with torch.cuda.device(self.device):
            st = self.lib.lpbf_b200_advance_rows(
                T_in.data_ptr(), T_out.data_ptr(), ctypes.byref(ks), plan.ctypes.data, len(plan),
                ctypes.byref(self.opts), ctypes.byref(rw),
                ring.data_ptr() if ring is not None else None, self.work.data_ptr(),
                self.work.numel(), _stream_handle(None))
        _lib.check(st, "lpbf_b200_advance_rows")

    def read_error(self) -> int:
        err = ctypes.c_uint(0)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_read_error(self.work.data_ptr(), _stream_handle(None),
                                                     ctypes.byref(err)), "read_error")
        return err.value


class LocalExchange:
    """Boundary rows between adjacent strips held by this process (bufs[i]
    is strip i's current buffer, a (rows, nx) tensor)."""

    def __call__(self, strips: list[Strip], bufs: list[torch.Tensor], halo: int) -> None:
        for i in range(len(strips) - 1):
            up, dn = strips[i], strips[i + 1]
            # up's last owned rows -> dn's top halo; dn's first owned rows -> up's bottom halo
            bufs[i + 1][dn.lo - halo:dn.lo].copy_(bufs[i][up.hi - halo:up.hi])
            bufs[i][up.hi:up.hi + halo].copy_(bufs[i + 1][dn.lo:dn.lo + halo])


class DistExchange:
    """Boundary rows with the neighbouring ranks (rank i holds strip i):
    one send and one receive per neighbour, posted together."""

    def __init__(self, rank: int, world: int, group=None):
        self.rank, self.world, self.group = rank, world, group

    def __call__(self, strips: list[Strip], bufs: list[torch.Tensor], halo: int) -> None:
        import torch.distributed as dist
        (s,), (buf,) = strips, bufs
        ops = []
        # row ranges of a row-major (rows, nx) buffer are contiguous views
        if self.rank > 0:
            ops.append(dist.P2POp(dist.isend, buf[s.lo:s.lo + halo], self.rank - 1, self.group))
            ops.append(dist.P2POp(dist.irecv, buf[s.lo - halo:s.lo], self.rank - 1, self.group))
        if self.rank < self.world - 1:
            ops.append(dist.P2POp(dist.isend, buf[s.hi - halo:s.hi], self.rank + 1, self.group))
            ops.append(dist.P2POp(dist.irecv, buf[s.hi:s.hi + halo], self.rank + 1, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


class ShardedField:
    """The strips of one field that this process holds, advanced together.

    ``local(...)``: every strip in this process (strips exchange by copies);
    ``distributed(...)``: strip `rank` of `world`, one per rank.  `depth`
    steps per launch, and as many halo rows per side.  `stepper` advances
    one strip by one launch (default: the CUDA kernel).  With the CUDA
    kernel, the local form gives each strip its own stepper (workspace) and
    stream, so the strips' launches overlap one another's start and tail;
    the boundary rows are exchanged once all of a step's launches are done."""

    def __init__(self, k: StepConst, layout: list[Strip], mine: list[int], exchange,
                 stepper, *, depth: int, device: torch.device, T0=None, gather_fn=None):
        if not 1 <= depth <= 4:
            raise ValueError("depth must be 1..4")
        self.k = StepConst.from_buffer_copy(bytes(k))
        self.nx, self.ny = k.nx, k.ny
        self.layout, self.mine = layout, mine
        self.strips = [layout[i] for i in mine]
        self.exchange, self.stepper = exchange, stepper
        self.steppers = None               # per-strip steppers on their own streams
        self._streams = None
        self.depth = self.halo = depth
        self.device = device
        self._gather_fn = gather_fn
        self.ks = [strip_const(self.k, s) for s in self.strips]
        self.bufs = [[torch.empty((s.rows, self.nx), dtype=torch.float64, device=device)
                      for _ in range(2)] for s in self.strips]
        self.cur = 0
        self.set_field(k.Tamb if T0 is None else T0)

    # -- construction --------------------------------------------------------
    @classmethod
    def local(cls, k: StepConst, parts: int, *, depth: int = 3, device=None, T0=None,
              stepper=None, **opts) -> "ShardedField":
        dev = torch.device(device) if device is not None else torch.device("cuda")
        layout = strip_layout(k.ny, parts, depth)
        if stepper is not None:
            return cls(k, layout, list(range(parts)), LocalExchange(), stepper, depth=depth,
                       device=dev, T0=T0)
        steps = [CudaStripStepper(dev, **opts) for _ in range(parts)]
        f = cls(k, layout, list(range(parts)), LocalExchange(), steps[0], depth=depth,
                device=dev, T0=T0)
        if parts > 1:
            f.steppers = steps
            f._streams = [torch.cuda.Stream(device=dev) for _ in range(parts)]
        return f

    @classmethod
    def distributed(cls, k: StepConst, rank: int, world: int, *, depth: int = 3, device=None,
                    T0=None, group=None, stepper=None, **opts) -> "ShardedField":
        dev = torch.device(device) if device is not None else torch.device("cuda")
        layout = strip_layout(k.ny, world, depth)
        step = stepper if stepper is not None else CudaStripStepper(dev, **opts)
        return cls(k, layout, [rank], DistExchange(rank, world, group), step, depth=depth,
                   device=dev, T0=T0, gather_fn=_DistGather(rank, world, group))

    # -- state ---------------------------------------------------------------
    def set_field(self, T0) -> None:
        """Scalar, or the whole (ny, nx) field (every strip takes its rows,
        halo included)."""
        for s, pair in zip(self.strips, self.bufs):
            dst = pair[self.cur]
            if np.isscalar(T0):
                dst.fill_(float(T0))
            else:
                full = np.asarray(T0, dtype=np.float64).reshape(self.ny, self.nx)
                dst.copy_(torch.as_tensor(full[s.row0:s.row0 + s.rows]))

    def owned(self, i: int) -> torch.Tensor:
        """Owned rows of this process's i-th strip (current values)."""
        s = self.strips[i]
        return self.bufs[i][self.cur][s.lo:s.hi]

    def field(self) -> torch.Tensor:
        """The whole current field (collective in the distributed form)."""
        if self._gather_fn is not None:
            return self._gather_fn(self.owned(0), self.layout)
        return torch.cat([self.owned(i) for i in range(len(self.strips))], 0)

    # -- execution -----------------------------------------------------------
    def advance(self, plan: np.ndarray, rings: bool = True) -> list[torch.Tensor] | None:
        """Advance every strip along the plan; returns each strip's ring of
        per-step Partials (uint8 tensors, 24 bytes per step) or None."""
        plan = np.ascontiguousarray(plan, dtype=TICK_DTYPE)
        n = len(plan)
        out = ([torch.zeros(24 * max(n, 1), dtype=torch.uint8, device=self.device)
                for _ in self.strips] if rings else None)
        for s0 in range(0, n, self.depth):
            kk = min(self.depth, n - s0)
            if self._streams is not None:
                main = torch.cuda.current_stream(self.device)
                start = main.record_event()
                done = []
                for i, s in enumerate(self.strips):
                    st = self._streams[i]
                    st.wait_event(start)
                    ring = out[i][24 * s0:24 * (s0 + kk)] if rings else None
                    with torch.cuda.stream(st):
                        self.steppers[i](self.bufs[i][self.cur], self.bufs[i][1 - self.cur],
                                         self.ks[i], self.ny, s, plan[s0:s0 + kk], ring)
                        done.append(st.record_event())
                for e in done:
                    main.wait_event(e)
            else:
                for i, s in enumerate(self.strips):
                    ring = out[i][24 * s0:24 * (s0 + kk)] if rings else None
                    self.stepper(self.bufs[i][self.cur], self.bufs[i][1 - self.cur], self.ks[i],
                                 self.ny, s, plan[s0:s0 + kk], ring)
            self.cur = 1 - self.cur
            self.exchange(self.strips, [pair[self.cur] for pair in self.bufs], self.halo)
        return out

    def read_error(self) -> int:
        """The error words of this process's strip launches, or-ed."""
        err = 0
        for st in (self.steppers or [self.stepper]):
            err |= st.read_error()
        return err

    def partials(self, rings: list[torch.Tensor]) -> np.ndarray:
        """The field's per-step Partials from the strips' rings (collective
        in the distributed form)."""
        if self._gather_fn is not None:
            all_rings = self._gather_fn.rings(rings[0])
        else:
            all_rings = [r.cpu().numpy() for r in rings]
        return combine_partials(all_rings, self.nx, self.ny)


class _DistGather:
    """Collectives of the distributed form: every rank receives the field
    (owned rows padded to the longest strip) or every strip's ring."""

    def __init__(self, rank: int, world: int, group=None):
        self.rank, self.world, self.group = rank, world, group

    def __call__(self, owned: torch.Tensor, layout: list[Strip]) -> torch.Tensor:
        import torch.distributed as dist
        h = max(s.b - s.a for s in layout)
        pad = torch.zeros((h, owned.shape[1]), dtype=owned.dtype, device=owned.device)
        pad[:owned.shape[0]].copy_(owned)
        parts = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(parts, pad, group=self.group)
        return torch.cat([p[:s.b - s.a] for p, s in zip(parts, layout)], 0)

    def rings(self, ring: torch.Tensor) -> list[np.ndarray]:
        import torch.distributed as dist
        parts = [torch.empty_like(ring) for _ in range(self.world)]
        dist.all_gather(parts, ring.contiguous(), group=self.group)
        return [p.cpu().numpy() for p in parts]


__all__ = ["split_rows", "Strip", "strip_layout", "combine_partials", "strip_const",
           "CudaStripStepper", "LocalExchange", "DistExchange", "ShardedField"]
