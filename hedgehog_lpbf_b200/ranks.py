# SPDX-License-Identifier: 0BSD
"""Multi-process plumbing of the benchmark: one process per GPU, independent
work per rank (no data-path collective), device-timed regions reduced as
the maximum over ranks.

* ``shard``: the scenarios of a process map dealt round-robin to ranks
  (scenario i on rank i mod world): every scenario exactly once.
* ``max_over_ranks`` / ``sum_over_ranks``: one all-reduce of a scalar (the
  only collectives; they carry timings and unit counts, never field data).
* ``throughput``: units of all ranks divided by the slowest rank's time.

The functions work with any torch.distributed backend (NCCL on the GPUs,
gloo in the CPU tests).
"""
from __future__ import annotations

import torch


def shard(n_items: int, rank: int, world: int) -> list[int]:
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"rank {rank} of {world}")
    return list(range(rank, n_items, world))


def _reduce(x: float, op, device=None) -> float:
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, device=None) -> float:
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x: float, device=None) -> float:
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, device)


def throughput(units_this_rank: float, ms_this_rank: float, device=None) -> tuple[float, float]:
    """(all ranks' units / the slowest rank's seconds, that slowest ms)."""
    ms = max_over_ranks(ms_this_rank, device)
    units = sum_over_ranks(units_this_rank, device)
    return units / (ms * 1e-3), ms
