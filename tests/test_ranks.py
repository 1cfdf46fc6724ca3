# SPDX-License-Identifier: 0BSD
"""The benchmark's multi-process logic on CPU: two gloo ranks (127.0.0.1),
round-robin scenario shards, and timings reduced as the maximum over ranks
with unit counts summed (hedgehog_lpbf_b200.ranks)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from hedgehog_lpbf_b200.ranks import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from hedgehog_lpbf_b200 import process_map as PM
    from hedgehog_lpbf_b200.ranks import max_over_ranks, shard, sum_over_ranks, throughput
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard(13, rank, world)
        # every rank takes the same collective steps in the same order
        n_all = sum_over_ranks(len(mine))
        cells = sum(PM.draw(i).side ** 2 for i in mine)
        ms = 10.0 + 5.0 * rank                       # rank 1 is the slower one
        rate, ms_max = throughput(cells * 100, ms)
        slow = max_over_ranks(ms)
        out[rank] = (mine, n_all, rate, ms_max, slow)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn",
                       join=True)
    assert sorted(out.keys()) == [0, 1]
    shards = [out[r][0] for r in range(world)]
    assert sorted(shards[0] + shards[1]) == list(range(13))
    assert not set(shards[0]) & set(shards[1])
    from hedgehog_lpbf_b200 import process_map as PM
    total_cells = sum(PM.draw(i).side ** 2 for i in range(13))
    for r in range(world):
        _, n_all, rate, ms_max, slow = out[r]
        assert n_all == 13
        assert ms_max == slow == 15.0                # the slowest rank's time
        assert rate == pytest.approx(total_cells * 100 / 15e-3)


def test_shard_covers_everything_once():
    for world in (1, 2, 3, 8):
        got = sorted(i for r in range(world) for i in shard(256, r, world))
        assert got == list(range(256))
    assert shard(3, 5, 8) == []
    with pytest.raises(ValueError):
        shard(4, 2, 2)
