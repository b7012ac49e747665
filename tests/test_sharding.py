"""Multi-process host logic on CPU (two gloo ranks): the deterministic split of
independent systems over ranks and the max-over-ranks reduction of times."""
import os
import socket

import numpy as np
import pytest

from cie_b200.sharding import shard_by_weight


def test_shards_cover_every_item_once_and_balance():
    rng = np.random.default_rng(0)
    w = rng.integers(1, 1000, 512)
    for world in (1, 2, 3, 8):
        shards = [shard_by_weight(w, world, r) for r in range(world)]
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(w)))
        loads = [w[s].sum() for s in shards]
        assert max(loads) - min(loads) <= w.max()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from cie_b200.sharding import max_over_ranks, shard_by_weight
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        got = max_over_ranks([rank + 1.0, 10.0 - rank, 0.5])
        mine = shard_by_weight([5, 3, 3, 2, 1, 1], world, rank)
        out.put((rank, got, mine))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_shards_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    assert results[0][1] == results[1][1] == [2.0, 10.0, 0.5]
    shards = [r[2] for r in results]
    assert sorted(shards[0] + shards[1]) == list(range(6)) and not set(shards[0]) & set(shards[1])
