"""Host-side helpers for runs over several processes, one per GPU (torchrun).

The linear-solve path shards only where its units are independent: the systems
of a batched solve are dealt out to the ranks by nonzero count, each rank solves
its own systems with no exchange in the data path, and the only collective is
the max over ranks of the measured times."""
import numpy as np

__all__ = ["shard_by_weight", "max_over_ranks"]


def shard_by_weight(weights, world, rank):
    """Indices (ascending) of the items rank `rank` of `world` takes: largest
    weight first, each to the least-loaded rank (ties to the lower rank), so every
    rank computes the same deterministic split and the heaviest load exceeds the
    lightest by at most the largest single weight."""
    weights = np.asarray(weights, dtype=np.float64)
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        load[r] += weights[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def max_over_ranks(values):
    """Element-wise max of a list of floats over the ranks of the default process
    group (the values themselves when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()
