"""Work partitioning across ranks (one process per GPU).

The grid Fock builds of different molecules are independent, so a batch is
sharded by molecule with no data-path collective: every rank builds its own
share, and the only collectives are a barrier around the timed region and
the maximum of the ranks' times (torch.distributed, NCCL on GPUs, gloo on the
host).
"""


def shard_by_cost(costs, world):
    """Greedy longest-processing-time partition of items with the given costs
    over `world` ranks: items sorted by cost (descending, ties by index), each
    given to the currently least-loaded rank (ties by rank).  Returns a list
    of index lists, each in ascending order; deterministic."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def max_over_ranks(value, dist=None, device=None):
    """The maximum of `value` over all ranks (itself without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
