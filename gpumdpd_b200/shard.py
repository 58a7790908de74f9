"""Replica and job sharding over ranks (one process per GPU): the host-side scheduler of a
batched sweep or a job list run on several GPUs.

Replicas (or served jobs) are independent, so they are spread over the ranks with no
exchange on the step path: `assign` is a longest-processing-time split of the units by
their cost (particles x steps), the same on every rank; each rank runs its own share
(one packed batch per rank) and `gather` brings the per-unit results together on every
rank (torch.distributed all_gather_object: host objects, gloo or NCCL).  The reference
runs one system on device 0 only (src/main/utils.cuh:52-53).
"""
import heapq


def assign(costs, world):
    """Unit indices of each rank: units sorted by decreasing cost (ties by index), each
    given to the least-loaded rank (ties by rank).  Deterministic, so every rank computes
    the same split without communicating."""
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(world)]
    shares = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(s) for s in shares]


def gather(local, world):
    """Merge every rank's {unit index: result} into one list ordered by unit index."""
    if world == 1:
        merged = dict(local)
    else:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, local)
        merged = {}
        for p in parts:
            merged.update(p)
    return [merged[k] for k in sorted(merged)]


def run_sharded(units, costs, fn, world, rank):
    """Run fn(list of this rank's units) -> {unit index: result} on this rank's share and
    gather every rank's results, ordered by unit index."""
    mine = assign(costs, world)[rank]
    local = fn(mine) if mine else {}
    return gather(local, world)
