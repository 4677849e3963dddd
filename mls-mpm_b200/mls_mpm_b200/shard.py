"""Scene sharding across GPUs: one process per GPU, each advancing its own
share of independent scenes with no data-path collective (scenes never
exchange particles); the host side only assigns scenes and gathers results.

The reference runs one scene per page; this is the multi-GPU form of the
batched and served workloads.
"""
import heapq


def assign(costs, world_size, capacity=None):
    """Deterministic longest-processing-time assignment of items with the
    given costs (e.g. particle-updates) to `world_size` ranks.  With
    `capacity` (per-rank limit on the summed cost, e.g. device bytes) an item
    goes to the least-loaded rank that still has room; an item that fits no
    rank raises ValueError.  Returns the rank of every item."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world_size)]
    heapq.heapify(heap)
    out = [None] * len(costs)
    for i in order:
        popped = []
        while heap:
            load, r = heapq.heappop(heap)
            if capacity is None or load + costs[i] <= capacity:
                out[i] = r
                heapq.heappush(heap, (load + costs[i], r))
                break
            popped.append((load, r))
        for x in popped:
            heapq.heappush(heap, x)
        if out[i] is None:
            raise ValueError(f"item {i} (cost {costs[i]}) fits no rank")
    return out


def my_items(costs, world_size, rank, capacity=None):
    """Indices of the items rank `rank` owns under `assign`."""
    return [i for i, r in enumerate(assign(costs, world_size, capacity)) if r == rank]


def gather(obj, group=None):
    """Every rank's `obj` (a picklable result) on every rank, in rank order
    (torch.distributed all_gather_object over the default or given group);
    a single process returns [obj]."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return [obj]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out
