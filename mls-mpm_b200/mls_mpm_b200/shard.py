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


def scene_cost(scene, substeps):
    """Particle-updates of `substeps` substeps of a scene: what a rank's share
    costs on the device (the substep is bound per particle)."""
    return int(scene.n) * int(substeps)


class ShardedBatch:
    """This rank's share of a list of independent scenes, advanced as one
    batch on this rank's GPU (the multi-GPU form of the batched workload).

    Scenes are assigned by `assign` on their particle-updates, so every rank
    computes the same assignment without communicating; `gather_results`
    brings every rank's per-scene results to every rank, keyed by the scene's
    index in the full list.  `make_batch(particle_capacity, cell_capacity,
    scene_capacity)` builds the batch (mls_mpm_b200.batch.Batch on the
    device; any object with add_scene/step/sync/read works)."""

    def __init__(self, scene_list, substeps, world_size, rank, make_batch=None, params=None):
        if make_batch is None:
            from .batch import Batch

            def make_batch(p, c, s):
                return Batch(p, c, s)
        self.scenes = scene_list
        self.rank = rank
        self.mine = my_items([scene_cost(s, substeps) for s in scene_list], world_size, rank)
        local = [scene_list[i] for i in self.mine]
        self.particles = sum(s.n for s in local)
        self.cells = sum(s.cells for s in local)
        self.batch = make_batch(max(1, self.particles), max(1, self.cells), max(1, len(local)))
        self.ids = {}
        for i in self.mine:
            p = params(scene_list[i]) if params is not None else None
            self.ids[i] = self.batch.add_scene(scene_list[i], params=p)

    def step(self, substeps):
        self.batch.step(substeps)

    def sync(self):
        self.batch.sync()

    def local_results(self, fn):
        """{scene index: fn(batch, scene id)} for this rank's scenes."""
        return {i: fn(self.batch, sid) for i, sid in self.ids.items()}

    def gather_results(self, fn, group=None):
        """Every rank's local_results(fn) merged, on every rank."""
        merged = {}
        for part in gather(self.local_results(fn), group):
            merged.update(part)
        return merged


def shard_jobs(jobs, world_size, rank):
    """Indices of the served jobs [(scene, substeps), ...] this rank runs
    (assigned on particle-updates; arrival order is kept within a rank)."""
    return my_items([scene_cost(sc, k) for sc, k in jobs], world_size, rank)
