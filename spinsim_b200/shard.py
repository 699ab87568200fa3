"""Multi-GPU sharding of instance batches (one process per GPU, torch.distributed).

Instances are independent (each is one evaluate() call), so a batch shards across GPUs with no
collective on the data path: ``partition`` assigns instances to ranks by work (integration steps,
longest first onto the least-loaded rank, so ranks finish together), every rank runs its share as
one persistent launch, and ``gather_final_states`` collects a small per-instance summary (the final
state) on rank 0 when asked.  The weak-scaling benchmark (bench.py under torchrun) instead gives
every rank its own full batch.
"""
import heapq

import numpy as np


def work(instance):
    n = max(0, int((float(instance.time_end) - float(instance.time_start)) / float(instance.time_step_output)))
    k = int(np.floor(float(instance.time_step_output) / float(instance.time_step_integration) + 0.5))
    return n * max(k, 1) * (4 if instance.spin.dimension == 3 else 1)


def partition(instances, world_size):
    """List of index lists, one per rank: longest-processing-time-first onto the least-loaded rank."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(instances)), key=lambda i: -work(instances[i]))
    heap = [(0, r) for r in range(world_size)]
    out = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + work(instances[i]), r))
    for lst in out:
        lst.sort()
    return out


def run_shard(instances, rank, world_size, **batch_kwargs):
    """Run this rank's share; returns (indices, Batch or None)."""
    from .batch import Batch
    mine = partition(instances, world_size)[rank]
    if not mine:
        return mine, None
    b = Batch([instances[i] for i in mine], **batch_kwargs)
    b.run()
    return mine, b


def gather_final_states(indices, finals, n_total, group=None):
    """Collect every rank's (index, final state) on all ranks; returns a list of length n_total
    (complex arrays).  Uses all_gather_object: a small host-side exchange, not a data-path collective."""
    import torch.distributed as dist
    mine = [(int(i), np.asarray(f)) for i, f in zip(indices, finals)]
    world = dist.get_world_size(group)
    bucket = [None] * world
    dist.all_gather_object(bucket, mine, group=group)
    out = [None] * n_total
    for part in bucket:
        for i, f in part:
            out[i] = f
    return out
