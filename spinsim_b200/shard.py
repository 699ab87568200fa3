"""Multi-GPU sharding (one process per GPU, torch.distributed).

Many instances: instances are independent (each is one evaluate() call), so a batch shards across
GPUs with no collective on the data path: ``partition`` assigns instances to ranks by work
(integration steps, longest first onto the least-loaded rank, so ranks finish together), every
rank runs its share as one persistent launch, and ``gather_final_states`` collects a small
per-instance summary (the final state) when asked.  The weak-scaling benchmark (bench.py under
torchrun) instead gives every rank its own full batch.

One long instance: its output steps are independent too, and only the state needs the steps
before it.  ``evaluate_split`` gives each rank a piece of consecutive output steps (``Piece``):
the rank computes the piece's operators (time indices of the whole call, so every operator and
time is the one the unsplit call computes), the piece's product P_r = U[last] ... U[first], and
after ONE exchange of the d x d products (``exchange_products``: an all-gather of 64 or 144 bytes
per rank) the state entering its piece, P_{r-1} ... P_0 psi0, from which it scans its own states.
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


# ------------------------------------------------------------------ one instance over several ranks
def piece_ranges(n_out, pieces):
    """(first, count) of ``pieces`` consecutive runs of output steps covering 0 .. n_out - 1."""
    if pieces < 1:
        raise ValueError("pieces must be >= 1")
    cuts = [(n_out * r) // pieces for r in range(pieces + 1)]
    return [(cuts[r], cuts[r + 1] - cuts[r]) for r in range(pieces)]


def incoming_states(products, psi0):
    """States entering each piece: psi_in[0] = psi0, psi_in[r] = P_{r-1} ... P_0 psi0 (FP64)."""
    v = np.asarray(psi0, np.complex128).reshape(-1)
    out = []
    for p in products:
        out.append(v.copy())
        v = np.asarray(p, np.complex128) @ v
    return out


def exchange_products(product, group=None):
    """All-gather every rank's d x d piece product (a complex128 tensor on this rank's device; NCCL
    between GPUs, gloo on the host); returns the products in rank order as numpy arrays."""
    import torch
    import torch.distributed as dist
    mine = torch.view_as_real(product.contiguous()).contiguous()
    bucket = [torch.empty_like(mine) for _ in range(dist.get_world_size(group))]
    dist.all_gather(bucket, mine, group=group)
    return [torch.view_as_complex(b).cpu().numpy() for b in bucket]


class Piece:
    """Output steps first .. first + count - 1 of one evaluate() (an ``Instance``): the operators and
    the piece's product on construction, the states after ``finish(psi_in)``."""

    def __init__(self, instance, first, count, **batch_kwargs):
        import dataclasses
        import torch
        from . import _lib
        from .batch import Batch
        self.dim = instance.spin.dimension
        self.batch = Batch([dataclasses.replace(instance, intervals=(first, count))], **batch_kwargs)
        self.first, self.count = first, count
        self.batch.run(with_state=False)
        self.lib = self.batch.lib
        ws = self.lib.spinsim_state_workspace_size(self.dim, max(1, count))
        self.workspace = torch.empty(ws, dtype=torch.uint8, device=self.batch.device)
        self.product = torch.eye(self.dim, dtype=torch.complex128, device=self.batch.device)
        if count:
            stream = torch.cuda.current_stream(self.batch.device).cuda_stream
            _lib.check(self.lib.spinsim_piece_product(self.dim, self.batch.u.data_ptr(), count, self.product.data_ptr(),
                                                      self.workspace.data_ptr(), ws, stream))

    def finish(self, psi_in):
        """Scan the piece's states from ``psi_in`` (the state entering the piece) on the device."""
        import ctypes
        import torch
        from . import _lib
        if not self.count:
            return
        v = np.asarray(psi_in, np.complex128).reshape(-1)
        host = (ctypes.c_double * (2 * self.dim))(*np.column_stack([v.real, v.imag]).reshape(-1))
        stream = torch.cuda.current_stream(self.batch.device).cuda_stream
        _lib.check(self.lib.spinsim_piece_states(self.dim, self.batch.u.data_ptr(), self.count, ctypes.addressof(host),
                                                 self.batch.state.data_ptr(), self.batch.spin.data_ptr(),
                                                 self.workspace.data_ptr(), self.workspace.numel(), stream))

    def results(self):
        return self.batch.result(0)


def evaluate_split(instance, group=None, **batch_kwargs):
    """This rank's piece of one evaluate() split over the ranks of ``group`` (a collective: every
    rank calls it with the same instance).  Returns (first output step, ``Results`` of the piece)."""
    import torch.distributed as dist
    from . import _lib
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    _, n_out, _, _ = _lib.normalise_steps(instance.time_start, instance.time_end, instance.time_step_integration,
                                          instance.time_step_output)
    first, count = piece_ranges(n_out, world)[rank]
    piece = Piece(instance, first, count, **batch_kwargs)
    products = exchange_products(piece.product, group)
    piece.finish(incoming_states(products, instance.state_init)[rank])
    return first, piece.results()
