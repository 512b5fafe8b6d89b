"""Multi-GPU shot distribution: one process per GPU, shots partitioned across
ranks, one sum all-reduce of the objective and gradient.

The reference spreads shot batches over Dask workers
(``fwix/workers.py:14-83`` ``_obj_grad_worker``: per partition, micro-batches of
``shots_per_gpu`` shots, objective and gradient accumulated per worker) and sums
the per-worker gradients with a streaming Zarr reduction
(``fwix/workers.py:154-177`` ``_reduce_vector``).  Shots are independent through
every depth, so here each rank runs its own shots with no communication and
the only exchange is one ``torch.distributed.all_reduce`` (NCCL over NVLink on
GPUs, gloo on CPU) of the model-sized gradient and the scalar objective.

Partitioning is longest-processing-time-first on the per-shot cost
nx * ny * nw * nz (the cell-steps of one sweep), so ranks with shots of
uneven aperture or frequency band end within one shot's cost of each other.
"""
from __future__ import annotations

import heapq

import torch


def shot_cost(nx, ny, nw, nz):
    """Cell-steps of one sweep of one shot."""
    return int(nx) * int(ny) * int(nw) * int(nz)


def partition(costs, world_size):
    """Shot indices per rank (each list in ascending order), balancing the summed
    cost greedily from the most expensive shot down; ties go to the lower rank,
    so every rank computes the same partition."""
    if world_size < 1:
        raise ValueError("world_size must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world_size)]
    parts = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def _world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def allreduce_sum_(t, group=None):
    """In-place sum over ranks (no-op without an initialised process group)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def objective_and_gradient(costs, work, like, group=None):
    """Runs ``work(i) -> (J_i, g_i)`` for this rank's shots and returns the sums
    over all shots of every rank: (J, g).  ``like`` is a tensor with the
    gradient's shape, dtype and device (the accumulator is created from it)."""
    world, rank = _world()
    mine = partition(costs, world)[rank]
    g = torch.zeros_like(like)
    J = torch.zeros(1, dtype=torch.float64, device=like.device)
    for i in mine:
        Ji, gi = work(i)
        J += float(Ji)
        g += gi
    allreduce_sum_(g, group)
    allreduce_sum_(J, group)
    return float(J.item()), g
