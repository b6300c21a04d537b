"""Shot-parallel execution across GPUs: one process per GPU, shots dealt to
ranks, one sum of the images (or gradients) and of the FP64 misfit at the end.

The reference is single-GPU (no NCCL or MPI anywhere); its shots are
independent (src/migration_main.cpp:13-19, src/inversion/inversion.cu:123-138),
so the only exchange is the final sum.  Collectives go through
torch.distributed (NCCL between GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(nshots: int, world: int, rank: int, costs=None) -> list[int]:
    """Shots of `rank`.  Without costs: round robin.  With per-shot costs
    (e.g. receivers or aperture cells): longest-processing-time-first, so the
    ranks finish together; ties go to the lower rank, and every rank sees the
    same assignment."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    if costs is None:
        return list(range(rank, nshots, world))
    costs = np.asarray(costs, float)
    if costs.shape != (nshots,):
        raise ValueError("one cost per shot")
    order = sorted(range(nshots), key=lambda s: (-costs[s], s))
    heap = [(0.0, r) for r in range(world)]
    owner = np.empty(nshots, int)
    for s in order:
        load, r = heapq.heappop(heap)
        owner[s] = r
        heapq.heappush(heap, (load + costs[s], r))
    return [s for s in range(nshots) if owner[s] == rank]


def sum_across_ranks(*tensors):
    """In-place sum of device (or CPU, under gloo) tensors over all ranks."""
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return tensors
    for t in tensors:
        dist.all_reduce(t)
    return tensors


def misfit_across_ranks(local_sum_sq: float) -> float:
    """FP64 sum of the per-rank misfits."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(local_sum_sq)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([local_sum_sq], dtype=torch.float64, device=dev)
    dist.all_reduce(t)
    return float(t.item())


def reduce_context_accumulators(ctx, img_buf, ill_buf):
    """Sum a library context's padded image and illumination over all ranks:
    copy them into caller device tensors, all-reduce, write them back."""
    ctx.get_accumulators_dev(img_buf.data_ptr(), ill_buf.data_ptr())
    sum_across_ranks(img_buf, ill_buf)
    ctx.set_accumulators_dev(img_buf.data_ptr(), ill_buf.data_ptr())
