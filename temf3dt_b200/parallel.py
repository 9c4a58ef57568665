"""Multi-GPU plumbing for the batched paths: one process per GPU.

The FETD hot path shards across RHS columns (transmitter positions) and
across independent models; nothing is exchanged per time step.  Each rank
factors its own copy of the step matrix and solves its block of columns; the
only collective is a final gather of the small receiver traces.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np


def shard_range(n_items: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous block [lo, hi) of n_items for `rank` of `world` (sizes differ by <= 1)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_traces(local: np.ndarray, world: int, group=None) -> List[np.ndarray]:
    """All-gather per-rank receiver traces (rows x rec_local x 9) of possibly
    different receiver counts; returns the list in rank order."""
    if world == 1:
        return [local]
    import torch.distributed as dist
    out: List[object] = [None] * world
    dist.all_gather_object(out, local, group=group)
    return [np.asarray(x) for x in out]


def assemble_traces(parts: List[np.ndarray]) -> np.ndarray:
    """Concatenate rank-ordered traces along the receiver axis."""
    return np.concatenate(parts, axis=1)


def reduce_gradients(local: np.ndarray, world: int, group=None) -> np.ndarray:
    """Sum per-rank adjoint gradients (each rank's sources) over all ranks:
    one all-reduce of the inversion-grid vector.  Works on the process
    group's backend (gloo on CPU tensors, NCCL on the rank's GPU)."""
    if world == 1:
        return np.asarray(local, dtype=np.float64)
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.as_tensor(np.asarray(local, dtype=np.float64), device=dev).clone()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()
