"""Multi-GPU sharding of the direct J/K and gradient builds.

The reference's unit of work is the canonical bra shell pair (src/direct.rs:
19-21, src/direct_grad.rs:140-142): contributions of different bra pairs
are independent and simply add.  One process per GPU therefore takes a
disjoint subset of bra pairs and builds private partial J/K (or gradient)
on its device; the only exchange is the final sum, one all-reduce over
NCCL (NVLink / NVSwitch) — or gloo on CPU.
"""
from __future__ import annotations

import numpy as np


def bra_shard(nbra: int, rank: int, world: int) -> np.ndarray:
    """Canonical bra-pair indices owned by `rank`: every world-th pair.
    Interleaving spreads near and far pairs (cheap and costly bras) evenly."""
    if not (0 <= rank < world):
        raise ValueError("rank %d outside world %d" % (rank, world))
    return np.arange(rank, nbra, world, dtype=np.uint32)


def all_reduce_sum(arrays, device=None):
    """Sum numpy arrays (or torch tensors) over the default process group in
    place and return them; a no-op when torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return arrays
    out = []
    for a in arrays:
        if isinstance(a, np.ndarray):
            t = torch.from_numpy(np.ascontiguousarray(a))
            if device is not None:
                t = t.to(device)
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            a[...] = t.cpu().numpy().reshape(a.shape)
            out.append(a)
        else:
            dist.all_reduce(a, op=dist.ReduceOp.SUM)
            out.append(a)
    return out
