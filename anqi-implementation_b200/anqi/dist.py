"""Multi-process plumbing: one process per GPU, index replicas, query shards.

The reference has no distributed path (one OpenMP process); queries are
independent, so N GPUs run N index replicas, each on its own batch, and the
only communication is the timing reduction (max over ranks) and, when a
caller wants one result set, a gather of CSR pieces.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced [begin, end) of n items for rank."""
    q, r = divmod(n, world)
    b = rank * q + min(rank, r)
    return b, b + q + (1 if rank < r else 0)


def max_over_ranks(values, device=None):
    """Element-wise max of a list of floats over all ranks (identity for one rank)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def gather_csr(off: np.ndarray, ids: np.ndarray):
    """Concatenates per-rank CSR pieces (in rank order) on every rank."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return off, ids
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, (np.asarray(off), np.asarray(ids)))
    offs, idss = [], []
    base = 0
    for o, i in parts:
        offs.append(o[:-1].astype(np.int64) + base)
        idss.append(i)
        base += int(o[-1])
    return np.concatenate(offs + [np.array([base])]).astype(np.uint32), np.concatenate(idss).astype(np.uint32)
