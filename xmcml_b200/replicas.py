"""Multi-GPU replicas: one process per GPU, each walking a disjoint range of photon ids.

Photons are independent and every random number depends only on (seed, photon id), so a job of
W ranks is W replicas of the single-GPU run on disjoint id ranges: no data exchange during the walk.
The only collectives are the max over ranks of the timings and, when a caller wants one combined
result, a sum of the 64-bit integer tallies (exact in any order, like the reference's MPI_Reduce of
tallies in base/xmcml/xmcmlLauncher/launcher_mpi.cpp:199-287).
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np


def photon_range(rank: int, world: int, n_per_rank: int, step: int = 0) -> Tuple[int, int]:
    """First photon id and count of `rank`'s share of step `step` (weak scaling: n_per_rank each)."""
    if not (0 <= rank < world):
        raise ValueError("rank out of range")
    first = (step * world + rank) * n_per_rank
    return first, n_per_rank


def split_total(rank: int, world: int, n_total: int) -> Tuple[int, int]:
    """First photon id and count of `rank`'s share of n_total photons (strong scaling), the split the
    reference's MPI launcher makes (launcher_mpi.cpp:398-403: the first `remainder` ranks take one more)."""
    base = n_total // world
    rem = n_total - base * world
    n = base + (1 if rank < rem else 0)
    first = rank * base + min(rank, rem)
    return first, n


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank scalar (a timing) over all ranks; identity without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_tallies(tallies: Dict[str, np.ndarray], dist=None, device=None) -> Dict[str, np.ndarray]:
    """Sum of every rank's integer tallies (uint64 fixed point or counts), returned on every rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return {k: v.copy() for k, v in tallies.items()}
    import torch
    out = {}
    for k in sorted(tallies):
        v = np.ascontiguousarray(tallies[k]).astype(np.uint64)
        t = torch.from_numpy(v.view(np.int64).copy()).to(device) if device is not None else torch.from_numpy(v.view(np.int64).copy())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)  # two's-complement sums equal uint64 sums mod 2^64
        out[k] = t.cpu().numpy().view(np.uint64).reshape(v.shape)
    return out
