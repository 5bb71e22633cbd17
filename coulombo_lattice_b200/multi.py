"""Multi-GPU decomposition of the integral path (one process per GPU, torch.distributed).

Three ways to spread work over ranks:

* One request over several GPUs, by prepared densities (both forms): the plan's left
  densities are dealt round-robin to the ranks (cl_compute_shard); each rank transforms its
  own left densities, forms every right density and returns the integrals of its steps, zeros
  elsewhere.  One all-reduce (sum, FP64) of the integral vector combines them -- the
  counterpart of the reference's MPI_Reduce of every calculate() (CoulombCalculator.cpp:170).

* One request over several GPUs: the integrals are sums over the 8 rounds kappa
  (CoulombCalculator.cpp:105-163 accumulates V_ += Ftemp round by round), so rank r takes the
  rounds kappa = r, r + world, ...  (cl_compute_rounds), and a single all-reduce (sum, FP64)
  of the integral vector -- 16 bytes per integral -- gives every rank the full result.  No
  grid data crosses NVLink.
* A batch of independent structures: structures are dealt whole to ranks by longest-
  processing-time order (cost ~ grid points x prepared densities); no collective at all.
"""
from __future__ import annotations

import numpy as np


def round_mask(rank: int, world: int) -> int:
    """Bit k set when round kappa = k belongs to `rank` (round-robin over ranks)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    mask = 0
    for k in range(8):
        if k % world == rank:
            mask |= 1 << k
    return mask


def allreduce_complex(values, group=None, device="cpu"):
    """Sum a complex128 vector over the ranks of `group` (one all-reduce of 2n float64)."""
    import torch
    import torch.distributed as dist
    v = np.ascontiguousarray(values, dtype=np.complex128)
    t = torch.from_numpy(v.view(np.float64).copy()).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().view(np.complex128).copy()


def compute_sharded(compute_rounds, specs, group=None, device="cpu"):
    """Full integrals of `specs` from this rank's share of the rounds.

    compute_rounds(specs, mask) -> complex vector of partial integrals (on a GPU rank this is
    CoulombCalculator.compute_rounds); every rank must call this with the same specs."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    mask = round_mask(rank, world) if rank < 8 else 0
    if mask:
        part = np.asarray(compute_rounds(specs, mask), dtype=np.complex128)
    else:
        part = np.zeros(len(specs), dtype=np.complex128)
    return allreduce_complex(part, group=group, device=device)


def compute_density_sharded(compute_shard, specs, group=None, device="cpu"):
    """Full integrals of `specs` from this rank's shard of the left densities.

    compute_shard(specs, shard, n_shards) -> complex vector with this shard's integrals and
    zeros elsewhere (on a GPU rank: CoulombCalculator.compute_shard); every rank calls this with
    the same specs."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    part = np.asarray(compute_shard(specs, rank, world), dtype=np.complex128)
    return allreduce_complex(part, group=group, device=device)


def partition_structures(costs, world):
    """Longest-processing-time assignment of independent structures to ranks.
    Returns a list (per rank) of structure indices."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return out
