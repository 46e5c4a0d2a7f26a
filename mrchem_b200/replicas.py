"""Host logic of the multi-GPU runs: one process per GPU, every process applying whole trees.

The batched applies shard by tree (orbitals, pair densities, mu values), the unit the reference
distributes over MPI ranks (src/parallel.cpp:118-120 assigns orbitals round-robin; the apply loop of
src/scf_solver/HelmholtzVector.cpp:77 skips the orbitals a rank does not own).  There is no exchange
inside an apply, so the only collective is the reduction of the step time (the max over ranks).
"""
from __future__ import annotations

import os


def dist_env():
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_ranges(weights, world):
    """Contiguous ranges [begin, end) of a batch, one per rank, balanced by weight (e.g. the input
    trees' node counts, which the apply's work follows).  Every item lands in exactly one range, in
    order; a rank may get an empty range when the batch has fewer items than ranks."""
    n = len(weights)
    if world < 1:
        raise ValueError("world size must be positive")
    total = float(sum(weights))
    bounds = [0]
    acc = 0.0
    i = 0
    for r in range(1, world):
        target = total * r / world
        while i < n and acc + 0.5 * weights[i] <= target:
            acc += weights[i]
            i += 1
        bounds.append(max(i, bounds[-1]))
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def max_over_ranks(value, device=None):
    """The maximum of a per-rank float over the process group (the value itself without one).
    `device`: where the reduction tensor lives (a CUDA device for NCCL, None for gloo on CPU)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(base, rank):
    """Seed of a rank's own batch in the weak-scaling runs: every rank applies a different batch."""
    return base + 1000 * rank
