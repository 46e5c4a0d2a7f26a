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


def apply_batched_sharded(prec, outs, ops, inps, flags=0, apply=None, group=None):
    """One batch split over the ranks of the process group (strong scaling): rank r applies the
    contiguous range shard_ranges(input node counts)[r] of the batch -- the orbitals it owns, as in the
    reference's per-rank loop (src/scf_solver/HelmholtzVector.cpp:77, ownership from
    src/parallel.cpp:118-120) -- and the per-tree results are then gathered for every rank.

    `outs`, `ops`, `inps`: the whole batch (every rank holds the input trees; only its own range is
    computed).  `apply(prec, outs, ops, inps, flags)` applies a list of trees; the default is
    mrchem_b200.mrcpp.apply_batched.  Returns (ranges, results) with results[i] = (square norm,
    node count) of output tree i, identical on every rank.  Without a process group this is one
    apply of the whole batch.  The only collective is the all-gather of those results: the apply
    itself exchanges nothing."""
    if apply is None:
        from mrchem_b200 import mrcpp as G

        apply = G.apply_batched
    import torch.distributed as dist

    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if dist_on else 1
    rank = dist.get_rank(group) if dist_on else 0
    n = len(inps)
    if not (len(outs) == len(ops) == n):
        raise ValueError("outs, ops and inps must have the same length")
    ranges = shard_ranges([t.nnodes() for t in inps], world)
    b, e = ranges[rank]
    if e > b:
        apply(prec, outs[b:e], ops[b:e], inps[b:e], flags)
    local = [(float(outs[i].square_norm()), int(outs[i].nnodes())) for i in range(b, e)]
    if world == 1:
        return ranges, local
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    results = [x for part in parts for x in part]
    if len(results) != n:
        raise RuntimeError("sharded batch: gathered results do not cover the batch")
    return ranges, results


def rank_seed(base, rank):
    """Seed of a rank's own batch in the weak-scaling runs: every rank applies a different batch."""
    return base + 1000 * rank
