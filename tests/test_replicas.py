"""Host logic of the multi-GPU runs, on CPU: the balanced contiguous split of a batch over ranks, the
per-rank batches of the weak-scaling runs, and the max-over-ranks step time, the last over a real
2-process `gloo` group (the same collective the GPU runs make over NCCL)."""
import json
import os
import socket

import numpy as np
import pytest

from mrchem_b200.replicas import max_over_ranks, rank_seed, shard_ranges


def test_shard_ranges_cover_and_balance():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 4, 8):
        for n in (0, 1, 5, 32, 136):
            w = rng.integers(500, 5000, n).tolist()
            r = shard_ranges(w, world)
            assert len(r) == world
            assert r[0][0] == 0 and r[-1][1] == n
            for (a, b), (c, d) in zip(r, r[1:]):
                assert b == c and a <= b
            if n >= 4 * world:
                loads = [sum(w[a:b]) for a, b in r]
                assert max(loads) <= sum(w) / world + max(w)
    assert shard_ranges([1.0] * 8, 4) == [(0, 2), (2, 4), (4, 6), (6, 8)]
    with pytest.raises(ValueError):
        shard_ranges([1.0], 0)


def test_rank_batches_differ():
    from mrchem_b200 import workloads as W

    a = W.orbitals(4, seed=rank_seed(2, 0))
    b = W.orbitals(4, seed=rank_seed(2, 1))
    assert not np.array_equal(a[0][1], b[0][1])
    assert rank_seed(2, 0) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        step_ms = [12.5, 40.25][rank]
        got = max_over_ranks(step_ms)
        ranges = shard_ranges([3, 1, 4, 1, 5, 9, 2, 6], world)
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": got, "range": ranges[rank]}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_processes(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert res[0]["max"] == res[1]["max"] == 40.25
    assert res[0]["range"][1] == res[1]["range"][0] and res[0]["range"][0] == 0 and res[1]["range"][1] == 8
    assert max_over_ranks(7.0) == 7.0  # no process group: the value itself


# ---- one batch sharded over ranks through the product's host API --------------------------------
# The per-rank apply is the CPU oracle here (gloo ranks have no GPU): the test checks the sharding --
# which trees each rank computes and what every rank ends up with -- against one process applying the
# whole batch.  On GPUs the default apply is mrchem_b200.mrcpp.apply_batched.

def _oracle_batch(prec, order=5, n=5):
    from mrchem_b200 import workloads as W
    from oracle import oracle as O

    m = O.MultiResolutionAnalysis(W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"], order, 10)
    orbs = W.orbitals(n, seed=3)
    mus = W.helmholtz_mus(n, seed=3)
    inps, ops, outs = [], [], []
    for f, mu in zip(orbs, mus):
        t = O.FunctionTree(m)
        O.project(prec, t, f)
        inps.append(t)
        ops.append(O.HelmholtzOperator(m, mu, prec))
        outs.append(O.FunctionTree(m))
    return O, inps, ops, outs


def _oracle_apply(O):
    def run(prec, outs, ops, inps, flags):
        for o, op, t in zip(outs, ops, inps):
            O.apply(prec, o, op, t)
    return run


def _shard_rank_main(rank, world, port, outdir):
    import datetime

    import torch.distributed as dist

    from mrchem_b200.replicas import apply_batched_sharded

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        O, inps, ops, outs = _oracle_batch(1e-3)
        ranges, res = apply_batched_sharded(1e-3, outs, ops, inps, apply=_oracle_apply(O))
        b, e = ranges[rank]
        computed = [i for i in range(len(outs)) if outs[i].nnodes() > 0]
        with open(os.path.join(outdir, f"shard{rank}.json"), "w") as f:
            json.dump({"ranges": ranges, "results": res, "computed": computed, "own": [b, e]}, f)
    finally:
        dist.destroy_process_group()


def test_sharded_batch_gloo_equals_single_process(tmp_path):
    import torch.multiprocessing as mp

    from mrchem_b200.replicas import apply_batched_sharded

    port = _free_port()
    mp.start_processes(_shard_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"shard{r}.json")) for r in range(2)]
    # every rank computed exactly its own range, and the two ranges cover the batch once
    for r in range(2):
        b, e = res[r]["own"]
        assert res[r]["computed"] == list(range(b, e))
    assert res[0]["own"][0] == 0 and res[0]["own"][1] == res[1]["own"][0] and res[1]["own"][1] == 5
    # every rank holds the same gathered results, equal to one process applying the whole batch
    assert res[0]["results"] == res[1]["results"]
    O, inps, ops, outs = _oracle_batch(1e-3)
    ranges, single = apply_batched_sharded(1e-3, outs, ops, inps, apply=_oracle_apply(O))
    assert ranges == [(0, 5)]
    assert [tuple(x) for x in res[0]["results"]] == [tuple(x) for x in single]
