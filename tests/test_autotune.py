"""The chunk-size autotuner's selection logic, on CPU with a fake context and timer."""
import pytest

from mrchem_b200.autotune import tune_chunk_triples


class FakeCtx:
    def __init__(self):
        self.value = {0: 48, 1: 48, 2: 48}
        self.history = []
        self.syncs = 0

    def set_chunk_triples(self, flags, triples):
        self.value[flags] = triples
        self.history.append((flags, triples))

    def synchronize(self):
        self.syncs += 1


def test_picks_the_fastest_and_leaves_it_set():
    ctx = FakeCtx()
    cost = {16: 9.0, 32: 7.5, 48: 6.0, 96: 6.5}
    calls = []

    def run():
        calls.append(ctx.value[1])

    res = tune_chunk_triples(ctx, run, 1, candidates=(16, 32, 48, 96), reps=3, warmup=1,
                             timer=lambda fn: (fn(), cost[ctx.value[1]])[1])
    assert res["best"] == 48 and ctx.value[1] == 48
    assert res["ms"] == cost
    assert ctx.value[0] == 48 and ctx.value[2] == 48  # other engines untouched
    assert len(calls) == 4 * (1 + 3)  # warm-up and timed calls per candidate


def test_median_and_ties():
    ctx = FakeCtx()
    seq = {24: iter([5.0, 100.0, 5.0]), 64: iter([5.0, 5.0, 5.0])}
    res = tune_chunk_triples(ctx, lambda: None, 2, candidates=(24, 64), reps=3, warmup=0,
                             timer=lambda fn: next(seq[ctx.value[2]]))
    assert res["ms"] == {24: 5.0, 64: 5.0}
    assert res["best"] == 24  # tie: the earlier candidate


def test_default_timer_synchronises():
    ctx = FakeCtx()
    res = tune_chunk_triples(ctx, lambda: None, 0, candidates=(32,), reps=2, warmup=0)
    assert res["best"] == 32 and ctx.syncs == 4


def test_rejects_empty_input():
    with pytest.raises(ValueError):
        tune_chunk_triples(FakeCtx(), lambda: None, 1, candidates=())
    with pytest.raises(ValueError):
        tune_chunk_triples(FakeCtx(), lambda: None, 1, reps=0)
