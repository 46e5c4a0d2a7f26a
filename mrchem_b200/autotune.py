"""Autotuner of the contraction's work split.

The contraction kernels run one CTA per chunk of (input node, term) pairs of one output node, cut so
that a chunk holds at most `chunk_triples` (output, input, term) triples.  Small chunks balance the
load across the 148 SMs, but an output node cut into several chunks writes partial blocks that a
reduction kernel adds afterwards.  Large chunks keep the node in one CTA.  The best value depends on
the engine (FP64, FP32, split-TF32, BF16x3), the order and the tree shapes, so it is measured on the
caller's own workload: `tune_chunk_triples` times a representative call under each candidate and
leaves the fastest set on the context.  Results agree to FP64 rounding for every value (only the
grouping of the partial sums changes).
"""
from __future__ import annotations

import statistics
import time

DEFAULT_CANDIDATES = (16, 24, 32, 48, 64, 96, 128, 192, 256)


def _wall_ms(run, sync):
    sync()
    t0 = time.perf_counter()
    run()
    sync()
    return (time.perf_counter() - t0) * 1e3


def tune_chunk_triples(ctx, run, flags, candidates=DEFAULT_CANDIDATES, reps=2, warmup=1, timer=None):
    """Time `run()` (a blocking call that applies a representative batch under `flags` on `ctx`) with
    each candidate chunk size and set the fastest on `ctx`.

    Each candidate gets `warmup` untimed calls, then `reps` timed ones; the score is their median.
    Ties go to the earlier candidate.  `timer(run) -> ms` replaces the default wall-clock timer (the
    library's calls are blocking, so host time around them is the device time plus launch gaps).
    Returns {"best": value, "ms": {value: median ms}, "flags": flags}.
    """
    if not candidates:
        raise ValueError("no candidates")
    if reps < 1:
        raise ValueError("reps must be >= 1")
    if timer is None:
        def timer(fn):
            return _wall_ms(fn, ctx.synchronize)
    scores = {}
    for c in candidates:
        ctx.set_chunk_triples(flags, int(c))
        for _ in range(warmup):
            run()
        scores[int(c)] = statistics.median(timer(run) for _ in range(reps))
    best = min(scores, key=lambda c: (scores[c], list(scores).index(c)))
    ctx.set_chunk_triples(flags, best)
    return {"best": best, "ms": scores, "flags": int(flags)}
