"""Project-written autotuner for the launch parameters of the step.

It times a few graph-replayed steps of the caller's loaded state for each
candidate of (neighbour-chunk width = lanes per particle in the neighbour
passes, block size of those passes, tree leaf size) and keeps the fastest.
Results do not depend on the lanes and block size; the leaf size changes which
tree nodes the walk accepts (accuracy within the same opening angle).
"""
from __future__ import annotations

import itertools
import time


def tune(ctx, lanes=(2, 4, 8), blocks=(128, 256), leaves=(6, 8, 12), steps=2, warmup=1):
    base = {k: getattr(ctx.config, k) for k in ("ngb_lanes", "block_size", "leaf_size")}
    results = []
    for nl, bs, lf in itertools.product(lanes, blocks, leaves):
        ctx.set_params(ngb_lanes=nl, block_size=bs, leaf_size=lf)
        ctx.step(warmup)
        ctx.sync()
        t0 = time.perf_counter()
        ctx.step(steps)
        ctx.sync()
        results.append(((time.perf_counter() - t0) / steps, dict(ngb_lanes=nl, block_size=bs,
                                                                  leaf_size=lf)))
    results.sort(key=lambda r: r[0])
    best = results[0][1] if results else base
    ctx.set_params(**best)
    return best, results
