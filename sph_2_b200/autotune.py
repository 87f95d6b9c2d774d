"""Project-written autotuner for the launch parameters of the step.

Three parameters change the speed of a step but not what it computes beyond
rounding and the bucket sizes of the tree:
  * ngb_lanes -- lanes per particle in the neighbour passes (the width of the
    chunk of a neighbour row that one pass over the row reads at once),
  * block_size -- threads per block of those passes,
  * leaf_size -- particles per tree bucket (8..64): the walk opens buckets
    into particle-particle interactions, so larger buckets trade cell
    interactions for exact pair terms (never less accurate at equal theta).
The tuner times graph-replayed steps of the caller's loaded state on the
device (CUDA events, sph_time_steps) for each candidate and walks the space
by coordinate descent: leaf size first (the walk is the largest phase), then
lanes, then block size.  Tuning advances the state by (warmup + steps) steps
per candidate.  The choice is stored in a JSON cache keyed by the workload's
signature (particles, clouds, precision, opening angles, GPU name), so the
next run of the same workload starts from it without searching.
"""
from __future__ import annotations

import json
import os

LANES = (2, 4, 8)
BLOCKS = (64, 128, 256)
LEAVES = (8, 12, 16, 24, 32, 48, 64)
PARAMS = ("leaf_size", "ngb_lanes", "block_size")


def default_cache() -> str:
    return os.environ.get("SPH_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "sph_2_b200", "tune.json"))


def signature(ctx) -> str:
    """Workload key of the cache: size, clouds, precision, walk settings and
    the device's name."""
    try:
        import torch
        dev = torch.cuda.get_device_name(0)
    except Exception:  # noqa: BLE001 - the key only needs to be stable
        dev = "cuda"
    c = ctx.config
    return (f"n{ctx.n}-c{ctx.n_clouds}-{c.precision}-t{c.theta:g}-tl{c.theta_local:g}"
            f"-ts{c.theta_small:g}-sc{c.small_cell}-{dev}")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, key, best):
    data = _load(path)
    data[key] = best
    try:
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        with open(path, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    except OSError:
        pass  # a read-only cache location only costs the search next time


def tune(ctx, lanes=LANES, blocks=BLOCKS, leaves=LEAVES, steps=2, warmup=1, cache=None,
         use_cache=True):
    """Pick (leaf_size, ngb_lanes, block_size) for the loaded workload and
    apply it.  Returns (best, [(ms_per_step, params), ...]); an entry of the
    cache is applied without timing (results then holds it alone with None)."""
    path = cache or default_cache()
    key = signature(ctx)
    if use_cache:
        hit = _load(path).get(key)
        if hit and all(k in hit for k in PARAMS):
            ctx.set_params(**{k: hit[k] for k in PARAMS})
            return dict(hit), [(None, dict(hit))]
    best = {k: getattr(ctx.config, k) for k in PARAMS}
    timed = {}

    def cost(p):
        k = tuple(p[q] for q in PARAMS)
        if k not in timed:
            ctx.set_params(**p)
            ctx.step(warmup)
            timed[k] = ctx.time_steps(steps) / steps
        return timed[k]

    for name, values in (("leaf_size", leaves), ("ngb_lanes", lanes), ("block_size", blocks)):
        cands = []
        for v in values:
            p = dict(best)
            p[name] = v
            cands.append((cost(p), p))
        best = min(cands, key=lambda r: r[0])[1]
    ctx.set_params(**best)
    results = sorted(((ms, dict(zip(PARAMS, k))) for k, ms in timed.items()), key=lambda r: r[0])
    _store(path, key, best)
    return best, results
