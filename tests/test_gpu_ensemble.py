"""The batched ensemble: independent clouds advanced by the same launches.

Clouds that overlap in space never interact: each cloud's SPH sums equal a
run of that cloud alone, its gravity equals its own direct sum within the tree
tolerance, and every cloud keeps its own time step.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sph_2_b200 import Config, Context, ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / (np.max(np.abs(b)) + 1e-300))


def test_clouds_do_not_interact():
    e = ic.ensemble(n_clouds=3, nmin=2000, nmax=6000, seed=21)   # all centred at the origin
    n = len(e["m"])
    rng = np.random.default_rng(0)
    vel = rng.normal(scale=0.1, size=(n, 3))
    ens = Context(Config(n_max=n, n_cloud_max=4, precision="fp64", theta=0.4, flags=16))
    ens.load(e["pos"], vel, e["m"], e["h"], e["u"], cloud=e["cloud"])
    ens.prologue()
    starts = np.concatenate([[0], np.cumsum(e["counts"])])
    for k in range(3):
        a, b = starts[k], starts[k + 1]
        one = Context(Config(n_max=b - a, precision="fp64", theta=0.4, flags=16))
        one.load(e["pos"][a:b], vel[a:b], e["m"][a:b], e["h"][a:b], e["u"][a:b])
        one.prologue()
        for f in ("h", "rho", "P", "divV", "dudt"):
            assert rel(ens.get(f)[a:b], one.get(f)) < 1e-11, (k, f)
        assert rel(ens.get_acc("sph")[a:b], one.get_acc("sph")) < 1e-11
        # gravity of cloud k only: its own direct sum
        ids = ens.ids()
        inv = np.empty(n, np.int64)
        inv[ids] = np.arange(n)
        sel = inv[a:b]
        ad, _ = ens.gravity_direct(sel.astype(np.int32))
        ag = ens.get_acc("grav", storage_order=True)[sel]
        err = np.sqrt(np.mean(np.sum((ag - ad) ** 2, 1) / np.sum(ad ** 2, 1)))
        assert err < 3e-4, (k, err)
        one.close()
    dts = ens.dt
    assert len(dts) == 3 and np.all(dts > 0) and len(set(np.round(dts, 12))) == 3
    ens.close()


def test_ensemble_steps_and_keys():
    e = ic.ensemble(n_clouds=5, nmin=1500, nmax=4000, seed=5)
    n = len(e["m"])
    ctx = Context(Config(n_max=n, n_cloud_max=8, precision="mixed"))
    ctx.load(e["pos"], e["vel"], e["m"], e["h"], e["u"], cloud=e["cloud"])
    ctx.prologue()
    ctx.step(3)
    ctx.sync()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0
    # every cloud still occupies its own contiguous, key-sorted range
    ctx.sort()
    keys, perm = ctx.sort_info()
    pos = ctx.get_pos(storage_order=True)
    cl = np.repeat(np.arange(5), e["counts"])
    ok = O.morton_keys(*(pos[:, k].copy() for k in range(3)), cloud=cl)
    assert np.array_equal(keys, ok)
    assert np.array_equal(perm, O.sort_perm(ok))


def test_mixed_walk_with_supergroups_per_cloud():
    """The mixed walk with group and super-group expansions and the
    small-cell opening angle on overlapping clouds: super-groups never mix
    clouds, each cloud's gravity matches its own FP64 direct sum, and no
    super-group falls back for lack of list room."""
    e = ic.ensemble(n_clouds=4, nmin=20000, nmax=40000, seed=8)
    n = len(e["m"])
    ctx = Context(Config(n_max=n, n_cloud_max=4, precision="mixed", theta=0.35,
                         theta_local=0.28, theta_small=0.45, small_cell=4))
    ctx.load(e["pos"], e["vel"], e["m"], e["h"], e["u"], cloud=e["cloud"])
    ctx.sort()
    ctx.build_tree()
    ctx.gravity()
    cnt = ctx.counters()
    assert cnt["sg_far_cells"] > 0 and cnt["sg_fallback"] == 0
    ids = ctx.ids()
    inv = np.empty(n, np.int64)
    inv[ids] = np.arange(n)
    starts = np.concatenate([[0], np.cumsum(e["counts"])])
    rng = np.random.default_rng(1)
    for k in range(4):
        a, b = starts[k], starts[k + 1]
        sel = inv[rng.choice(np.arange(a, b), 1000, replace=False)]
        ad, _ = ctx.gravity_direct(sel.astype(np.int32))
        ag = ctx.get_acc("grav", storage_order=True)[sel]
        err = np.sqrt(np.mean(np.sum((ag - ad) ** 2, 1) / np.sum(ad ** 2, 1)))
        assert err < 3e-4, (k, err)
    ctx.close()


def test_autotuner_picks_valid_parameters_and_keeps_accuracy(tmp_path):
    """The autotuner searches leaf size 8..64, lanes per particle and block
    size on an uneven 4-cloud ensemble, stores its choice per workload, applies
    a cached choice without timing, and the gravity at the chosen settings
    stays within the opening angle's error bound against the FP64 direct sum."""
    from sph_2_b200.autotune import BLOCKS, LANES, LEAVES, tune
    e = ic.ensemble(n_clouds=4, nmin=20_000, nmax=60_000, seed=3)
    n = len(e["m"])
    ctx = Context(Config(n_max=n, n_cloud_max=4, precision="mixed", theta=0.5))
    ctx.load(e["pos"], e["vel"], e["m"], e["h"], e["u"], cloud=e["cloud"])
    ctx.prologue()
    cache = str(tmp_path / "tune.json")
    best, res = tune(ctx, cache=cache, steps=1, warmup=1)
    assert best["leaf_size"] in LEAVES and best["ngb_lanes"] in LANES
    assert best["block_size"] in BLOCKS
    assert len(res) >= len(LEAVES) and all(ms > 0 for ms, _ in res)
    assert res[0][1] == best
    best2, res2 = tune(ctx, cache=cache)
    assert best2 == best and res2[0][0] is None
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
    ctx.load(e["pos"], e["vel"], e["m"], e["h"], e["u"], cloud=e["cloud"])
    ctx.prologue()
    tg = np.random.default_rng(0).choice(n, 2000, replace=False).astype(np.int32)
    ad, _ = ctx.gravity_direct(tg)
    a = ctx.get_acc("grav", True)[tg]
    err = np.sqrt(np.mean(np.sum((a - ad) ** 2, 1) / np.sum(ad * ad, 1)))
    assert err < 3.7e-4
