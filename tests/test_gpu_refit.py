"""Steps that refit the tree instead of sorting and splitting it again
(sph_config.rebuild_every > 1).

Between two full rebuilds the storage order, the tree topology and the
groups stay; every node's box, moments, h_max and opening radius are
recomputed from the drifted particles.  The neighbour lists must therefore
stay exact (the oracle's, bit for bit), the gravity must stay within the
opening angle's error of the every-step rebuild, and the schedule must be a
pure function of the step count: graph replay equals eager execution, and a
context resumed from a restart file repeats the one that wrote it.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sph_2_b200 import Config, Context, ic
from sph_2_b200 import _lib as L
from test_gpu_step_parity import check_step_state, infall, storage

pytestmark = pytest.mark.gpu


def evrard_ctx(precision, every, n=10_000, flags=0, dt=1e-3):
    d = ic.evrard(n, seed=42)
    ctx = Context(Config(n_max=n, precision=precision, theta=0.5, dt_fixed=dt,
                         av_mode="gadget", balsara=True, flags=flags, rebuild_every=every))
    ctx.load(d["pos"], infall(d), d["m"], d["h"], d["u"])
    ctx.prologue()
    return ctx


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_refit_steps_keep_lists_and_sums_exact(precision):
    """rebuild_every = 4: after each of three refit steps and the rebuild
    that follows, the step's lists equal the oracle's and rho, div v and
    |curl v| are within the step-parity tolerances; the refit steps keep the
    storage order."""
    dt = 1e-3
    ctx = evrard_ctx(precision, 4, dt=dt)
    ids0 = ctx.ids()
    for k in range(4):
        ctx.step(1)
        ctx.sync()
        st = ctx.status()
        assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
        check_step_state(ctx, dt, precision)
        if k < 3:
            assert np.array_equal(ctx.ids(), ids0), "a refit step changed the storage order"
    ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_refit_gravity_close_to_every_step_rebuild(precision):
    """Six steps with rebuild_every = 3 against six with a rebuild every
    step: the same state to the opening angle's error (the trees differ, the
    particles they hold do not)."""
    a = evrard_ctx(precision, 1)
    b = evrard_ctx(precision, 3)
    a.step(6)
    b.step(6)
    a.sync()
    b.sync()
    ga, gb = a.get_acc("grav"), b.get_acc("grav")
    rms = np.sqrt(np.mean(np.sum((ga - gb) ** 2, 1) / np.sum(ga * ga, 1)))
    assert rms < 1e-3, rms
    for f in ("x", "y", "z"):
        assert np.max(np.abs(a.get(f) - b.get(f))) < 1e-7, f
    # h converges to 1e-3: a particle whose iteration stops one Newton step
    # earlier or later on the other trajectory moves its rho by about that
    drho = np.abs(a.get("rho") / b.get("rho") - 1)
    assert np.percentile(drho, 99) < 1e-5 and np.max(drho) < 1e-2
    a.close()
    b.close()


def test_refit_graph_replay_equals_eager_bitwise():
    a = evrard_ctx("mixed", 3, n=4000)
    b = evrard_ctx("mixed", 3, n=4000, flags=L.FLAG_NO_GRAPH)
    a.step(7)
    b.step(7)
    a.sync()
    b.sync()
    for f in ("x", "vx", "u", "h", "rho", "ax_grav"):
        assert np.array_equal(a.get(f), b.get(f)), f


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_refit_restart_resumes_bit_for_bit(tmp_path, precision):
    """A restart file written between two rebuilds: the writing context and
    a context that reads the file both rebuild on the next step and then
    continue alike, bit for bit."""
    a = evrard_ctx(precision, 3, n=6000)
    a.step(4)  # refit, refit, rebuild, refit
    a.sync()
    path = tmp_path / "restart.bin"
    a.write_restart(path)
    a.step(4)
    a.sync()
    b = Context(Config(n_max=6000, precision=precision, theta=0.5, dt_fixed=1e-3,
                       av_mode="gadget", balsara=True, rebuild_every=3))
    b.read_restart(path)
    b.step(4)
    b.sync()
    for f in ("x", "y", "z", "vx", "vy", "vz", "u", "h", "rho", "ax_grav", "ax_sph"):
        assert np.array_equal(a.get(f), b.get(f)), f
    assert np.array_equal(a.ids(), b.ids())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tree_export_after_refit_steps_is_bitexact(precision):
    """A step stores the FP64 build records of the group nodes and above
    only; sph_get_tree recomputes the others, so the exported tree after two
    refit steps holds the oracle's moments of the current particles on the
    current topology, bit for bit."""
    ctx = evrard_ctx(precision, 4, n=5000)
    ctx.step(2)
    ctx.sync()
    t = ctx.tree()
    x, y, z, m, h = storage(ctx)
    node, hmax = O.tree_moments(t["child"], t["first"], t["last"], x, y, z, m, h)
    assert np.array_equal(t["node"].view(np.uint64), node.view(np.uint64))
    assert np.array_equal(t["hmax"], hmax)
    ctx.close()


def test_refit_ensemble_lists_exact():
    """A 3-cloud ensemble with rebuild_every = 3: after two refit steps the
    lists of every cloud equal the oracle's (the clouds overlap in space and
    must stay apart) and the per-cloud storage ranges are unchanged."""
    e = ic.ensemble(n_clouds=3, nmin=2000, nmax=6000, seed=5)
    n = len(e["m"])
    ctx = Context(Config(n_max=n, n_cloud_max=3, precision="mixed", theta=0.5, dt_fixed=1e-3,
                         rebuild_every=3))
    vel = e["vel"] + 0.05 * np.random.default_rng(5).normal(size=(n, 3))
    ctx.load(e["pos"], vel, e["m"], e["h"], e["u"], cloud=e["cloud"])
    ctx.prologue()
    ids0 = ctx.ids()
    ctx.step(2)
    ctx.sync()
    assert np.array_equal(ctx.ids(), ids0)
    x, y, z, m, h = storage(ctx)
    cl = np.repeat(np.arange(3), np.bincount(e["cloud"], minlength=3)).astype(np.int32)
    off, lst = ctx.neighbour_lists()
    oo, ol = O.neighbours(x, y, z, h, cloud=cl)
    assert np.array_equal(off, oo) and np.array_equal(lst, ol)
    ctx.close()
