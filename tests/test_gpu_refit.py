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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_kept_rows_match_a_fresh_search(precision):
    """rebuild_every = 4 with the candidate rows kept between the h
    iterations and with every particle searched each step: the refit steps
    keep most rows, the rebuild step keeps none, the lists stay the
    oracle's, and h agrees with the searching run to the rounding of the
    first Newton evaluation (same terms, another summation order)."""
    n, dt = 10_000, 1e-3
    a = evrard_ctx(precision, 4, n=n, dt=dt)
    b = evrard_ctx(precision, 4, n=n, dt=dt, flags=L.FLAG_NO_ROW_REUSE)
    assert a.rows_kept() == 0  # the prologue sorted: every particle searched
    kept = []
    for k in range(4):
        a.step(1)
        b.step(1)
        a.sync()
        b.sync()
        kept.append(a.rows_kept())
        assert b.rows_kept() == 0
        st = a.status()
        assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
        check_step_state(a, dt, precision)
        ha, hb = a.get("h", True), b.get("h", True)
        assert np.max(np.abs(ha / hb - 1.0)) < 1e-5, k
    # the prologue's rows were searched before its first lists (their reach
    # towards the largest neighbour h is unknown): the first refit step may
    # search again; the later ones keep most rows
    assert max(kept[:3]) > n // 2 and kept[3] == 0, kept
    a.close()
    b.close()


def test_kept_rows_follow_moves_through_set_fields():
    """Positions set from the host between steps count as moves: a small
    shift of every particle keeps the rows, a large jump of a few particles
    makes the groups near them search again (and no other cloud's), and the
    lists stay exact either way, per cloud in an ensemble."""
    e = ic.ensemble(n_clouds=3, nmin=3000, nmax=6000, seed=7)
    n = len(e["m"])
    ctx = Context(Config(n_max=n, n_cloud_max=3, precision="mixed", theta=0.5, dt_fixed=1e-4,
                         rebuild_every=50))
    ctx.load(e["pos"], e["vel"], e["m"], e["h"], e["u"], cloud=e["cloud"])
    ctx.prologue()
    # the prologue's rows lack the reach of its first lists; after one step
    # that keeps few rows the next searches every particle
    ctx.step(2)
    ctx.sync()
    counts = np.bincount(e["cloud"], minlength=3)
    cl = np.repeat(np.arange(3), counts).astype(np.int32)

    def lists_exact():
        x, y, z, m, h = storage(ctx)
        off, lst = ctx.neighbour_lists()
        oo, ol = O.neighbours(x, y, z, h, cloud=cl)
        assert np.array_equal(off, oo) and np.array_equal(lst, ol)

    lists_exact()
    pos = ctx.get_pos(True)
    h = ctx.get("h", True)
    # a shift far below every h: rows kept almost everywhere
    ctx.set_fields({"x": pos[:, 0] + 1e-3 * float(h.min())}, storage_order=True)
    ctx.step(1)
    ctx.sync()
    assert ctx.rows_kept() > n // 2
    lists_exact()
    # ten particles of cloud 0 jump by 3 h: the groups near them cannot keep
    # their rows, the other clouds keep theirs
    pos = ctx.get_pos(True)
    h = ctx.get("h", True)
    x = pos[:, 0].copy()
    x[:10] += 3.0 * h[:10]
    ctx.set_fields({"x": x}, storage_order=True)
    ctx.step(1)
    ctx.sync()
    kept = ctx.rows_kept()
    assert kept < n, (kept, counts)
    assert kept > (n - counts[0]) // 2, (kept, counts)
    lists_exact()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
    ctx.close()
