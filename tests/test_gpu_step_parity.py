"""Parity of the kernels the timed step runs, through the C ABI.

The step builds its lists, density, div/curl and Balsara factor in one pass
over the h iteration's candidate rows (the fused list + density kernel) and
sends the particles whose list that pass cannot prove complete to the tree
search.  These tests export what a step left behind and compare it with the
oracle: lists bit-exact, sums within the stated tolerance.  They also pin
the reference's own count iteration for h (h_smooth_fast_mpi), two steps of
the reference's loop (sph_mpi4_v4.py:278-416) against the golden outputs of
the reference itself, and the Courant step.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from sph_2_b200 import Config, Context, ic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    """max |a-b| / max |b| (scale-relative)."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


def storage(ctx):
    pos = ctx.get_pos(True)
    return (pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), ctx.get("m", True),
            ctx.get("h", True))


def infall(d, seed=5):
    rng = np.random.default_rng(seed)
    return -0.3 * d["pos"] + 0.05 * rng.normal(size=d["pos"].shape)


def pass_velocity(ctx, dt):
    """Velocities of the step's neighbour passes: the closing half kick
    v += (a_sph + a_grav) dt / 2 undone (storage order)."""
    v = ctx.get_vel(True)
    a = ctx.get_acc("sph", True) + ctx.get_acc("grav", True)
    return v - 0.5 * dt * a


# ------------------------------------------------- the step's own passes ---
# tolerances of the sums: FP64 sums in a different order (1e-11 of the
# scale); mixed: FP32 terms with Kahan compensation
SUM_TOL = {"fp64": 1e-11, "mixed": 2e-5}


def check_step_state(ctx, dt, precision, dc_tol_fac=10.0):
    """Lists, rho, div v and |curl v| left by the last step against the
    oracle on the stored positions, h and pass velocities."""
    x, y, z, m, h = storage(ctx)
    off, lst = ctx.neighbour_lists()
    oo, ol = O.neighbours(x, y, z, h)
    assert np.array_equal(off, oo), "list lengths differ from the oracle"
    assert np.array_equal(lst, ol), "list entries differ from the oracle"
    rho = O.density_list(x, y, z, m, h, oo, ol)
    tol = SUM_TOL[precision]
    assert rel(ctx.get("rho", True), rho) < tol
    v = pass_velocity(ctx, dt)
    dv, cv = O.divcurl_list(x, y, z, v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy(), rho, m, h,
                            oo, ol)
    assert rel(ctx.get("divV", True), dv) < dc_tol_fac * tol
    assert rel(ctx.get("curlV", True), cv) < dc_tol_fac * tol
    return off, lst


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_lists_density_divcurl_vs_oracle(precision):
    """The Evrard sphere at N = 10,000 and theta 0.5: after the prologue and
    three graph-replayed steps, the step's own lists (fused pass + tree
    search for the marked particles), rho, div v and |curl v| equal the
    oracle's on the state the step left behind."""
    n, dt = 10_000, 1e-3
    d = ic.evrard(n, seed=42)
    ctx = Context(Config(n_max=n, precision=precision, theta=0.5, dt_fixed=dt,
                         av_mode="gadget", balsara=True))
    ctx.load(d["pos"], infall(d), d["m"], d["h"], d["u"])
    ctx.prologue()
    ctx.step(3)
    ctx.sync()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
    check_step_state(ctx, dt, precision)
    # h of the step solves (4 pi/3)(2h)^3 rho(h) = 64 m: one more oracle
    # Newton step from the step's h barely moves it
    x, y, z, m, h = storage(ctx)
    hh, _, _ = O.newton_h(x, y, z, m, h, max_iter=1)
    assert np.max(np.abs(hh / h - 1)) < 2e-3


def clump_in_halo(n_in=1000, n_out=3000, seed=21):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n_in, 3))
    a *= (0.35 * rng.random(n_in) ** (1 / 3) / np.linalg.norm(a, axis=1))[:, None]
    b = rng.normal(size=(n_out, 3))
    b *= (rng.random(n_out) ** (1 / 3) / np.linalg.norm(b, axis=1))[:, None]
    return np.concatenate([a, b])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_lists_with_steep_h_contrast(precision):
    """A dense clump in a sparse halo: h jumps by up to 2.6x between
    neighbours at the clump's edge, beyond the candidate radius' reach, so the
    fused pass marks particles for the tree search inside the step.  The
    lists stay exact and the densities of the re-searched particles are
    recomputed."""
    pos = clump_in_halo()
    n, dt = len(pos), 1e-4
    ctx = Context(Config(n_max=n, precision=precision, dt_fixed=dt))
    ctx.load(pos, np.zeros((n, 3)), np.full(n, 1.0 / n), np.full(n, 0.05), np.full(n, 0.05))
    ctx.prologue()
    ctx.step(1)
    ctx.sync()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0, st
    flags = ctx.debug_array("tree_search")
    assert flags[-1] == 0, "every particle went to the tree search"
    assert flags[:-1].sum() > 0, "the tree-search repair did not run"
    check_step_state(ctx, dt, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_lists_far_from_origin(precision):
    """A sphere centred at (2e4, -3e4, 1e4): the search boxes are FP32
    rounded outward, a few 1e-3 wide there, and the prefilter works in
    coordinates relative to each group's centre.  The step's lists stay
    exact and its sums match the oracle (gravity plays no part in the check:
    the dynamics only move the particles the lists are taken on)."""
    n, dt = 6000, 1e-4
    d = ic.evrard(n, seed=8)
    pos = d["pos"] + np.array([2e4, -3e4, 1e4])
    ctx = Context(Config(n_max=n, precision=precision, dt_fixed=dt, av_mode="gadget",
                         balsara=True))
    ctx.load(pos, infall(d), d["m"], d["h"], d["u"])
    ctx.prologue()
    ctx.step(2)
    ctx.sync()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
    check_step_state(ctx, dt, precision)


def test_step_lists_and_density_at_1M():
    """N = 1,000,000 Evrard in mixed precision with the headline's walk
    settings: every list of the step is bit-exact with the oracle, rho
    within the mixed tolerance on a seeded 10k subset."""
    n, dt = 1_000_000, 1e-4
    d = ic.evrard(n, seed=42)
    ctx = Context(Config(n_max=n, precision="mixed", theta=0.35, theta_local=0.28,
                         theta_small=0.45, small_cell=128, dt_fixed=dt))
    ctx.load(d["pos"], infall(d), d["m"], d["h"], d["u"])
    ctx.prologue()
    ctx.step(1)
    ctx.sync()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0, st
    x, y, z, m, h = storage(ctx)
    off, lst = ctx.neighbour_lists()
    oo, ol = O.neighbours(x, y, z, h)
    assert np.array_equal(off, oo) and np.array_equal(lst, ol)
    sub = np.random.default_rng(7).choice(n, 10_000, replace=False)
    rho = O.density_list(x, y, z, m, h, oo, ol)
    r = ctx.get("rho", True)
    assert np.max(np.abs(r[sub] / rho[sub] - 1)) < SUM_TOL["mixed"]
    ctx.close()


# ------------------------------------------- the reference's h iteration ---
@pytest.mark.parametrize("fixture", ["ref_sph_evrard_n600.npz", "ref_sph_ragged_n64.npz"])
def test_count_h_equals_reference_golden(fixture):
    """h_smooth_fast_mpi from the reference's own starting h (half the 50th
    neighbour distance) gives the reference's h bit for bit, coincident
    particles included."""
    g = dict(np.load(os.path.join(GOLD, fixture)))
    n = len(g["m"])
    ctx = Context(Config(n_max=n, precision="fp64", max_ngb=256))
    ctx.load(g["pos"], g["v"], g["m"], g["h0"], g["u"])
    ctx.sort(); ctx.build_tree()
    ctx.smoothing_h_count()
    assert ctx.status()["h_noconv"] == 0
    assert np.array_equal(ctx.get("h"), g["h"])


def test_count_h_equals_oracle_on_evrard():
    """The count iteration at N = 5,000 from a deliberately poor start
    (h off by factors 0.6..1.6, so particles take up to ~160 iterations and
    several candidate searches), bit-exact with the oracle's restatement."""
    n = 5_000
    d = ic.evrard(n, seed=4)
    h0 = d["h"] * np.random.default_rng(3).uniform(0.6, 1.6, n)
    ctx = Context(Config(n_max=n, precision="fp64"))
    ctx.load(d["pos"], d["vel"], d["m"], h0, d["u"])
    ctx.sort(); ctx.build_tree()
    ctx.smoothing_h_count()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["h_retry"] > 0, st
    ho = O.ref_h_smooth_fast(0, n, np.ascontiguousarray(d["pos"]), h0)
    assert np.array_equal(ctx.get("h"), ho)


# ------------------------------------------- two steps of the reference ---
def test_reference_loop_two_steps_vs_golden():
    """The reference's loop (sph_mpi4_v4.py:278-416) as the golden fixture
    ran it -- count iteration for h, spline-softened direct gravity with
    eps = 0.1, Gadget viscosity with the Balsara switch, fixed dt = 1e-3,
    KDK with du/dt after the closing kick and the trapezoidal u -- composed
    from the C ABI's phase entry points on the GPU: positions, velocities,
    u, h, rho and the total acceleration after two steps equal the
    reference's."""
    g = dict(np.load(os.path.join(GOLD, "ref_sph_evrard_n600.npz")))
    n, dt = len(g["m"]), 1e-3
    ctx = Context(Config(n_max=n, precision="fp64", av_mode="gadget", balsara=True,
                         alpha=1.0, beta=2.0, eta=0.1, gamma=5.0 / 3.0, dt_fixed=dt))
    ctx.load(g["pos"], np.zeros((n, 3)), g["m"], g["h"], np.full(n, 0.05))

    def gravity():
        a = ctx.gravity_direct_spline(g["eps"], np.arange(n))
        for k, f in enumerate(("ax_grav", "ay_grav", "az_grav")):
            ctx.set(f, a[:, k], storage_order=True)

    # forces at t = 0 and u += du/dt dt (sph_mpi4_v4.py:106-265)
    ctx.sort(); ctx.build_tree(); ctx.neighbours(); ctx.density()
    gravity()
    ctx.divcurl(); ctx.forces(); ctx.dudt(); ctx.update_u(first=True)
    for _ in range(2):
        ctx.kick(0.5); ctx.drift()
        ctx.sort(); ctx.build_tree(); ctx.smoothing_h_count()
        ctx.neighbours(); ctx.density()
        gravity()
        ctx.divcurl(); ctx.forces()
        ctx.kick(0.5); ctx.dudt(); ctx.update_u()
    assert ctx.status()["h_noconv"] == 0
    assert rel(ctx.get_pos(), g["step_r"]) < 1e-13
    assert rel(ctx.get_vel(), g["step_v"]) < 1e-11
    assert rel(ctx.get("u"), g["step_u"]) < 1e-11
    assert np.array_equal(ctx.get("h"), g["step_h"])
    assert rel(ctx.get("rho"), g["step_rho"]) < 1e-11
    assert rel(ctx.get_acc("sph") + ctx.get_acc("grav"), g["step_acc"]) < 1e-10


# ---------------------------------------------------------- Courant step ---
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_courant_dt_vs_oracle(precision, tol):
    """The step's Courant dt of every cloud (a 3-cloud ensemble) equals
    courant * min_i min(h_i / v_sig,i, sqrt(h_i / |a_i|)) of the oracle's
    signal velocities over the same lists."""
    e = ic.ensemble(n_clouds=3, nmin=2000, nmax=6000, seed=8)
    n = len(e["m"])
    rng = np.random.default_rng(2)
    vel = e["vel"] + 0.1 * rng.normal(size=(n, 3))
    ctx = Context(Config(n_max=n, n_cloud_max=3, precision=precision, courant=0.25,
                         av_mode="mg83"))
    ctx.load(e["pos"], vel, e["m"], e["h"], e["u"], cloud=e["cloud"])
    ctx.prologue()
    dt_gpu = ctx.dt
    x, y, z, m, h = storage(ctx)
    v = ctx.get_vel(True)
    cl = np.repeat(np.arange(3), np.bincount(e["cloud"], minlength=3))
    off, lst = ctx.neighbour_lists()
    rho, P, c = ctx.get("rho", True), ctx.get("P", True), ctx.get("c", True)
    dv, cv = ctx.get("divV", True), ctx.get("curlV", True)
    _, _, vs = O.force_list(x, y, z, v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy(), rho, P, c,
                            h, m, dv, cv, 1.0, 2.0, 0.1, 0, 0, off, lst)
    a = ctx.get_acc("sph", True) + ctx.get_acc("grav", True)
    dt_o = O.courant_dt(h, vs, a, 0.25, cl)
    assert len(dt_gpu) == 3 and np.all(dt_gpu > 0)
    assert np.max(np.abs(dt_gpu / dt_o - 1)) < tol


# ------------------------------------------------- individual time steps ---
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-5)])
def test_individual_dt_vs_oracle(precision, tol):
    """Per-particle steps of the reference's six criteria (dt_array_indiv_dt)
    over the neighbour lists, dh/dt and the power-of-two bins, after a
    prologue and two steps run with the individual step, against the
    oracle's restatement on the state the step left behind."""
    n = 10_000
    d = ic.evrard(n, seed=42)
    ctx = Context(Config(n_max=n, precision=precision, theta=0.5, dt_mode="individual",
                         courant=0.25, alpha=1.0))
    ctx.load(d["pos"], infall(d), d["m"], d["h"], d["u"])
    ctx.prologue()
    ctx.step(2)
    ctx.sync()
    dt_step = ctx.dt[0]
    r = ctx.dt_individual()
    ids = ctx.ids()
    x, y, z, m, h = storage(ctx)
    v = ctx.get_vel(True)
    off, lst = ctx.neighbour_lists()
    dto, dho = O.dt_individual(x, y, z, v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy(), m, h,
                               ctx.get("rho", True), ctx.get("c", True), ctx.get_acc("sph", True),
                               ctx.get_acc("grav", True), 1e-2, 0.25, 1.0, off, lst)
    dt_g, dh_g = r["dt"][ids], r["dhdt"][ids]            # storage order
    assert np.max(np.abs(dt_g / dto - 1)) < tol
    assert rel(dh_g, dho) < 10 * tol
    # the step's own dt was the minimum of the same estimates, and the call
    # stores that minimum again
    assert abs(dt_step / dto.min() - 1) < tol
    assert abs(ctx.dt[0] / dto.min() - 1) < tol
    # bins: ref / 2^k <= dt_i < ref / 2^(k-1), ref = the largest step
    b = r["bin"]
    ref = r["dt"].max()
    assert b.min() >= 0 and np.all(ref / 2.0 ** b <= r["dt"] * (1 + 1e-15))
    assert np.all((b == 0) | (ref / 2.0 ** (b - 1) > r["dt"]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_h_and_lists_with_sparse_outskirts(precision):
    """A dense unit ball inside a halo that thins out to 5 radii (h grows
    20-fold outwards): the wide groups of the halo widen the FP32
    prefilter's margin; the Newton h still matches the oracle and the lists
    stay exact."""
    rng = np.random.default_rng(31)
    core = rng.normal(size=(5000, 3))
    core *= (rng.random(5000) ** (1 / 3) / np.linalg.norm(core, axis=1))[:, None]
    halo = rng.normal(size=(1500, 3))
    halo *= ((1.0 + 4.0 * rng.random(1500) ** 2) / np.linalg.norm(halo, axis=1))[:, None]
    pos = np.ascontiguousarray(np.concatenate([core, halo]))
    n = len(pos)
    h0 = 1.1 * O.ref_smoothing_length(0, n, pos)
    ctx = Context(Config(n_max=n, precision=precision, max_ngb=512))
    ctx.load(pos, np.zeros((n, 3)), np.full(n, 1.0 / n), h0, np.full(n, 0.05))
    ctx.sort(); ctx.build_tree()
    ctx.smoothing_h()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
    x, y, z, m, h = storage(ctx)
    hh, _, _ = O.newton_h(x, y, z, m, h, max_iter=1)
    assert np.max(np.abs(hh / h - 1)) < 2e-3
    ctx.neighbours()
    off, lst = ctx.neighbour_lists()
    oo, ol = O.neighbours(x, y, z, h)
    assert np.array_equal(off, oo) and np.array_equal(lst, ol)


# ------------------------------------------- the reference's starting h ---
@pytest.mark.parametrize("fixture", ["ref_sph_evrard_n600.npz", "ref_sph_ragged_n64.npz"])
def test_kth_neighbour_h_equals_reference_golden(fixture):
    """smoothing_length_mpi's half 50th-neighbour distance, from a search
    radius that starts 30 % short, equals the reference's h0 bit for bit."""
    g = dict(np.load(os.path.join(GOLD, fixture)))
    n = len(g["m"])
    ctx = Context(Config(n_max=n, precision="fp64", max_ngb=256))
    ctx.load(g["pos"], g["v"], g["m"], 0.7 * g["h0"], g["u"])
    ctx.sort(); ctx.build_tree()
    ctx.smoothing_length_kth(50)
    assert ctx.status()["h_noconv"] == 0
    assert np.array_equal(ctx.get("h"), g["h0"])


def test_kth_neighbour_h_equals_oracle_on_evrard():
    n = 5_000
    d = ic.evrard(n, seed=6)
    h0 = d["h"] * np.random.default_rng(4).uniform(0.3, 2.0, n)
    ctx = Context(Config(n_max=n, precision="mixed"))
    ctx.load(d["pos"], d["vel"], d["m"], h0, d["u"])
    ctx.sort(); ctx.build_tree()
    ctx.smoothing_length_kth(50)
    assert ctx.status()["h_noconv"] == 0
    ho = O.ref_smoothing_length(0, n, np.ascontiguousarray(d["pos"]))
    assert np.array_equal(ctx.get("h"), ho)
