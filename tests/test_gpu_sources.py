"""Outflow injection and the isothermal galaxy potential (the reference's
outflow_injector2 and galaxy_isothermal_potential, hfvCLibs_v7_hfv_v2.h:
1094-1235) through the C ABI, against the oracle's restatement."""
import numpy as np
import pytest

from oracle import oracle as O
from sph_2_b200 import Config, Context, ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_outflow_pairs_join_the_step(precision):
    n, dt = 4000, 1e-3
    d = ic.evrard(n, seed=12)
    ctx = Context(Config(n_max=n + 200, precision=precision, dt_fixed=dt))
    ctx.load(d["pos"], d["vel"], d["m"], d["h"], d["u"])
    ctx.prologue()
    m = 1.0 / n
    mdot = (20.3 * m) / dt                       # 10 pairs and 0.3 m left over
    # a gentle outflow (v_in well below the sound speed): the test is about
    # the bookkeeping, and a violent one drives u negative by pdV expansion
    kw = dict(v_in=0.05, m_particle=m, u_inject=0.05, r_max=0.02, h_first=0.05)
    added, left = ctx.outflow_inject(mdot, seed=7, **kw)
    assert added == 20 and abs(left / (0.3 * m) - 1) < 1e-9
    assert ctx.n == n + 20
    pos, vel = O.outflow_pairs(7, 10, 0.02, 0.05)
    assert rel(ctx.get_pos()[n:], pos) < 1e-14
    assert rel(ctx.get_vel()[n:], vel) < 1e-14
    assert np.all(ctx.get("m")[n:] == m) and np.all(ctx.get("h")[n:] == 0.05)
    assert np.all(ctx.get("u")[n:] == 0.05)
    # they are particles of the next steps like any other
    ctx.step(2)
    ctx.sync()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
    pos_s = ctx.get_pos(True)
    h_s = ctx.get("h", True)
    off, lst = ctx.neighbour_lists()
    oo, ol = O.neighbours(pos_s[:, 0].copy(), pos_s[:, 1].copy(), pos_s[:, 2].copy(), h_s)
    assert np.array_equal(off, oo) and np.array_equal(lst, ol)
    # the next pairs take the h of the particle injected last, and the
    # left-over mass carries over
    h_last = ctx.get("h")[n + 19]
    added2, left2 = ctx.outflow_inject(mdot, seed=8, leftover=left, **kw)
    assert added2 == 20 and abs(left2 / (0.6 * m) - 1) < 1e-9
    assert np.all(ctx.get("h")[n + 20:] == h_last)
    ctx.step(2)
    ctx.sync()
    st = ctx.status()
    assert st["h_noconv"] == 0 and st["ngb_overflow"] == 0 and st["stack_overflow"] == 0, st
    assert np.isfinite(ctx.get_pos()).all() and np.all(ctx.get("u") > 0)
    # nothing is injected past the capacity
    with pytest.raises(Exception):
        ctx.outflow_inject(1e6, seed=9, **kw)
    assert ctx.n == n + 40


def test_isothermal_potential_added_to_gravity():
    n = 6000
    d = ic.evrard(n, seed=2)
    acc = {}
    for sg in (0.0, 0.3):
        ctx = Context(Config(n_max=n, precision="fp64", theta=0.5, ext_sigma=sg))
        ctx.load(d["pos"], d["vel"], d["m"], d["h"], d["u"])
        ctx.sort(); ctx.build_tree(); ctx.gravity()
        acc[sg] = ctx.get_acc("grav")
        ctx.close()
    x, y, z = (d["pos"][:, k].copy() for k in range(3))
    assert rel(acc[0.3] - acc[0.0], O.isothermal_acc(x, y, z, 0.3)) < 1e-12
