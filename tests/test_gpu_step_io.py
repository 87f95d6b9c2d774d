"""sph_step_io (one step with its host transfers, the results copied out
while the step runs) against the same step through sph_set_fields +
sph_step + sph_get_fields: the same bits, in both precisions."""
import numpy as np
import pytest

from sph_2_b200 import Config, Context, ic

pytestmark = pytest.mark.gpu

IN = ["x", "y", "z", "vx", "vy", "vz", "u", "h"]
# every readiness point of the step: positions and masses after the sort, h
# after the neighbour pass, velocities after the closing kick, the rest at
# the end
OUT = IN + ["m", "rho", "ax_grav", "ay_sph", "dudt", "u_prev"]


def _pair(precision, n=20_000, seed=8):
    d = ic.evrard(n, seed=seed)
    vel = -0.3 * d["pos"] + 0.05 * np.random.default_rng(seed).normal(size=d["pos"].shape)
    ctxs = []
    for _ in range(2):
        c = Context(Config(n_max=n, precision=precision, theta=0.5))
        c.load(d["pos"], vel, d["m"], d["h"], d["u"])
        c.prologue()
        ctxs.append(c)
    return ctxs


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_io_equals_set_step_get(precision):
    a, b = _pair(precision)
    n = a.n
    state = a.get_fields(IN)
    # a perturbation the host applies between steps, fed to both contexts
    state["u"] = state["u"] * 1.01
    for k in range(3):
        a.set_fields(state)
        a.step(1)
        ref = a.get_fields(OUT)
        got = b.step_io(state, {f: np.empty(n) for f in OUT})
        for f in OUT:
            assert np.array_equal(got[f], ref[f]), (k, f)
        state = {f: ref[f].copy() for f in IN}
    a.close()
    b.close()


def test_step_io_same_arrays_in_and_out():
    """The host arrays of the inputs may receive the outputs."""
    a, b = _pair("mixed", n=8_000, seed=3)
    bufs = {f: np.ascontiguousarray(a.get(f)) for f in IN}
    a.set_fields(bufs)
    a.step(1)
    ref = a.get_fields(IN)
    b.step_io(bufs, bufs)
    for f in IN:
        assert np.array_equal(bufs[f], ref[f]), f
    a.close()
    b.close()
