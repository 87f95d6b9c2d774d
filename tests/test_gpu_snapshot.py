"""Context.load_ic / write_ic / write_snapshot (native host I/O in the
library) against the NumPy readers of the reference formats."""
import numpy as np
import pytest

from sph_2_b200 import Config, Context, ic
from sph_2_b200 import _lib as L
from sph_2_b200 import snapshot as S

pytestmark = pytest.mark.gpu


def _ic_file(path, n=3000, seed=4):
    d = ic.evrard(n, seed=seed)
    p, v = d["pos"], np.random.default_rng(seed).normal(scale=0.1, size=(n, 3))
    eps = np.full(n, 0.01)
    S.write_ic(path, p[:, 0], p[:, 1], p[:, 2], v[:, 0], v[:, 1], v[:, 2], d["u"], d["h"],
               d["m"], eps=eps)
    return S.read_ic(path)


def test_load_ic_and_write_back(tmp_path):
    f = _ic_file(tmp_path / "ic.bin")
    ctx = Context(Config(n_max=4096, precision="fp64"))
    eps = ctx.load_ic(tmp_path / "ic.bin", want_eps=True)
    assert ctx.n == f["N"]
    for ours, ref in (("x", "x"), ("y", "y"), ("z", "z"), ("vx", "vx"), ("vy", "vy"),
                      ("vz", "vz"), ("u", "u"), ("h", "h"), ("m", "mass")):
        assert np.array_equal(ctx.get(ours), f[ref].astype(np.float64)), ours
    assert np.array_equal(eps, f["eps"].astype(np.float64))
    ctx.write_ic(tmp_path / "back.bin", eps=eps)
    assert (tmp_path / "back.bin").read_bytes() == (tmp_path / "ic.bin").read_bytes()
    ctx.close()


def test_snapshot_after_prologue(tmp_path):
    _ic_file(tmp_path / "ic.bin")
    ctx = Context(Config(n_max=4096, precision="mixed"))
    ctx.load_ic(tmp_path / "ic.bin")
    ctx.write_snapshot(tmp_path / "s0.bin")
    assert (S.read_snapshot(tmp_path / "s0.bin")["debug"] == -1).all()
    ctx.prologue()
    ctx.step(2)
    ctx.sort()
    ctx.build_tree()
    ctx.smoothing_h()
    ctx.neighbours()
    ion = np.linspace(0, 1, 5, dtype=np.float32)
    ctx.write_snapshot(tmp_path / "s1.bin", ion_frac=ion)
    r = S.read_snapshot(tmp_path / "s1.bin")
    assert r["N"] == ctx.n and (r["Typ"] == 0).all()
    for ours, ref in (("x", "x"), ("vz", "vz"), ("rho", "rho"), ("h", "h"), ("u", "u"),
                      ("m", "mass")):
        assert np.array_equal(r[ref], ctx.get(ours).astype(np.float32)), ours
    off, _ = ctx.neighbour_lists()
    cnt = np.diff(off)
    ids = ctx.ids()
    want = np.empty(ctx.n, np.int64)
    want[ids] = cnt
    assert np.array_equal(r["debug"], want)
    assert np.array_equal(r["ionFrac"], ion)
    ctx.close()


def test_ic_with_other_particle_types_is_rejected(tmp_path):
    n = 10
    z = np.zeros(n)
    typ = np.zeros(n, np.int32)
    typ[3] = -1                                  # a black hole
    S.write_ic(tmp_path / "bh.bin", z, z, z, z, z, z, z + 1, z + 0.1, z + 0.1, typ=typ)
    ctx = Context(Config(n_max=64))
    with pytest.raises(L.SphError) as e:
        ctx.load_ic(tmp_path / "bh.bin")
    assert e.value.code == -1
    with pytest.raises(L.SphError):
        Context(Config(n_max=4)).load_ic(tmp_path / "bh.bin")
    ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_resumes_bit_for_bit(tmp_path, precision):
    """A context that reads an FP64 restart file continues exactly as the one
    that wrote it: three more steps (Courant dt per cloud, a 3-cloud ensemble)
    give the same bits in every field and step."""
    e = ic.ensemble(n_clouds=3, nmin=2000, nmax=5000, seed=12)
    n = len(e["m"])
    rng = np.random.default_rng(3)
    vel = e["vel"] + 0.05 * rng.normal(size=(n, 3))
    cfg = dict(n_max=n, n_cloud_max=3, precision=precision, theta=0.5, balsara=True,
               av_mode="gadget")
    a = Context(Config(**cfg))
    a.load(e["pos"], vel, e["m"], e["h"], e["u"], cloud=e["cloud"])
    a.prologue()
    a.step(4)
    a.sync()
    path = tmp_path / "restart.bin"
    a.write_restart(path)
    a.step(3)
    a.sync()
    b = Context(Config(**cfg))
    b.read_restart(path)
    assert b.n == n and b.n_clouds == 3
    b.step(3)
    b.sync()
    for f in ("x", "y", "z", "vx", "vy", "vz", "u", "h", "rho", "dudt", "ax_grav", "ax_sph"):
        assert np.array_equal(a.get(f), b.get(f)), f
    assert np.array_equal(a.dt, b.dt)
    assert np.array_equal(a.ids(), b.ids())
