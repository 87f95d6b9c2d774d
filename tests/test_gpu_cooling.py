"""Implicit cooling and the MLP surrogate on the GPU against the CPU oracle.

* the FP64 bracket-and-bisect solve equals the oracle's restatement of
  DoCooling (myPhotoLibsGPU.h:615-686) over the same synthetic table;
* the tensor-core forward pass and gradient equal a NumPy restatement with the
  same BF16 rounding points;
* training on exact-solver labels lowers the loss, and the surrogate path
  (prediction + one Newton step + residual check + exact fallback) stays
  within its error tolerance of the exact solution on every row.
"""
import time

import numpy as np
import pytest

from oracle import oracle as O
from sph_2_b200 import Config, Context, cooling

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(Config(n_max=1024, precision="mixed"))
    cooling.setup(c)
    yield c
    c.close()


def test_exact_solve_matches_oracle(ctx):
    p = cooling.DEFAULT
    rho, u, dt = cooling.sample_states(20_000, seed=5)
    u_gpu, it_gpu = ctx.cool_solve(rho, u, dt)
    table = cooling.ic.cooling_table(p["n_bins"], p["logT0"], p["logT1"])
    u_orc, it_orc = O.do_cooling(table, p["logT0"], p["logT1"], p["mu"], p["gamma"], p["XH"],
                                 p["gamma_heat"], rho, u, dt, tol=p["tol"], max_iter=p["max_iter"])
    assert (it_gpu > 0).all() and (it_orc > 0).all()
    rel = np.abs(u_gpu / u_orc - 1)
    # same bracketing and bisection: equal up to the bisection tolerance where a
    # last-ulp difference of log10/pow flips one branch decision
    assert np.median(rel) < 1e-12
    assert rel.max() < 4 * p["tol"]
    assert np.mean(it_gpu == it_orc) > 0.99


def test_mlp_forward_matches_oracle(ctx):
    P = cooling.init_params(seed=3)
    P[192:256] = np.linspace(-0.1, 0.1, 64)
    P[4352:4416] = np.linspace(0.1, -0.1, 64)
    P[4480] = 0.05
    ctx.mlp_set(P, np.array([0, 0, 0, 1, 1, 1, 0, 1], np.float32))
    X = np.random.default_rng(1).normal(size=(1000, 3)).astype(np.float32)
    y = ctx.mlp_forward(X)
    yo, _ = O.mlp_forward_bf16(X, *cooling.unpack(P))
    assert np.max(np.abs(y - yo)) < 2e-3 * (np.max(np.abs(yo)) + 1e-6)


def test_mlp_gradient_matches_oracle(ctx):
    P = cooling.init_params(seed=4)
    ctx.mlp_set(P, np.array([0, 0, 0, 1, 1, 1, 0, 1], np.float32))
    rng = np.random.default_rng(2)
    X = rng.normal(size=(1500, 3)).astype(np.float32)     # 6 blocks, a ragged last one
    t = np.tanh(X @ np.array([0.5, -1.0, 0.3], np.float32)).astype(np.float32)
    g, loss = ctx.mlp_grad(X, t)
    go, lo = O.mlp_grad_bf16(X, t, *cooling.unpack(P))
    assert abs(loss - lo) < 1e-3 * lo
    for a, b, name in [(0, 192, "W1"), (192, 256, "b1"), (256, 4352, "W2"), (4352, 4416, "b2"),
                       (4416, 4480, "W3"), (4480, 4481, "b3")]:
        num = np.linalg.norm(g[a:b] - go[a:b])
        den = np.linalg.norm(go[a:b]) + 1e-12
        assert num / den < 2e-2, name
        cos = float(g[a:b] @ go[a:b]) / (np.linalg.norm(g[a:b]) * np.linalg.norm(go[a:b]) + 1e-30)
        assert cos > 0.999, name


def test_training_and_surrogate_within_tolerance():
    c = Context(Config(n_max=1024, precision="mixed"))
    p = cooling.setup(c)
    Xn, yn, norm, raw = cooling.training_set(c, n=200_000, seed=11)
    c.mlp_set(cooling.init_params(seed=0), norm)
    _, loss0 = c.mlp_grad(Xn[:20000], yn[:20000])
    loss = cooling.train(c, Xn, yn, steps=3000, batch=4096, lr=2e-3)
    _, loss1 = c.mlp_grad(Xn[:20000], yn[:20000])
    assert loss1 < 0.1 * loss0, (loss0, loss1, loss)
    # unseen states: surrogate path vs exact solve
    rho, u, dt = cooling.sample_states(100_000, seed=99)
    t0 = time.perf_counter()
    u_ex, _ = c.cool_solve(rho, u, dt)
    t1 = time.perf_counter()
    u_ml, fb = c.cool_solve_mlp(rho, u, dt)
    t2 = time.perf_counter()
    err = np.abs(u_ml / u_ex - 1)
    # rows answered by the surrogate are within the tolerance the estimate
    # promises (plus the exact solve's own bisection tolerance)
    acc = fb == 0
    assert acc.mean() > 0.5
    assert np.percentile(err[acc], 99.9) < p["mlp_err_tol"] + 2 * p["tol"]
    assert err.max() < 10 * p["mlp_err_tol"]
    c.close()
    print(f"surrogate rows {acc.mean():.3f}, exact {t1 - t0:.3f}s, surrogate {t2 - t1:.3f}s")


def test_surrogate_gain_over_exact_solve():
    """What the trained network buys: the cooling solve of 2^20 unseen states
    through the surrogate path (prediction, one Newton step, acceptance test,
    exact fallback for the rows it does not answer) against the exact
    bracket-and-bisect solve of the same states, both on the device, both
    timed with CUDA events on the library's stream."""
    import ctypes as C

    import torch

    from sph_2_b200 import _lib as L

    n = 1 << 20
    c = Context(Config(n_max=n, precision="mixed"))
    p = cooling.setup(c)
    Xn, yn, norm, _ = cooling.training_set(c, n=200_000, seed=11)
    c.mlp_set(cooling.init_params(seed=0), norm)
    cooling.train(c, Xn, yn, steps=3000, batch=4096, lr=2e-3)
    rho, u, dt = cooling.sample_states(n, seed=99)
    s = torch.cuda.Stream()
    c.set_stream(s.cuda_stream)
    dv = [torch.as_tensor(np.ascontiguousarray(a, np.float64), device="cuda") for a in (rho, u, dt)]
    ue, um = torch.empty_like(dv[1]), torch.empty_like(dv[1])
    fb = torch.empty(n, dtype=torch.int32, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())
    lib = L.load()
    torch.cuda.synchronize()

    def exact():
        L.check(lib.sph_cool_solve(c.handle, n, ptr(dv[0]), ptr(dv[1]), ptr(dv[2]), ptr(ue), None, 0),
                "sph_cool_solve", c.handle)

    def surrogate():
        L.check(lib.sph_cool_solve_mlp(c.handle, n, ptr(dv[0]), ptr(dv[1]), ptr(dv[2]), ptr(um),
                                       ptr(fb)), "sph_cool_solve_mlp", c.handle)

    def timed(fn, reps=3):
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    t_exact, t_mlp = timed(exact), timed(surrogate)
    u_ex, u_ml, f = ue.cpu().numpy(), um.cpu().numpy(), fb.cpu().numpy()
    err = np.abs(u_ml / u_ex - 1)
    acc = f == 0
    assert acc.mean() > 0.5
    assert np.percentile(err[acc], 99.9) < p["mlp_err_tol"] + 2 * p["tol"]
    assert err.max() < 10 * p["mlp_err_tol"]
    print(f"cooling solve of {n} states: exact {t_exact:.3f} ms, surrogate {t_mlp:.3f} ms "
          f"({t_exact / t_mlp:.2f}x), answered by the surrogate {acc.mean():.3f}")
    assert t_mlp < t_exact
    c.close()


def test_cooling_collapse_stays_positive():
    """An Evrard sphere scaled so that u = 0.05 is 1e6 K at 100 H/cm^3 cools
    by orders of magnitude in its first steps; the trapezoidal u update with
    the pre-cooling du/dt would then overshoot below zero.  The cooled run
    keeps u positive and every field finite."""
    from sph_2_b200 import ic
    n = 20_000
    d = ic.evrard(n, seed=42)
    kb, mh, gcgs, mu, gam = 1.380649e-16, 1.6726e-24, 6.674e-8, 1.22, 5.0 / 3.0
    unit_u = kb * 1e6 / ((gam - 1.0) * mu * mh) / 0.05
    R = (3.0 * unit_u / gcgs / (4.0 * np.pi * 100.0 * mu * mh)) ** 0.5
    M = unit_u * R / gcgs
    units = {"unit_rho": M / R ** 3, "unit_u": unit_u, "unit_t": (R ** 3 / (gcgs * M)) ** 0.5}
    c = Context(Config(n_max=n, precision="mixed", theta=0.5, flags=2))   # cooling on
    cooling.setup(c, units)
    c.load(d["pos"], d["vel"], d["m"], d["h"], d["u"])
    c.prologue()
    c.step(10)
    c.sync()
    u = c.get("u")
    assert np.all(u > 0) and u.max() < 0.05
    assert np.isfinite(c.get("x")).all() and np.isfinite(c.get("vx")).all()
    st = c.status()
    assert st["nonfinite"] == 0 and st["h_noconv"] == 0 and st["cool_noconv"] == 0
    c.close()


# ------------------------------------------------- table backend (hcoolingx) ---
def test_table_cooling_matches_oracle(tmp_path):
    """The grid-file backend (hcoolingx, hfvCLibs_v7_hfv_v2.h:1240-1418) on a
    seeded synthetic grid in the reference's coolHeatGridNew.bin layout: new
    u and ion fractions bit-exact with the oracle's restatement, inside and
    outside the grid's ranges; then two steps with the table backend on."""
    from oracle import oracle as O
    from sph_2_b200 import Config, Context, cooling, ic
    from sph_2_b200 import _lib as L
    path = tmp_path / "coolHeatGridNew.bin"
    cooling.write_table_file(path, **cooling.synthetic_table(seed=3))
    tab = cooling.read_table_file(path)
    n, dt = 5000, 2e-3
    d = ic.evrard(n, seed=5)
    rng = np.random.default_rng(9)
    rho = 10 ** rng.uniform(-3.5, 3.0, n)          # code units; n_H 1e-3 .. 4e4 cm^-3
    u = 10 ** rng.uniform(-3.0, 3.5, n)
    units = dict(unit_rho=1.0e-24, unit_u=1.0e10, unit_t=1.0e14, unit_length=3.0 * 3.086e21)
    ctx = Context(Config(n_max=n, precision="fp64", dt_fixed=dt,
                         flags=L.FLAG_COOLING | L.FLAG_COOLING_TABLE))
    ctx.load(d["pos"], d["vel"], d["m"], d["h"], u)
    ctx.set("rho", rho)
    ctx.cooling_table_load(path, **units)
    ctx.cooling_table()
    un, ion = O.cool_table(tab, *(d["pos"][:, k].copy() for k in range(3)), rho, u, dt,
                           unit_rho=units["unit_rho"], unit_u=units["unit_u"],
                           unit_t=units["unit_t"], unit_len=units["unit_length"])
    assert np.array_equal(ctx.get("u"), un)
    assert np.array_equal(ctx.ion_frac(tab["frac"].shape[4]), ion)
    assert np.any(un != u)
    # in the step: cooling with the table after the u update
    ctx.load(d["pos"], d["vel"], d["m"], d["h"], np.full(n, 0.05))
    ctx.prologue()
    ctx.step(2)
    ctx.sync()
    assert np.isfinite(ctx.get("u")).all() and np.all(ctx.get("u") > 0)
    f = ctx.ion_frac(tab["frac"].shape[4])
    assert np.allclose(f.sum(axis=1), 1.0, atol=1e-5)


def test_tcgen05_inference_matches_warp_mma(ctx):
    """The surrogate's inference on tcgen05.mma with a TMEM accumulator (128
    rows per CTA) against the warp-level mma.sync path: the same BF16 products
    with FP32 accumulation, so the outputs agree to FP32 rounding, over a
    ragged row count (partial last tile), and no wait gave up."""
    from sph_2_b200 import _lib as L
    P = cooling.init_params(seed=5)
    P[192:256] = np.linspace(-0.2, 0.2, 64)
    ctx.mlp_set(P, np.array([0, 0, 0, 1, 1, 1, 0, 1], np.float32))
    X = np.random.default_rng(6).normal(size=(1000, 3)).astype(np.float32)
    ctx.status(reset=True)
    y_tc = ctx.mlp_forward(X)
    base = ctx.config.flags
    ctx.set_params(flags=base | L.FLAG_MLP_WARP_MMA)
    try:
        y_w = ctx.mlp_forward(X)
    finally:
        ctx.set_params(flags=base)
    assert np.isfinite(y_tc).all()
    assert np.max(np.abs(y_tc - y_w)) < 1e-4 * (np.max(np.abs(y_w)) + 1e-6)
    yo, _ = O.mlp_forward_bf16(X, *cooling.unpack(P))
    assert np.max(np.abs(y_tc - yo)) < 2e-3 * (np.max(np.abs(yo)) + 1e-6)
    assert ctx.status()["wait_timeout"] == 0
