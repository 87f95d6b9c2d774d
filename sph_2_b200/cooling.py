"""Cooling on the device: the implicit solve and its learned surrogate.

The physics is the implicit per-particle energy update of the reference's
DoCooling (GPU_sph/With_cooling/Model_C/myPhotoLibsGPU.h:615-686) over a
synthetic power-law cooling table (see ic.cooling_table).  The surrogate is a
3 -> 64 -> 64 -> 1 MLP trained on the device by the library's own BF16
tensor-core kernels on (log10 rho, log10 u, log10 dt) -> log10(u_new/u_old)
samples labelled by the exact solver; at run time its prediction is refined by
one Newton step and checked by a residual error estimate, with the exact solve
as fallback.  Everything here only moves arrays and launches library calls.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from . import ic

DEFAULT = dict(n_bins=128, max_iter=200, logT0=1.0, logT1=8.0, mu=1.22, gamma=5.0 / 3.0, XH=0.7,
               gamma_heat=2e-26, tol=1e-6, unit_rho=1.0, unit_u=1.0, unit_t=1.0, mlp_err_tol=1e-3)
# sampling box of the training set (cgs): densities of ~2 to 2e5 H/cm^3,
# temperatures 30 K .. 1e6 K, steps of 3e9 .. 1e13 s
RANGES = dict(log_rho=(-23.5, -18.5), log_T=(1.5, 6.0), log_dt=(9.5, 13.0))


def setup(ctx, units: dict | None = None, **kw) -> dict:
    p = dict(DEFAULT)
    if units:
        p.update({k: units[k] for k in ("unit_rho", "unit_u", "unit_t")})
    p.update(kw)
    table = ic.cooling_table(p["n_bins"], p["logT0"], p["logT1"])
    ctx.cooling_setup(p, table)
    p["table"] = table
    return p


def u_of_T(T, mu=1.22, gamma=5.0 / 3.0):
    return ic.KB * T / ((gamma - 1.0) * mu * ic.MH)


def sample_states(n, seed=42, ranges=RANGES, mu=1.22, gamma=5.0 / 3.0):
    rng = np.random.default_rng(seed)
    lr = rng.uniform(*ranges["log_rho"], n)
    lT = rng.uniform(*ranges["log_T"], n)
    ldt = rng.uniform(*ranges["log_dt"], n)
    return 10.0 ** lr, u_of_T(10.0 ** lT, mu, gamma), 10.0 ** ldt


def training_set(ctx, n=5_000_000, seed=42, ranges=RANGES):
    """Features, targets and their normalisation from the exact GPU solve."""
    rho, u, dt = sample_states(n, seed, ranges)
    u_new, it = ctx.cool_solve(rho, u, dt)
    X = np.stack([np.log10(rho), np.log10(u), np.log10(dt)], 1)
    y = np.log10(u_new / u)
    mean, scale = X.mean(0), X.std(0)
    ym, ys = y.mean(), y.std() + 1e-12
    norm = np.array([*mean, *scale, ym, ys], np.float32)
    Xn = ((X - mean) / scale).astype(np.float32)
    yn = ((y - ym) / ys).astype(np.float32)
    return Xn, yn, norm, dict(rho=rho, u=u, dt=dt, u_new=u_new, iters=it)


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    W1 = rng.normal(scale=np.sqrt(2.0 / 3.0), size=(3, 64))
    W2 = rng.normal(scale=np.sqrt(2.0 / 64.0), size=(64, 64))
    W3 = rng.normal(scale=np.sqrt(1.0 / 64.0), size=64)
    return np.concatenate([W1.ravel(), np.zeros(64), W2.ravel(), np.zeros(64), W3, [0.0]]).astype(np.float32)


def unpack(P):
    P = np.asarray(P, np.float32)
    return (P[:192].reshape(3, 64), P[192:256], P[256:4352].reshape(64, 64), P[4352:4416],
            P[4416:4480].reshape(64, 1), P[4480:4481])


def train(ctx, Xn, yn, steps=4000, batch=4096, lr=2e-3):
    """Adam on the device; X and y are uploaded once (torch owns the buffers)."""
    import torch
    dX = torch.as_tensor(np.ascontiguousarray(Xn), device="cuda")
    dy = torch.as_tensor(np.ascontiguousarray(yn), device="cuda")
    loss = C.c_float()
    rc = L.load().sph_mlp_train(ctx.handle, len(yn), C.c_void_p(dX.data_ptr()),
                                C.c_void_p(dy.data_ptr()), batch, steps, C.c_float(lr),
                                C.byref(loss))
    L.check(rc, "sph_mlp_train", ctx.handle)
    return float(loss.value)


# ---- grid files of the table backend ---------------------------------------
TABLE_DIMS = ("N_kpc", "N_nH", "N_Z", "N_T", "N_M", "N_Time")


def write_table_file(path, kpc, nH, Z, T, time_s, u_evol, mu, frac):
    """Write a heating/cooling grid in the layout of the reference's
    coolHeatGridNew.bin (read by hfvGpuSphBHtree_v3_check_v1_cooling_t3_
    Evrard.cu:137-179): int32 N_kpc, N_nH, N_Z, N_T, N_M, N_Time; float32
    grids kpc, nH, Z, T, time; float32 u_evol and mu [kpc][T][nH][Z][time];
    float32 ion fractions [kpc][T][nH][Z][M][time]."""
    kpc, nH, Z, T, time_s = (np.asarray(a, np.float32) for a in (kpc, nH, Z, T, time_s))
    u_evol = np.asarray(u_evol, np.float32)
    frac = np.asarray(frac, np.float32)
    nk, nt, nh, nz, ntime = u_evol.shape
    nm = frac.shape[4]
    assert (nk, nh, nz, nt, ntime) == (len(kpc), len(nH), len(Z), len(T), len(time_s))
    assert frac.shape == (nk, nt, nh, nz, nm, ntime) and np.shape(mu) == u_evol.shape
    with open(path, "wb") as f:
        np.array([nk, nh, nz, nt, nm, ntime], np.int32).tofile(f)
        for a in (kpc, nH, Z, T, time_s, u_evol, np.asarray(mu, np.float32), frac):
            np.ascontiguousarray(a).tofile(f)


def read_table_file(path):
    """The arrays of a grid file written by write_table_file (or by the
    reference's own table builder)."""
    raw = np.fromfile(path, np.uint8)
    nk, nh, nz, nt, nm, ntime = (int(v) for v in raw[:24].view(np.int32))
    f = raw[24:].view(np.float32)
    out, o = {}, 0
    for name, k in (("kpc", nk), ("nH", nh), ("Z", nz), ("T", nt), ("time_s", ntime)):
        out[name] = f[o:o + k].copy()
        o += k
    c5 = nk * nt * nh * nz * ntime
    out["u_evol"] = f[o:o + c5].reshape(nk, nt, nh, nz, ntime).copy()
    o += c5
    out["mu"] = f[o:o + c5].reshape(nk, nt, nh, nz, ntime).copy()
    o += c5
    out["frac"] = f[o:o + c5 * nm].reshape(nk, nt, nh, nz, nm, ntime).copy()
    return out


def synthetic_table(seed=0, n_kpc=4, n_nH=40, n_Z=3, n_T=60, n_M=3, n_time=12, mu=1.22):
    """A seeded synthetic grid in the reference's layout (the reference's
    CHIMES-made coolHeatGridNew.bin is not in its repository): radius 0.01-10
    kpc, n_H 1e-2-1e4 cm^-3, T 1e1-1e8 K, times 1e8-1e14 s; u(t) relaxes from
    the initial u(T) towards the equilibrium of a cooling time that falls with
    n_H and is shortest near 1e5 K, and the M ion fractions are a normalised
    seeded function of (T, n_H)."""
    rng = np.random.default_rng(seed)
    kpc = np.logspace(-2, 1, n_kpc)
    nH = np.logspace(-2, 4, n_nH)
    Z = np.array([-2.0, -1.0, 0.0][:n_Z] + [0.5] * max(0, n_Z - 3))
    T = np.logspace(1, 8, n_T)
    time_s = np.logspace(8, 14, n_time)
    u0 = u_of_T(T, mu)                                    # [T]
    u_eq = u_of_T(1e4, mu)
    lt = np.log10(T)
    tcool = 1e13 / nH[None, :] * (1.0 + 30.0 * np.exp(-((lt[:, None] - 5.0) / 0.8) ** 2)) ** -1
    shape = (n_kpc, n_T, n_nH, n_Z, n_time)
    u_evol = np.empty(shape)
    for k in range(n_kpc):
        heat = 1.0 + 0.2 * k
        for z in range(n_Z):
            zf = 1.0 + 0.3 * z
            decay = np.exp(-time_s[None, None, :] * zf / tcool[:, :, None])   # [T, nH, time]
            u_evol[k, :, :, z, :] = heat * u_eq + (u0[:, None, None] - heat * u_eq) * decay
    mu_arr = np.full(shape, mu) * (1.0 + 0.05 * rng.random(shape))
    w = rng.random((n_kpc, n_T, n_nH, n_Z, n_M, n_time)) + 0.1
    w[:, :, :, :, 0, :] *= (1.0 / (1.0 + (T / 1e4) ** 4))[None, :, None, None, None]
    frac = w / w.sum(axis=4, keepdims=True)
    return dict(kpc=kpc, nH=nH, Z=Z, T=T, time_s=time_s, u_evol=u_evol, mu=mu_arr, frac=frac)
