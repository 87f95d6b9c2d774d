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
