"""Seeded initial conditions.

* Evrard sphere (the reference's adiabatic collapse test; the reference reads
  pre-made positions from Evrard_*.pkl, MPI_sph/sph_code/sph_mpi4_v4.py:44-53,
  or stretches a 100^3 grid, Particles_in_BH_Tree_II/Evrard_test/
  IC_evrard4.cu:94-176): uniform points in the unit ball (r = U^(1/3))
  stretched r -> r^(3/2), i.e. r = U^(1/2), giving rho ~ 1/r; M = R = G = 1,
  m = M/N, u = 0.05, v = 0.
* an ensemble of independent Evrard spheres (log-uniform particle counts,
  mass, radius and u0 jittered by +-20 %).
* the cooling cloud: a uniform sphere at n = 100 cm^-3, T = 1e4 K, mu = 1.22
  with a Gaussian random velocity field of power spectrum P(k) ~ k^-4
  normalised to RMS Mach 2.

All generators draw from numpy.random.default_rng(seed) (default 42, the seed
of sph_mpi4_v4.py:17).
"""
from __future__ import annotations

import numpy as np

KB = 1.380649e-16
MH = 1.6726e-24
GCGS = 6.674e-8
MSUN = 1.989e33
PC = 3.086e18


def _ball_dirs(rng, n):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    return d


def evrard_h_guess(r, m, n_ngb=64.0, M=1.0, R=1.0):
    """Smoothing length from the analytic profile rho = M/(2 pi R^2 r)."""
    rho = M / (2.0 * np.pi * R * R * np.maximum(r, 1e-3 * R))
    return 0.5 * (3.0 * n_ngb * m / (4.0 * np.pi * rho)) ** (1.0 / 3.0)


def evrard(n, seed=42, M=1.0, R=1.0, u0=0.05, n_ngb=64.0, rng=None):
    rng = rng if rng is not None else np.random.default_rng(seed)
    r = R * np.sqrt(rng.random(n))
    pos = _ball_dirs(rng, n) * r[:, None]
    m = np.full(n, M / n)
    h = evrard_h_guess(r, m, n_ngb, M, R)
    return dict(pos=pos, vel=np.zeros((n, 3)), m=m, h=h, u=np.full(n, u0))


def ensemble(n_clouds=64, nmin=20_000, nmax=500_000, seed=42, jitter=0.2, n_ngb=64.0,
             spacing=0.0):
    """Independent Evrard spheres; cloud k occupies its own particle range.
    Positions of different clouds may overlap: they never interact."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(nmin), np.log(nmax), n_clouds)).astype(np.int64)
    parts = []
    for k, nk in enumerate(counts):
        M = 1.0 * rng.uniform(1 - jitter, 1 + jitter)
        R = 1.0 * rng.uniform(1 - jitter, 1 + jitter)
        u0 = 0.05 * rng.uniform(1 - jitter, 1 + jitter)
        ic = evrard(int(nk), M=M, R=R, u0=u0, n_ngb=n_ngb, rng=rng)
        ic["pos"] = ic["pos"] + np.array([spacing * k, 0.0, 0.0])
        ic["cloud"] = np.full(int(nk), k, np.int32)
        parts.append(ic)
    out = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    out["counts"] = counts
    return out


def turbulent_velocity(pos, rng, slope=-4.0, ngrid=64):
    """Gaussian random field with P(k) ~ k^slope on a periodic grid covering
    the particles, interpolated (nearest grid point) to the particles."""
    k1 = np.fft.fftfreq(ngrid) * ngrid
    kx, ky, kz = np.meshgrid(k1, k1, k1, indexing="ij")
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    kk[0, 0, 0] = 1.0
    amp = kk ** (slope / 2.0)
    amp[0, 0, 0] = 0.0
    v = []
    for _ in range(3):
        f = (rng.normal(size=kk.shape) + 1j * rng.normal(size=kk.shape)) * amp
        v.append(np.real(np.fft.ifftn(f)))
    lo = pos.min(0)
    ext = (pos.max(0) - lo).max() * (1 + 1e-9)
    idx = np.clip(((pos - lo) / ext * ngrid).astype(int), 0, ngrid - 1)
    vel = np.stack([vi[idx[:, 0], idx[:, 1], idx[:, 2]] for vi in v], 1)
    return vel - vel.mean(0)


def cooling_cloud(n, seed=42, n_cgs=100.0, T=1e4, mu=1.22, mach=2.0, M_sun=1000.0, gamma=5.0 / 3.0,
                  n_ngb=64.0):
    """Uniform turbulent sphere in code units (G = 1, unit mass = cloud mass,
    unit length = cloud radius) plus the code -> cgs unit factors."""
    rng = np.random.default_rng(seed)
    rho_cgs = n_cgs * mu * MH
    M = M_sun * MSUN
    R = (3.0 * M / (4.0 * np.pi * rho_cgs)) ** (1.0 / 3.0)
    unit_l, unit_m = R, M
    unit_t = np.sqrt(unit_l ** 3 / (GCGS * unit_m))
    unit_v = unit_l / unit_t
    unit_rho = unit_m / unit_l ** 3
    unit_u = unit_v ** 2
    r = rng.random(n) ** (1.0 / 3.0)
    pos = _ball_dirs(rng, n) * r[:, None]
    m = np.full(n, 1.0 / n)
    u_cgs = KB * T / ((gamma - 1.0) * mu * MH)
    cs = np.sqrt(gamma * KB * T / (mu * MH)) / unit_v
    vel = turbulent_velocity(pos, rng)
    vel *= mach * cs / np.sqrt((vel ** 2).sum(1).mean())
    rho_code = 3.0 / (4.0 * np.pi)
    h = np.full(n, 0.5 * (3.0 * n_ngb * m[0] / (4.0 * np.pi * rho_code)) ** (1.0 / 3.0))
    return dict(pos=pos, vel=vel, m=m, h=h, u=np.full(n, u_cgs / unit_u),
                units=dict(unit_rho=unit_rho, unit_u=unit_u, unit_t=unit_t, unit_l=unit_l,
                           unit_m=unit_m))


def cooling_table(n_bins=128, logT0=1.0, logT1=8.0, seed=None):
    """Synthetic piecewise power-law Lambda(T) [erg cm^3 s^-1] on n_bins+1
    log-spaced edges: a steep rise through 1e4 K, a peak near 1e5 K, a trough
    near 1e7 K and a bremsstrahlung-like T^0.5 rise; floor of 1e-27 below
    1e4 K.  Returns log10 Lambda at the edges."""
    lt = np.linspace(logT0, logT1, n_bins + 1)
    low = -27.0 + 0.5 * np.clip(lt - 1.0, 0, None)                    # slow molecular/metal tail
    hi = -21.7 - 1.5 * ((lt - 5.2) / 0.9) ** 2                         # H/He peak
    brem = -26.6 + 0.5 * (lt - 5.0)                                    # free-free
    rise = -21.7 - 10.0 * np.clip(4.2 - lt, 0, None)                   # cut-off below ~1.5e4 K
    peak = np.minimum(hi, rise)
    logL = np.log10(10 ** low + 10 ** peak + 10 ** brem)
    return logL
