"""Drop-in replacements for the reference's step-level CPU functions, with the
same names, argument order and return shapes as MPI_sph/sph_code/libsx.py and
shear.py, computed by this package's CUDA kernels.

The reference evaluates every pair (i, j) for the rows i in [nbeg, nend) and
returns new NumPy arrays; the MPI driver (sph_mpi4_v4.py:57-65) gives each rank
a row range and gathers the pieces.  Here one GPU holds all particles: each
call loads the arrays into a device context kept per (N, precision), builds the
Morton order, the radix tree and the exact neighbour lists of the caller's h
(|r_ij| <= h_i + h_j, the support of the kernel at h_ij = (h_i + h_j)/2, so
the sums equal the reference's all-pairs sums), runs the one phase asked for
and returns rows nbeg..nend-1.  Inputs may be NumPy arrays (copied) or torch
CUDA tensors (device-to-device copies, no host round trip).  There is no CPU
path: without the library or a GPU every call raises.

h_smooth_fast_mpi / h_smooth_fast run the reference's own +-0.3 % count
iteration (libsx.py:806-902) on the GPU and return the same h bit for bit.
The project's Newton smoothing length, which solves (4 pi / 3)(2h)^3 rho(h) =
N_ngb m, is offered under its own name, h_newton_mpi.

smoothing_length_mpi (half the 50th-neighbour distance, libsx.py:777-800) is
the reference's too, bit for bit.

Differences from the reference, by design:
* getPressure / getCsound / getKE are elementwise host formulas (no kernel is
  worth a launch there); getPE is the FP64 sum of the tree walk's Plummer
  potential.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .core import Config, Context

__all__ = [
    "getDensity", "getDensity_mpi", "div_curlVel", "div_curlVel_mpi", "getPressure", "getCsound",
    "getAcc_sph", "getAcc_sph_mpi", "getAcc_sph_mpiXXX", "get_dU", "get_dU_mpi",
    "get_dU_mpiXXXX", "getAcc_sph_shear", "getAcc_sph_shear_mpi", "get_dU_shear",
    "get_dU_shear_mpi", "getAcc_g_smth_mimj_mpi", "h_smooth_fast_mpi", "h_smooth_fast",
    "h_newton_mpi",
    "smoothing_length_mpi", "getKE", "getPE", "precision", "release",
]

_PREC = ["fp64"]
_CTX: dict = {}


def precision(p: str | None = None) -> str:
    """Get or set the arithmetic of later calls: "fp64" (default, as the
    reference) or "mixed" (FP32 sums with Kahan compensation)."""
    if p is not None:
        if p not in L.PREC:
            raise ValueError(f"precision must be one of {sorted(L.PREC)}")
        _PREC[0] = p
    return _PREC[0]


def release():
    """Free every cached device context."""
    for c in _CTX.values():
        c.close()
    _CTX.clear()


def _ctx(n: int) -> Context:
    key = (n, _PREC[0])
    c = _CTX.get(key)
    if c is None:
        c = Context(Config(n_max=max(n, 1), precision=_PREC[0], max_ngb=512))
        _CTX[key] = c
    return c


def _is_cuda_tensor(a) -> bool:
    return hasattr(a, "is_cuda") and bool(getattr(a, "is_cuda"))


def _column(a, k=None):
    """A C-contiguous float64 column: (pointer, host flag, keep-alive)."""
    if _is_cuda_tensor(a):
        import torch
        t = (a[:, k] if k is not None else a).to(torch.float64).contiguous()
        # the library reads it on its own stream: let torch's work finish first
        torch.cuda.current_stream().synchronize()
        return C.c_void_p(t.data_ptr()), 0, t
    x = np.ascontiguousarray(np.asarray(a)[:, k] if k is not None else a, dtype=np.float64)
    return x.ctypes.data_as(C.c_void_p), 1, x


def _load_state(pos, m, h, v=None):
    """Load positions (and velocities, masses, h) into the cached context and
    bring it to Morton order with a fresh tree."""
    n = int(pos.shape[0])
    ctx = _ctx(n)
    keep, args, hosts = [], [], set()
    cols = [(pos, 0), (pos, 1), (pos, 2)]
    cols += [(v, 0), (v, 1), (v, 2)] if v is not None else [None, None, None]
    cols += [(m, None), (h, None)]
    for c in cols:
        if c is None:
            args.append(None)
            continue
        p, host, k = _column(*c)
        args.append(p)
        hosts.add(host)
        keep.append(k)
    if len(hosts) != 1:
        raise ValueError("mix of host arrays and CUDA tensors in one call")
    host = hosts.pop()
    u = np.zeros(n) if host else _zeros_like_dev(n)
    pu = u.ctypes.data_as(C.c_void_p) if host else C.c_void_p(u.data_ptr())
    x, y, z, vx, vy, vz, pm, ph = args
    ctx._chk(ctx._L.sph_load(ctx._h, n, None, x, y, z, vx, vy, vz, pm, ph, pu, host), "sph_load")
    ctx.sync()   # the copies have read `keep` before it goes out of scope
    ctx.sort()
    ctx.build_tree()
    return ctx


def _load(pos, m, h, v=None):
    """_load_state plus the exact neighbour lists of the given h."""
    ctx = _load_state(pos, m, h, v)
    ctx.neighbours()
    st = ctx.status(reset=True)
    if st["ngb_overflow"] or st["stack_overflow"]:
        raise L.SphError(-5, "neighbour lists", "(more than 512 neighbours for some particle)")
    return ctx


def _zeros_like_dev(n):
    import torch
    return torch.zeros(n, dtype=torch.float64, device="cuda")


def _set(ctx, name, a):
    p, host, keep = _column(a)
    ctx._chk(ctx._L.sph_set_field(ctx._h, L.FIELD[name], p, host, 0), f"set {name}")
    return keep


def _out(ctx, name, like):
    """Field in original order, as a NumPy array or (for CUDA inputs) a tensor."""
    if _is_cuda_tensor(like):
        import torch
        t = torch.empty(ctx.n, dtype=torch.float64, device="cuda")
        ctx._chk(ctx._L.sph_get_field(ctx._h, L.FIELD[name], C.c_void_p(t.data_ptr()), 0, 0),
                 f"get {name}")
        return t
    return ctx.get(name)


def _rows(a, nbeg, nend):
    return a[nbeg:nend]


def _physics(ctx, av, balsara, alpha, beta=2.0, eta=0.1, gama=None):
    kw = dict(av_mode=av, balsara=balsara, alpha=float(alpha), beta=float(beta), eta=float(eta))
    if gama is not None:
        kw["gamma"] = float(gama)
    ctx.set_params(**kw)


# ---- density and velocity derivatives -----------------------------------
def getDensity_mpi(nbeg, nend, pos, m, h):
    """libsx.py:52-86: rho_i = sum_j m_j W(r_ij, h_ij), rows nbeg..nend-1."""
    ctx = _load(pos, m, h)
    ctx.density()
    return _rows(_out(ctx, "rho", pos), nbeg, nend)


def getDensity(pos, m, h):
    """libsx.py:11-47 (all rows)."""
    return getDensity_mpi(0, pos.shape[0], pos, m, h)


def div_curlVel_mpi(nbeg, nend, pos, v, rho, m, h):
    """shear.py:78-142: (|div v|, |curl v|) of rows nbeg..nend-1."""
    ctx = _load(pos, m, h, v)
    _set(ctx, "rho", rho)
    ctx.divcurl()
    return (_rows(_out(ctx, "divV", pos), nbeg, nend), _rows(_out(ctx, "curlV", pos), nbeg, nend))


def div_curlVel(pos, v, rho, m, h):
    """shear.py:8-73 (all rows)."""
    return div_curlVel_mpi(0, pos.shape[0], pos, v, rho, m, h)


# ---- SPH accelerations and du/dt ------------------------------------------
def _sph_pass(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, want):
    ctx = _load(pos, m, h, v)
    keep = [_set(ctx, "rho", rho), _set(ctx, "P", P), _set(ctx, "c", c)]
    if divV is not None:
        keep += [_set(ctx, "divV", divV), _set(ctx, "curlV", curlV)]
    if want == "acc":
        ctx.forces()
        if _is_cuda_tensor(pos):
            import torch
            a = torch.stack([_out(ctx, f"a{k}_sph", pos) for k in "xyz"], 1)
        else:
            a = ctx.get_acc("sph")
        return a[nbeg:nend]
    ctx.dudt()
    return _rows(_out(ctx, "dudt", pos), nbeg, nend)


def getAcc_sph_shear_mpi(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, alpha):
    """shear.py:243-330: signal-velocity viscosity with the Balsara switch."""
    ctx = _ctx(int(pos.shape[0]))
    _physics(ctx, "gadget", True, alpha)
    return _sph_pass(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, "acc")


def getAcc_sph_shear(pos, v, rho, P, c, h, m, divV, curlV, alpha):
    """shear.py:151-238 (all rows)."""
    return getAcc_sph_shear_mpi(0, pos.shape[0], pos, v, rho, P, c, h, m, divV, curlV, alpha)


def get_dU_shear_mpi(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, alpha):
    """shear.py:413-485."""
    ctx = _ctx(int(pos.shape[0]))
    _physics(ctx, "gadget", True, alpha)
    return _sph_pass(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, "du")


def get_dU_shear(pos, v, rho, P, c, h, m, divV, curlV, alpha):
    """shear.py:334-408 (all rows)."""
    return get_dU_shear_mpi(0, pos.shape[0], pos, v, rho, P, c, h, m, divV, curlV, alpha)


def getAcc_sph_mpiXXX(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """libsx.py:185-262: Monaghan & Gingold (1983) viscosity."""
    ctx = _ctx(int(pos.shape[0]))
    _physics(ctx, "mg83", False, alpha, beta, eta, gama)
    return _sph_pass(nbeg, nend, pos, v, rho, P, c, h, m, None, None, "acc")


def getAcc_sph(pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """libsx.py:102-180 (Monaghan & Gingold, all rows)."""
    return getAcc_sph_mpiXXX(0, pos.shape[0], pos, v, rho, P, c, h, m, gama, eta, alpha, beta)


def getAcc_sph_mpi(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """libsx.py:270-350: signal-velocity viscosity without the Balsara switch."""
    ctx = _ctx(int(pos.shape[0]))
    _physics(ctx, "gadget", False, alpha, beta, eta, gama)
    return _sph_pass(nbeg, nend, pos, v, rho, P, c, h, m, None, None, "acc")


def get_dU_mpiXXXX(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """libsx.py:429-497 (Monaghan & Gingold)."""
    ctx = _ctx(int(pos.shape[0]))
    _physics(ctx, "mg83", False, alpha, beta, eta, gama)
    return _sph_pass(nbeg, nend, pos, v, rho, P, c, h, m, None, None, "du")


def get_dU(pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """libsx.py:355-424 (Monaghan & Gingold, all rows)."""
    return get_dU_mpiXXXX(0, pos.shape[0], pos, v, rho, P, c, h, m, gama, eta, alpha, beta)


def get_dU_mpi(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """libsx.py:498-566 (signal velocity, no Balsara switch)."""
    ctx = _ctx(int(pos.shape[0]))
    _physics(ctx, "gadget", False, alpha, beta, eta, gama)
    return _sph_pass(nbeg, nend, pos, v, rho, P, c, h, m, None, None, "du")


# ---- gravity -------------------------------------------------------------
def getAcc_g_smth_mimj_mpi(nbeg, nend, pos, mass, G, epsilon):
    """libsx.py:910-947: spline-softened direct sum with eps_ij = (eps_i +
    eps_j)/2 as an (N, 3) field (FP64 on the GPU).  For rows [nbeg, nend) it
    is the reference's partial field: each pair (i, j), i < j, with i in the
    rows adds to both i and j, so the fields of the MPI ranks' row ranges sum
    to the full field."""
    n = int(pos.shape[0])
    if not 0 <= nbeg <= nend <= n:
        raise ValueError("rows [nbeg, nend) must lie in [0, N)")
    ctx = _ctx(n)
    ctx.set_params(G=float(G))
    ones = np.ones(n) if not _is_cuda_tensor(pos) else _zeros_like_dev(n) + 1.0
    ctx = _load_state(pos, mass, ones)
    eps = _host(epsilon)
    if (nbeg, nend) == (0, n):
        inv = np.empty(n, np.int32)
        inv[ctx.ids()] = np.arange(n, dtype=np.int32)  # storage slot of each particle
        acc = ctx.gravity_direct_spline(eps, inv)
    else:
        acc = ctx.gravity_direct_spline_rows(eps, nbeg, nend)
    if _is_cuda_tensor(pos):
        import torch
        return torch.from_numpy(acc).to(pos.device)
    return acc


def getPE(pos, m, G, epsilon):
    """Total potential energy.  libsx.py:585-620 sums the spline-softened pair
    potential; here the Plummer potential of the quadrupole tree walk with
    eps = mean(epsilon), summed in FP64 on the GPU (sph_energies)."""
    n = int(pos.shape[0])
    ctx = _ctx(n)
    ones = np.ones(n) if not _is_cuda_tensor(pos) else _zeros_like_dev(n) + 1.0
    ctx.set_params(G=float(G), eps=float(np.mean(_host(epsilon))),
                   flags=ctx.config.flags | L.FLAG_POTENTIAL)
    try:
        ctx = _load_state(pos, m, ones)
        ctx.gravity()
        return ctx.energies()["PE"]
    finally:
        ctx.set_params(flags=ctx.config.flags & ~L.FLAG_POTENTIAL)


def _host(a):
    return np.ascontiguousarray(a.detach().cpu().numpy() if _is_cuda_tensor(a) else a,
                                dtype=np.float64)


# ---- smoothing lengths ---------------------------------------------------
def h_smooth_fast_mpi(nbeg, nend, pos, h, max_iter=10000):
    """libsx.py:854-902: from h, h <- h - 0.003 h while more than 55
    particles (self included) lie within |r_ij| < 2h and h <- h + 0.003 h
    while fewer than 45 do; rows nbeg..nend-1.  Bit-exact with the reference.
    The reference keeps iterating without bound (it prints after 100
    iterations); a row still outside the window after max_iter iterations
    raises SphError (SPH_ERR_NOCONV) here."""
    n = int(pos.shape[0])
    mm = np.full(n, 1.0 / n) if not _is_cuda_tensor(pos) else _zeros_like_dev(n) + 1.0 / n
    ctx = _load_state(pos, mm, h)
    ctx.smoothing_h_count(50, 5, 0.003, max_iter)
    st = ctx.status(reset=True)
    if st["h_noconv"]:
        raise L.SphError(-4, "h_smooth_fast_mpi", f"({st['h_noconv']} rows did not converge)")
    return _rows(_out(ctx, "h", pos), nbeg, nend)


def h_smooth_fast(pos, h, max_iter=10000):
    """libsx.py:806-850 (all rows)."""
    return h_smooth_fast_mpi(0, pos.shape[0], pos, h, max_iter)


def h_newton_mpi(nbeg, nend, pos, h, m=None, n_ngb=50.0):
    """The project's smoothing length (no reference counterpart): the
    bracketed Newton solution of (4 pi / 3)(2h)^3 rho(h) = n_ngb m, started
    from h; rows nbeg..nend-1."""
    n = int(pos.shape[0])
    mm = (np.full(n, 1.0 / n) if not _is_cuda_tensor(pos) else _zeros_like_dev(n) + 1.0 / n) \
        if m is None else m
    ctx = _ctx(n)
    ctx.set_params(n_ngb=float(n_ngb))
    ctx = _load_state(pos, mm, h)
    ctx.smoothing_h()
    st = ctx.status(reset=True)
    if st["h_noconv"]:
        raise L.SphError(-4, "h_newton_mpi", f"({st['h_noconv']} rows did not converge)")
    return _rows(_out(ctx, "h", pos), nbeg, nend)


def smoothing_length_mpi(nbeg, nend, pos):
    """libsx.py:777-800: half the distance to the 50th neighbour (the sorted
    distances' entry 50, the particle itself at entry 0), rows nbeg..nend-1,
    bit-exact with the reference."""
    n = int(pos.shape[0])
    p = _host(pos)
    ext = np.ptp(p, axis=0).prod() if n > 1 else 1.0
    h0 = 0.5 * (max(ext, 1e-300) * 50.0 / max(n, 1)) ** (1.0 / 3.0)   # search start
    h = np.full(n, h0) if not _is_cuda_tensor(pos) else _zeros_like_dev(n) + h0
    mm = np.full(n, 1.0 / n) if not _is_cuda_tensor(pos) else _zeros_like_dev(n) + 1.0 / n
    ctx = _load_state(pos, mm, h)
    ctx.smoothing_length_kth(50)
    st = ctx.status(reset=True)
    if st["h_noconv"]:
        raise L.SphError(-4, "smoothing_length_mpi", f"({st['h_noconv']} rows did not converge)")
    return _rows(_out(ctx, "h", pos), nbeg, nend)


# ---- elementwise formulas and energies -----------------------------------
def getPressure(rho, u, gama):
    """libsx.py:92-96: P = (gamma - 1) rho u."""
    return (gama - 1.0) * rho * u


def getCsound(u, gama):
    """c = sqrt(gamma (gamma - 1) u) (hfvCLibs_v7_hfv_v2.h:589-612)."""
    return (gama * (gama - 1.0) * u) ** 0.5


def getKE(v, m):
    """libsx.py:571-580: sum 0.5 m |v|^2."""
    v, m = _host(v), _host(m)
    return float(0.5 * np.sum(m * np.sum(v * v, axis=1)))
