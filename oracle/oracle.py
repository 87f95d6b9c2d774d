"""CPU oracle -- test infrastructure only.

ctypes wrapper over ``oracle/liboracle.so`` (built from ``sph_oracle.c`` by
``oracle/Makefile``) plus a NumPy restatement of the cooling-surrogate MLP.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference
arm of ``bench.py`` import this module; the product package never does.

Every function cites the reference code it restates (paths relative to the
reference's ``11_Dec_2022/`` directory) or says that it pins a project-defined
method that has no reference counterpart.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
vp = C.c_void_p


def reference_root() -> str:
    """The reference's 11_Dec_2022 directory: $SPH2_REFERENCE, else its
    location in the build container."""
    return os.environ.get("SPH2_REFERENCE", "/root/reference/11_Dec_2022")


def build() -> str:
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    ref = reference_root()
    if os.path.isdir(ref):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"SPH2_REFERENCE={ref}"], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        I, D = C.c_int, C.c_double
        sig = {
            "ref_density": [I, f64p, f64p, f64p, I, I, f64p],
            "ref_div_curl": [I, f64p, f64p, f64p, f64p, f64p, I, I, f64p, f64p],
            "ref_acc_sph": [I, f64p, f64p, f64p, f64p, f64p, f64p, f64p, f64p, f64p, D, D, D, I, I, I, I, f64p],
            "ref_dudt": [I, f64p, f64p, f64p, f64p, f64p, f64p, f64p, f64p, f64p, D, D, D, I, I, I, I, f64p],
            "ref_acc_g_smth": [I, f64p, f64p, D, f64p, I, I, f64p],
            "ref_h_smooth_fast": [I, f64p, f64p, I, I, I, f64p],
            "ref_smoothing_length": [I, f64p, I, I, f64p],
            "orc_cloud_boxes": [I, i32p, f64p, f64p, f64p, f64p],
            "orc_morton_keys": [I, f64p, f64p, f64p, i32p, f64p, I, u64p],
            "orc_neighbours": [I, f64p, f64p, f64p, f64p, vp, vp, vp, vp],
            "orc_newton_h": [I, f64p, f64p, f64p, f64p, vp, f64p, D, D, I, f64p, vp],
            "orc_density_list": [I, f64p, f64p, f64p, f64p, f64p, i64p, i32p, f64p],
            "orc_divcurl_list": [I, f64p, f64p, f64p, f64p, f64p, f64p, f64p, f64p, f64p, i64p, i32p, f64p, f64p],
            "orc_force_list": [I] + [f64p] * 13 + [D, D, D, I, I, i64p, i32p, vp, vp, vp, vp, vp],
            "orc_grav_direct": [I, f64p, f64p, f64p, f64p, vp, D, D, I, i32p, f64p, f64p, f64p, vp],
            "orc_dt_individual": [I] + [f64p] * 12 + [D, D, D, i64p, i32p, f64p, f64p],
            "orc_outflow_pairs": [C.c_uint64, I, D, D] + [f64p] * 6,
            "orc_isothermal": [I, f64p, f64p, f64p, D, f64p, f64p, f64p],
            "orc_cool_table": [i32p, f32p, f32p, f32p, I, I] + [f64p] * 6 + [D] * 7 + [f64p, f32p],
            "orc_build_radix_tree": [I, u64p, i32p, i32p, i32p, i32p],
            "orc_tree_moments": [I, i32p, i32p, i32p, C.c_void_p, f64p, f64p, f64p, f64p, f64p,
                                 f64p, f64p],
            "orc_open_r2": [I, f64p, D, f64p],
            "orc_walk": [I, f64p, f64p, f64p, f64p, i32p, i32p, i32p, f64p, f64p, I, i32p, i32p, i32p,
                         I, D, D, f64p, f64p, f64p, vp, vp, vp],
            "orc_do_cooling_batch": [f64p, I, D, D, D, D, D, D, I, f64p, f64p, f64p, D, I, f64p, vp],
            "orc_num_threads": [],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
        L.ref_h_smooth_fast.restype = I
        L.orc_newton_h.restype = I
        L.orc_num_threads.restype = I
        L.ref_ke.argtypes = [I, f64p, f64p]
        L.ref_ke.restype = D
        L.ref_pe.argtypes = [I, f64p, f64p, D, f64p]
        L.ref_pe.restype = D
        _LIB = L
    return _LIB


def _c(a, dt=np.float64):
    return np.ascontiguousarray(a, dtype=dt)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def num_threads() -> int:
    return lib().orc_num_threads()


# --------------------------------------------------------------------------
# (A) the reference CPU step, restated (MPI_sph/sph_code/libsx.py, shear.py)
# --------------------------------------------------------------------------
def ref_getDensity(nbeg, nend, pos, m, h):
    """getDensity_mpi, MPI_sph/sph_code/libsx.py:52-86."""
    pos, m, h = _c(pos), _c(m), _c(h)
    out = np.zeros(nend - nbeg)
    lib().ref_density(len(m), pos, m, h, nbeg, nend, out)
    return out


def ref_div_curlVel(nbeg, nend, pos, v, rho, m, h):
    """div_curlVel_mpi, MPI_sph/sph_code/shear.py:78-142."""
    d = np.zeros(nend - nbeg)
    c = np.zeros(nend - nbeg)
    lib().ref_div_curl(len(m), _c(pos), _c(v), _c(rho), _c(m), _c(h), nbeg, nend, d, c)
    return d, c


def ref_getAcc_sph(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, alpha, beta=2.0, eta=0.1,
                   mode=1, balsara=1):
    """mode=1,balsara=1: getAcc_sph_shear_mpi (shear.py:243-330);
    mode=0,balsara=0: getAcc_sph_mpiXXX (libsx.py:185-262, Monaghan-Gingold)."""
    out = np.zeros((nend - nbeg) * 3)
    lib().ref_acc_sph(len(m), _c(pos), _c(v), _c(rho), _c(P), _c(c), _c(h), _c(m), _c(divV),
                      _c(curlV), alpha, beta, eta, mode, balsara, nbeg, nend, out)
    return out.reshape(-1, 3)


def ref_get_dU(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, alpha, beta=2.0, eta=0.1,
               mode=1, balsara=1):
    """get_dU_shear_mpi (shear.py:413-485) / get_dU_mpiXXXX (libsx.py:427-497)."""
    out = np.zeros(nend - nbeg)
    lib().ref_dudt(len(m), _c(pos), _c(v), _c(rho), _c(P), _c(c), _c(h), _c(m), _c(divV),
                   _c(curlV), alpha, beta, eta, mode, balsara, nbeg, nend, out)
    return out


def ref_getAcc_g_smth_mimj(nbeg, nend, pos, mass, G, epsilon):
    """getAcc_g_smth_mimj_mpi, libsx.py:910-947 (partial N x 3 field)."""
    out = np.zeros(len(mass) * 3)
    lib().ref_acc_g_smth(len(mass), _c(pos), _c(mass), G, _c(epsilon), nbeg, nend, out)
    return out.reshape(-1, 3)


def ref_h_smooth_fast(nbeg, nend, pos, h, max_iter=10000):
    """h_smooth_fast_mpi, libsx.py:854-902."""
    out = np.zeros(nend - nbeg)
    lib().ref_h_smooth_fast(len(h), _c(pos), _c(h), nbeg, nend, max_iter, out)
    return out


def ref_smoothing_length(nbeg, nend, pos):
    """smoothing_length_mpi, libsx.py:781-802."""
    out = np.zeros(nend - nbeg)
    pos = _c(pos)
    lib().ref_smoothing_length(pos.shape[0], pos, nbeg, nend, out)
    return out


def ref_getKE(v, m):
    """getKE, libsx.py:571-580."""
    return lib().ref_ke(len(m), _c(v), _c(m))


def ref_getPE(pos, m, G, epsilon):
    """getPE, libsx.py:585-620."""
    return lib().ref_pe(len(m), _c(pos), _c(m), G, _c(epsilon))


def ref_pressure(rho, u, gama):
    """getPressure, libsx.py:92-96."""
    return (gama - 1.0) * rho * u


def ref_sound_speed(u, gama):
    """c = sqrt(gamma (gamma-1) u), sph_mpi4_v4.py:349."""
    return np.sqrt(gama * (gama - 1.0) * u)


# --------------------------------------------------------------------------
# (B) the project method
# --------------------------------------------------------------------------
def cloud_starts(cloud):
    """Start index of each cloud's contiguous range (ids 0..K-1 ascending)."""
    cloud = np.asarray(cloud)
    k = int(cloud.max()) + 1 if len(cloud) else 0
    counts = np.bincount(cloud, minlength=k)
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)


def morton_bits(ncloud: int) -> int:
    """Bits per axis when the cloud id takes the top bits of a 63-bit key."""
    cb = 0
    while (1 << cb) < ncloud:
        cb += 1
    return (63 - cb) // 3


def cloud_boxes(x, y, z, cloud_start):
    k = len(cloud_start) - 1
    box = np.zeros(6 * k)
    lib().orc_cloud_boxes(k, _c(cloud_start, np.int32), _c(x), _c(y), _c(z), box)
    return box.reshape(k, 6)


def morton_keys(x, y, z, cloud=None, bits=None):
    """63-bit keys (cloud id in the top bits).  No reference counterpart:
    the reference bins into a 10^3 grid (Particles_in_BH_Tree_II/Evrard_test/
    ngb_v3.h:58-117); the key definition is the project's."""
    n = len(x)
    if cloud is None:
        cloud = np.zeros(n, np.int32)
    cloud = _c(cloud, np.int32)
    # boxes are computed over each cloud's members, wherever they are stored
    k = int(cloud.max()) + 1 if n else 1
    box = np.zeros((k, 6))
    for c in range(k):
        sel = cloud == c
        if sel.any():
            box[c, :3] = [x[sel].min(), y[sel].min(), z[sel].min()]
            box[c, 3:] = [x[sel].max(), y[sel].max(), z[sel].max()]
    if bits is None:
        bits = morton_bits(k)
    keys = np.zeros(n, np.uint64)
    lib().orc_morton_keys(n, _c(x), _c(y), _c(z), cloud, _c(box.ravel()), bits, keys)
    return keys


def sort_perm(keys):
    """Stable sort of the current storage order by key."""
    return np.argsort(keys, kind="stable").astype(np.int32)


def neighbours(x, y, z, h, cloud=None):
    """Exact lists: j in L(i) iff |r_ij|^2 <= (h_i+h_j)^2 (FP64, rounding as
    written), i.e. q = r/h_ij <= 2 with h_ij = (h_i+h_j)/2 -- the support of
    the reference kernels (libsx.py:69-80).  Returns CSR (offsets, lists)
    with each row sorted ascending."""
    n = len(x)
    x, y, z, h = _c(x), _c(y), _c(z), _c(h)
    cl = None if cloud is None else _c(cloud, np.int32)
    counts = np.zeros(n, np.int32)
    lib().orc_neighbours(n, x, y, z, h, _ptr(cl), _ptr(counts), None, None)
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum(counts)
    lst = np.zeros(max(int(off[-1]), 1), np.int32)
    lib().orc_neighbours(n, x, y, z, h, _ptr(cl), None, _ptr(off), _ptr(lst))
    return off, lst[: off[-1]]


def newton_h(x, y, z, m, h0, n_ngb=64.0, tol=1e-3, max_iter=64, cloud=None):
    """Newton iteration on (4pi/3)(2h)^3 rho(h) = n_ngb m (project method,
    replaces h_smooth_fast_mpi, libsx.py:854-902)."""
    n = len(x)
    out = np.zeros(n)
    it = np.zeros(n, np.int32)
    cl = None if cloud is None else _c(cloud, np.int32)
    bad = lib().orc_newton_h(n, _c(x), _c(y), _c(z), _c(m), _ptr(cl), _c(h0), n_ngb, tol,
                             max_iter, out, _ptr(it))
    return out, it, bad


def density_list(x, y, z, m, h, off, lst):
    out = np.zeros(len(x))
    lib().orc_density_list(len(x), _c(x), _c(y), _c(z), _c(m), _c(h), _c(off, np.int64),
                           _c(lst, np.int32), out)
    return out


def divcurl_list(x, y, z, vx, vy, vz, rho, m, h, off, lst):
    n = len(x)
    d, c = np.zeros(n), np.zeros(n)
    lib().orc_divcurl_list(n, _c(x), _c(y), _c(z), _c(vx), _c(vy), _c(vz), _c(rho), _c(m),
                           _c(h), _c(off, np.int64), _c(lst, np.int32), d, c)
    return d, c


def force_list(x, y, z, vx, vy, vz, rho, P, c, h, m, divV, curlV, alpha, beta, eta, mode,
               balsara, off, lst):
    n = len(x)
    ax, ay, az, du, vs = (np.zeros(n) for _ in range(5))
    lib().orc_force_list(n, _c(x), _c(y), _c(z), _c(vx), _c(vy), _c(vz), _c(rho), _c(P), _c(c),
                         _c(h), _c(m), _c(divV), _c(curlV), alpha, beta, eta, mode, balsara,
                         _c(off, np.int64), _c(lst, np.int32), _ptr(ax), _ptr(ay), _ptr(az),
                         _ptr(du), _ptr(vs))
    return np.stack([ax, ay, az], 1), du, vs


def courant_dt(h, vsig, acc, courant, cloud=None):
    """Courant step per cloud of the project's global step (the survey's
    replacement of dt_array_indiv_dt, hfvCLibs_v7_hfv_v2.h:999-1078):
    dt_c = courant * min over the cloud's particles of min(h / v_sig,
    sqrt(h / |a|)), a = a_sph + a_grav; particles without a finite positive
    estimate are skipped."""
    h, vsig = np.asarray(h, float), np.asarray(vsig, float)
    amag = np.sqrt(np.sum(np.asarray(acc, float) ** 2, axis=1))
    t = h / np.maximum(vsig, 1e-300)
    with np.errstate(divide="ignore", invalid="ignore"):
        ta = np.where(amag > 0, np.sqrt(h / np.where(amag > 0, amag, 1.0)), np.inf)
    t = courant * np.minimum(t, ta)
    ok = np.isfinite(t) & (t > 0)
    cl = np.zeros(len(h), np.int64) if cloud is None else np.asarray(cloud, np.int64)
    out = np.full(int(cl.max()) + 1 if len(cl) else 1, np.inf)
    np.minimum.at(out, cl[ok], t[ok])
    return out


def dt_individual(x, y, z, vx, vy, vz, m, h, rho, c, asph, agrav, eps, courant, alpha, off,
                  lst):
    """Per-particle steps and dh/dt of dt_array_indiv_dt
    (hfvCLibs_v7_hfv_v2.h:999-1078) over the neighbour lists (see
    orc_dt_individual).  asph, agrav: (n, 3)."""
    n = len(x)
    dt, dh = np.zeros(n), np.zeros(n)
    a_s = _c(np.asarray(asph, float).T.reshape(-1))
    a_g = _c(np.asarray(agrav, float).T.reshape(-1))
    lib().orc_dt_individual(n, _c(x), _c(y), _c(z), _c(vx), _c(vy), _c(vz), _c(m), _c(h),
                            _c(rho), _c(c), a_s, a_g, eps, courant, alpha,
                            _c(off, np.int64), _c(lst, np.int32), dt, dh)
    return dt, dh


def outflow_pairs(seed, npairs, r_max, v_in):
    """Positions and velocities (2 npairs rows) of the outflow pairs
    (orc_outflow_pairs; outflow_injector2, hfvCLibs_v7_hfv_v2.h:1094-1210)."""
    out = [np.zeros(2 * npairs) for _ in range(6)]
    lib().orc_outflow_pairs(int(seed), int(npairs), float(r_max), float(v_in), *out)
    return np.stack(out[:3], 1), np.stack(out[3:], 1)


def isothermal_acc(x, y, z, sigma):
    """galaxy_isothermal_potential (hfvCLibs_v7_hfv_v2.h:1215-1235)."""
    n = len(x)
    a = [np.zeros(n) for _ in range(3)]
    lib().orc_isothermal(n, _c(x), _c(y), _c(z), float(sigma), *a)
    return np.stack(a, 1)


def cool_table(tab, x, y, z, rho, u, dt, unit_rho=1.0, unit_u=1.0, unit_t=1.0, unit_len=1.0,
               kpc_cm=3.086e21, XH=0.70, mH=1.6726e-24, z_row=1):
    """hcoolingx (hfvCLibs_v7_hfv_v2.h:1240-1418) on a grid dict of
    sph_2_b200.cooling.read_table_file: (u_new, ion fractions [n, N_M])."""
    nk, nt, nh, nz, ntime = tab["u_evol"].shape
    nm = tab["frac"].shape[4]
    dims = np.array([nk, nh, nz, nt, nm, ntime], np.int32)
    grid = np.concatenate([tab[k] for k in ("kpc", "nH", "Z", "T", "time_s")]).astype(np.float32)
    n = len(x)
    un = np.zeros(n)
    ion = np.zeros(n * nm, np.float32)
    lib().orc_cool_table(dims, grid, _c(tab["u_evol"], np.float32).reshape(-1),
                         _c(tab["frac"], np.float32).reshape(-1), int(z_row), n, _c(x), _c(y),
                         _c(z), _c(rho), _c(u), _c(np.broadcast_to(dt, (n,))), unit_rho, unit_u,
                         unit_t, unit_len, kpc_cm, XH, mH, un, ion)
    return un, ion.reshape(n, nm)


def grav_direct(x, y, z, m, G, eps, targets, cloud=None):
    """FP64 Plummer direct sum onto the target indices (all sources of the
    target's cloud).  The reference's direct sums (libsx.py:910-947,
    hfvCLibs_v7_hfv_v2.h:532-584) use spline softening; Plummer eps is the
    project's choice."""
    t = _c(targets, np.int32)
    ax, ay, az, pot = (np.zeros(len(t)) for _ in range(4))
    cl = None if cloud is None else _c(cloud, np.int32)
    lib().orc_grav_direct(len(x), _c(x), _c(y), _c(z), _c(m), _ptr(cl), G, eps, len(t), t, ax, ay,
                          az, _ptr(pot))
    return np.stack([ax, ay, az], 1), pot


def build_radix_tree(keys):
    """Karras (2012) radix tree over sorted keys (no reference counterpart:
    the reference inserts bodies into an octree under locks,
    Particles_in_BH_Tree_II/Evrard_test/bh_tree_iteration_v2.h:149-367)."""
    n = len(keys)
    nn = 2 * n - 1
    child = np.zeros(2 * nn, np.int32)
    parent = np.zeros(nn, np.int32)
    first = np.zeros(nn, np.int32)
    last = np.zeros(nn, np.int32)
    lib().orc_build_radix_tree(n, _c(keys, np.uint64), child, parent, first, last)
    return child, parent, first, last


def tree_moments(child, first, last, x, y, z, m, h, cloud=None):
    """FP64 node records: nodes of at most 32 particles of one cloud (inside
    a walk group) summed directly over their particle range, larger ones
    combined from their children, left first (project method; the reference
    octree accumulates masses with atomics, bh_tree_iteration_v2.h:149-367)."""
    n = len(x)
    nn = 2 * n - 1
    node = np.zeros(16 * nn)
    hmax = np.zeros(nn)
    cl = None if cloud is None else _c(cloud, np.int32)
    lib().orc_tree_moments(n, _c(child, np.int32), _c(first, np.int32), _c(last, np.int32),
                           None if cl is None else cl.ctypes.data_as(C.c_void_p), _c(x), _c(y),
                           _c(z), _c(m), _c(h), node, hmax)
    return node.reshape(nn, 16), hmax


def open_r2(node, theta):
    nn = node.shape[0]
    out = np.zeros(nn)
    lib().orc_open_r2(nn, _c(node.ravel()), theta, out)
    return out


def tree_groups(first, last, parent, cloud, gmax=32):
    """Walk/search groups: maximal tree nodes with at most gmax particles of
    one cloud, ordered by their first particle (project definition; the
    reference walks one particle per thread, bh_tree_iteration_v2.h:454)."""
    first, last, parent = np.asarray(first), np.asarray(last), np.asarray(parent)
    cloud = np.asarray(cloud)
    cnt = last - first + 1
    ok = (cnt <= gmax) & (cloud[first] == cloud[last])
    pp = np.where(parent < 0, 0, parent)
    top = ok & ((parent < 0) | ~ok[pp])
    idx = np.nonzero(top)[0]
    order = np.argsort(first[idx], kind="stable")
    idx = idx[order]
    return (first[idx].astype(np.int32), cnt[idx].astype(np.int32),
            cloud[first[idx]].astype(np.int32))


def cloud_roots(first, last, cloud_start, n):
    """Tree node whose particle range is exactly each cloud's range."""
    roots = []
    lut = {}
    for nd in range(len(first)):
        lut.setdefault((int(first[nd]), int(last[nd])), nd)
    for k in range(len(cloud_start) - 1):
        a, b = int(cloud_start[k]), int(cloud_start[k + 1]) - 1
        if a == b:
            roots.append(n - 1 + a)
        else:
            roots.append(lut[(a, b)])
    return np.array(roots, np.int32)


def bh_walk(x, y, z, m, h, keys_sorted, theta, eps, G=1.0, leaf_size=16, group_size=32,
            cloud_start=None, want_pot=False):
    """Group Barnes-Hut walk with monopole+quadrupole nodes (project method;
    the reference walk is monopole-only, bh_tree_iteration_v2.h:454-588)."""
    n = len(x)
    if cloud_start is None:
        cloud_start = np.array([0, n], np.int32)
    child, parent, first, last = build_radix_tree(keys_sorted)
    cloud = np.repeat(np.arange(len(cloud_start) - 1), np.diff(cloud_start))
    node, hmax = tree_moments(child, first, last, x, y, z, m, h, cloud)
    r2 = open_r2(node, theta)
    gs, gc, gk = tree_groups(first, last, parent, cloud, group_size)
    roots = cloud_roots(first, last, cloud_start, n)
    groot = roots[gk].astype(np.int32)
    ax, ay, az = np.zeros(n), np.zeros(n), np.zeros(n)
    pot = np.zeros(n) if want_pot else None
    nc = np.zeros(n, np.int64)
    npart = np.zeros(n, np.int64)
    lib().orc_walk(n, _c(x), _c(y), _c(z), _c(m), child, first, last, _c(node.ravel()), r2,
                   len(gs), gs, gc, groot, leaf_size, G, eps, ax, ay, az, _ptr(pot), _ptr(nc),
                   _ptr(npart))
    return np.stack([ax, ay, az], 1), pot, nc, npart


def do_cooling(logL, logT0, logT1, mu, gamma, XH, gamma_heat, rho, u_old, dt, tol=1e-6,
               max_iter=200):
    """Implicit cooling solve with the bracket-and-bisect structure of
    GPU_sph/With_cooling/Model_C/myPhotoLibsGPU.h:615-686, FP64, over the
    synthetic power-law cooling table."""
    logL = _c(logL)
    rho, u_old, dt = _c(rho), _c(u_old), _c(np.broadcast_to(dt, np.shape(rho)))
    out = np.zeros(len(rho))
    it = np.zeros(len(rho), np.int32)
    lib().orc_do_cooling_batch(logL, len(logL) - 1, logT0, logT1, mu, gamma, XH, gamma_heat,
                               len(rho), rho, u_old, dt, tol, max_iter, out, _ptr(it))
    return out, it


# ---- FP32 bisection pinned against the reference's compiled DoCooling ----
def ref_cooling_lib():
    """oracle/_ref/libphcool.so (the reference's myPhotoLibsGPU.h built on the
    host), or None when it has not been built."""
    p = os.path.join(_HERE, "_ref", "libphcool.so")
    if not os.path.exists(p):
        return None
    L = C.CDLL(p)
    F = C.c_float
    L.ref_DoCooling.argtypes = [F, F, F, F]
    L.ref_DoCooling.restype = F
    L.ref_coolingRateFromU.argtypes = [F, F, F]
    L.ref_coolingRateFromU.restype = F
    return L


def do_cooling_f32_with_ref_rate(rho, u_old, dt, XH):
    """FP32 restatement of DoCooling (myPhotoLibsGPU.h:615-686) driven by the
    reference's own coolingRateFromU."""
    R = ref_cooling_lib()
    if R is None:
        raise FileNotFoundError("oracle/_ref/libphcool.so not built")
    L = lib()
    F = C.c_float
    RATE = C.CFUNCTYPE(F, F, F, F)
    L.orc_do_cooling_f32.argtypes = [RATE, F, F, F, F]
    L.orc_do_cooling_f32.restype = F
    cb = RATE(("ref_coolingRateFromU", R))
    return L.orc_do_cooling_f32(cb, rho, u_old, dt, XH)


# --------------------------------------------------------------------------
# MLP cooling surrogate (no reference counterpart): NumPy FP32 restatement
# of the forward and backward passes the GPU kernels implement.
# --------------------------------------------------------------------------
def gelu_tanh(x):
    k = np.float32(0.7978845608028654)
    return 0.5 * x * (1.0 + np.tanh(k * (x + np.float32(0.044715) * x ** 3)))


def gelu_tanh_grad(x):
    k = 0.7978845608028654
    t = np.tanh(k * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * k * (1.0 + 3 * 0.044715 * x * x)


def mlp_forward(X, W1, b1, W2, b2, W3, b3):
    """X [B,3] (normalised inputs); W1 [3,64], W2 [64,64], W3 [64,1]."""
    z1 = X @ W1 + b1
    a1 = gelu_tanh(z1)
    z2 = a1 @ W2 + b2
    a2 = gelu_tanh(z2)
    y = a2 @ W3 + b3
    return y[:, 0], (X, z1, a1, z2, a2)


def mlp_backward(cache, dy, W2, W3):
    """Gradients of sum(dy * y) w.r.t. all parameters."""
    X, z1, a1, z2, a2 = cache
    dy = dy[:, None]
    gW3 = a2.T @ dy
    gb3 = dy.sum(0)
    da2 = dy @ W3.T
    dz2 = da2 * gelu_tanh_grad(z2)
    gW2 = a1.T @ dz2
    gb2 = dz2.sum(0)
    da1 = dz2 @ W2.T
    dz1 = da1 * gelu_tanh_grad(z1)
    gW1 = X.T @ dz1
    gb1 = dz1.sum(0)
    return gW1, gb1, gW2, gb2, gW3, gb3


def bf16(x):
    """Round float32 to bfloat16 (nearest even), returned as float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b >> 16) & 1) + 0x7FFF
    return ((b + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def mlp_forward_bf16(X, W1, b1, W2, b2, W3, b3):
    """Forward with the rounding points of the tensor-core kernels: matmul
    operands in BF16, accumulation, bias, GELU and the last layer in FP32."""
    z1 = bf16(X) @ bf16(W1) + b1
    a1 = gelu_tanh(z1).astype(np.float32)
    z2 = bf16(a1) @ bf16(W2) + b2
    a2 = gelu_tanh(z2).astype(np.float32)
    y = a2 @ W3 + b3
    return y[:, 0], (X, z1, a1, z2, a2)


def mlp_grad_bf16(X, t, W1, b1, W2, b2, W3, b3):
    """Gradient of 0.5*mean((y-t)^2) with the kernels' rounding points."""
    y, (X, z1, a1, z2, a2) = mlp_forward_bf16(X, W1, b1, W2, b2, W3, b3)
    n = len(t)
    dy = ((y - t) / n).astype(np.float32)[:, None]
    loss = 0.5 * np.mean((y - t) ** 2)
    gW3 = a2.T @ dy
    gb3 = dy.sum(0)
    dz2 = (dy @ W3.T) * gelu_tanh_grad(z2)
    gb2 = dz2.sum(0)
    gW2 = bf16(a1).T @ bf16(dz2)
    da1 = bf16(dz2) @ bf16(W2).T
    dz1 = da1 * gelu_tanh_grad(z1)
    gb1 = dz1.sum(0)
    gW1 = bf16(X).T @ bf16(dz1)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3]).astype(np.float32)
    return g, float(loss)

