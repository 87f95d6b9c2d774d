"""Host side of the B200 SPH step: a thin owner of one libsphb200 context.

The methods keep the reference's step-level vocabulary (smoothing length,
density, div/curl, SPH acceleration, du/dt, gravity, kick/drift; see
MPI_sph/sph_code/sph_mpi4_v4.py:278-442 for the reference's loop) and move
NumPy arrays in and out in the caller's original particle order.  All compute
runs in the CUDA library; nothing here computes physics.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import asdict, dataclass, field, fields

import numpy as np

from . import _lib as L


@dataclass
class Config:
    """Mirror of ``sph_config`` (include/sph_b200.h); defaults follow the
    Evrard workload: N_ngb = 64, Monaghan-Gingold viscosity alpha = 1,
    beta = 2, eta = 0.1 (sph_mpi4_v4.py:22-26), Plummer eps = 1e-2,
    theta = 0.5, Courant 0.25, gamma = 5/3, G = 1."""
    n_max: int = 1 << 20
    n_cloud_max: int = 1
    precision: str = "mixed"
    av_mode: str = "mg83"
    balsara: bool = False
    leaf_size: int = 8
    ngb_lanes: int = 4
    block_size: int = 128
    max_ngb: int = 256
    h_max_iter: int = 64
    flags: int = 0
    walk_blocks: int = 0
    n_ngb: float = 64.0
    h_tol: float = 1e-3
    gamma: float = 5.0 / 3.0
    alpha: float = 1.0
    beta: float = 2.0
    eta: float = 0.1
    G: float = 1.0
    eps: float = 1e-2
    theta: float = 0.5
    courant: float = 0.25
    dt_max: float = 0.0
    dt_fixed: float = 0.0
    theta_local: float = 0.0
    theta_small: float = 0.0
    small_cell: int = 0
    dt_mode: str = "courant"
    ext_sigma: float = 0.0
    rebuild_every: int = 1

    def to_c(self) -> L.SphConfig:
        c = L.SphConfig()
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "precision":
                v = L.PREC[v]
            elif f.name == "av_mode":
                v = L.AV[v]
            elif f.name == "dt_mode":
                v = L.DT_MODE[v]
            elif f.name == "balsara":
                v = int(bool(v))
            setattr(c, f.name, v)
        return c


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def ic_count(path) -> int:
    """Particle count of a reference IC file, its size checked (no GPU)."""
    n = C.c_int32(0)
    L.check(L.load().sph_ic_count(str(path).encode(), C.byref(n)), "sph_ic_count")
    return int(n.value)


class Context:
    """One device context (capacity n_max particles, n_cloud_max clouds)."""

    def __init__(self, config: Config | None = None, **kw):
        self.config = config or Config(**kw)
        self._L = L.load()
        self._h = C.c_void_p()
        cfg = self.config.to_c()
        L.check(self._L.sph_ctx_create(C.byref(cfg), C.byref(self._h)), "sph_ctx_create")

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self._h:
            self._L.sph_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, rc, where):
        return L.check(rc, where, self._h)

    @property
    def handle(self):
        return self._h

    @property
    def n(self) -> int:
        return self._L.sph_count(self._h)

    @property
    def n_clouds(self) -> int:
        return self._L.sph_cloud_count(self._h)

    def device_bytes(self) -> int:
        return int(self._L.sph_device_bytes(self._h))

    def set_params(self, **kw):
        for k, v in kw.items():
            setattr(self.config, k, v)
        cfg = self.config.to_c()
        self._chk(self._L.sph_set_params(self._h, C.byref(cfg)), "sph_set_params")

    # -- data ---------------------------------------------------------------
    def load(self, pos, vel=None, m=None, h=None, u=None, cloud=None):
        pos = _f64(pos)
        n = pos.shape[0]
        x, y, z = (_f64(pos[:, k]) for k in range(3))
        vel = np.zeros((n, 3)) if vel is None else _f64(vel)
        vx, vy, vz = (_f64(vel[:, k]) for k in range(3))
        m = _f64(np.full(n, 1.0 / max(n, 1)) if m is None else m)
        h = _f64(np.full(n, 0.05) if h is None else h)
        u = _f64(np.zeros(n) if u is None else u)
        cl = None if cloud is None else np.ascontiguousarray(cloud, dtype=np.int32)
        self._keep = (x, y, z, vx, vy, vz, m, h, u, cl)
        self._chk(self._L.sph_load(self._h, n, _ptr(cl), _ptr(x), _ptr(y), _ptr(z), _ptr(vx),
                                   _ptr(vy), _ptr(vz), _ptr(m), _ptr(h), _ptr(u), 1), "sph_load")

    def load_ic(self, path, want_eps=False):
        """Replace the particles with those of a reference IC file
        (IC_evrard4.cu:245-260 layout); returns the file's eps column if asked."""
        n = ic_count(path)
        eps = np.zeros(max(n, 1)) if want_eps else None
        self._chk(self._L.sph_load_ic(self._h, str(path).encode(), _ptr(eps)), "sph_load_ic")
        return eps[:n] if want_eps else None

    def write_ic(self, path, eps=None):
        """Write the particles as a reference IC file (eps defaults to h)."""
        e = None if eps is None else _f64(eps)
        self._chk(self._L.sph_write_ic(self._h, str(path).encode(), _ptr(e)), "sph_write_ic")

    def write_snapshot(self, path, ion_frac=None):
        """Write a snapshot in the reference's saveArraysToBinary layout
        (hfvCLibs_v7_hfv_v2.h:107-143)."""
        ion = None if ion_frac is None else np.ascontiguousarray(ion_frac, dtype=np.float32)
        nion = 0 if ion is None else int(ion.size)
        self._chk(self._L.sph_write_snapshot(self._h, str(path).encode(), _ptr(ion), nion),
                  "sph_write_snapshot")

    def write_restart(self, path):
        """FP64 restart file of the whole state (storage order kept)."""
        self._chk(self._L.sph_write_restart(self._h, str(path).encode()), "sph_write_restart")

    def read_restart(self, path):
        """Replace the particles with a restart file's; the next step
        continues exactly where the writing context would have."""
        self._chk(self._L.sph_read_restart(self._h, str(path).encode()), "sph_read_restart")

    def get(self, name: str, storage_order=False, out=None) -> np.ndarray:
        """Field in original (or storage) order.  `out`: an existing C-contiguous
        float64 array of n values (e.g. pinned host memory) to copy into."""
        if out is None:
            out = np.zeros(self.n)
        elif out.dtype != np.float64 or out.shape != (self.n,) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of n values")
        self._chk(self._L.sph_get_field(self._h, L.FIELD[name], _ptr(out), 1, int(storage_order)),
                  f"get {name}")
        return out

    def set(self, name: str, arr, storage_order=False):
        a = _f64(arr)
        self._chk(self._L.sph_set_field(self._h, L.FIELD[name], _ptr(a), 1, int(storage_order)),
                  f"set {name}")

    def set_fields(self, arrays: dict, storage_order=False):
        """Several fields in one library call ({name: array of n values})."""
        names = list(arrays)
        arrs = [_f64(arrays[k]) for k in names]
        ids = np.array([L.FIELD[k] for k in names], np.int32)
        ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        self._chk(self._L.sph_set_fields(self._h, len(arrs), _ptr(ids), ptrs, 1,
                                         int(storage_order)), "set_fields")

    def get_fields(self, names, storage_order=False, out=None) -> dict:
        """Several fields in one library call; `out`: {name: C-contiguous
        float64 array of n values} to copy into (e.g. pinned host memory)."""
        names = list(names)
        res = {}
        for k in names:
            a = None if out is None else out.get(k)
            if a is None:
                a = np.zeros(self.n)
            elif a.dtype != np.float64 or a.shape != (self.n,) or not a.flags.c_contiguous:
                raise ValueError("out arrays must be C-contiguous float64 arrays of n values")
            res[k] = a
        ids = np.array([L.FIELD[k] for k in names], np.int32)
        ptrs = (C.c_void_p * len(names))(*[res[k].ctypes.data for k in names])
        self._chk(self._L.sph_get_fields(self._h, len(names), _ptr(ids), ptrs, 1,
                                         int(storage_order)), "get_fields")
        return res

    def step_io(self, inputs: dict, outputs: dict):
        """One step with its host transfers (sph_step_io): the fields of
        `inputs` ({name: array of n values}) are copied in, one step runs, and
        the fields of `outputs` ({name: C-contiguous float64 array of n
        values}, e.g. pinned host memory) are filled with the step's results,
        copied out while the rest of the step runs.  Caller (original) order."""
        names_in = list(inputs)
        arrs = [_f64(inputs[k]) for k in names_in]
        ids_in = np.array([L.FIELD[k] for k in names_in], np.int32)
        ptr_in = (C.c_void_p * max(len(arrs), 1))(*[a.ctypes.data for a in arrs])
        names_out = list(outputs)
        for k in names_out:
            a = outputs[k]
            if a.dtype != np.float64 or a.shape != (self.n,) or not a.flags.c_contiguous:
                raise ValueError("output arrays must be C-contiguous float64 arrays of n values")
        ids_out = np.array([L.FIELD[k] for k in names_out], np.int32)
        ptr_out = (C.c_void_p * max(len(names_out), 1))(*[outputs[k].ctypes.data for k in names_out])
        self._chk(self._L.sph_step_io(self._h, len(arrs), _ptr(ids_in), ptr_in, len(names_out),
                                      _ptr(ids_out), ptr_out), "step_io")
        return outputs

    def get_pos(self, storage_order=False):
        return np.stack([self.get(k, storage_order) for k in "xyz"], 1)

    def get_vel(self, storage_order=False):
        return np.stack([self.get(k, storage_order) for k in ("vx", "vy", "vz")], 1)

    def get_acc(self, which="sph", storage_order=False):
        return np.stack([self.get(f"a{k}_{which}", storage_order) for k in "xyz"], 1)

    def ids(self) -> np.ndarray:
        out = np.zeros(self.n, np.int32)
        self._chk(self._L.sph_get_ids(self._h, _ptr(out), 1), "ids")
        return out

    def status(self, reset=False) -> dict:
        out = np.zeros(len(L.STATUS), np.int64)
        self._chk(self._L.sph_get_status(self._h, _ptr(out), int(reset)), "status")
        return dict(zip(L.STATUS, out.tolist()))

    @property
    def dt(self) -> np.ndarray:
        out = np.zeros(max(self.n_clouds, 1))
        self._chk(self._L.sph_get_dt(self._h, _ptr(out)), "dt")
        return out

    @dt.setter
    def dt(self, v):
        a = _f64(np.broadcast_to(v, (max(self.n_clouds, 1),)))
        self._chk(self._L.sph_set_dt(self._h, _ptr(a)), "set dt")

    # -- phases -------------------------------------------------------------
    def sort(self):
        self._chk(self._L.sph_sort(self._h), "sph_sort")

    def sort_info(self):
        keys = np.zeros(self.n, np.uint64)
        perm = np.zeros(self.n, np.int32)
        self._chk(self._L.sph_get_sort(self._h, _ptr(keys), _ptr(perm), 1), "sort_info")
        return keys, perm

    def build_tree(self):
        self._chk(self._L.sph_build_tree(self._h), "sph_build_tree")

    def tree(self):
        nn = 2 * self.n - 1
        node = np.zeros((nn, 16))
        child = np.zeros(2 * nn, np.int32)
        first = np.zeros(nn, np.int32)
        last = np.zeros(nn, np.int32)
        r2 = np.zeros(nn)
        hmax = np.zeros(nn)
        self._chk(self._L.sph_get_tree(self._h, _ptr(node), _ptr(child), _ptr(first), _ptr(last),
                                       _ptr(r2), _ptr(hmax), 1), "tree")
        return dict(node=node, child=child, first=first, last=last, open_r2=r2, hmax=hmax)

    def groups(self):
        """(count, start, size) of the walk/search groups of the last tree."""
        ng = C.c_int32()
        self._chk(self._L.sph_get_groups(self._h, C.byref(ng), None, None, 1), "groups")
        gs = np.zeros(max(ng.value, 1), np.int32)
        gc = np.zeros(max(ng.value, 1), np.int32)
        self._chk(self._L.sph_get_groups(self._h, C.byref(ng), _ptr(gs), _ptr(gc), 1), "groups")
        return ng.value, gs[: ng.value], gc[: ng.value]

    def smoothing_h(self):
        self._chk(self._L.sph_smoothing_h(self._h), "sph_smoothing_h")

    def smoothing_h_count(self, n_target=50, n_tol=5, step_frac=0.003, max_iter=10000):
        """The reference's own count iteration (libsx.py:854-902): h moves by
        -/+ step_frac h until n_target - n_tol <= #(|r_ij| < 2h) <= n_target
        + n_tol, bit-exact with the reference on the same positions."""
        self._chk(self._L.sph_smoothing_h_count(self._h, int(n_target), int(n_tol),
                                                float(step_frac), int(max_iter)),
                  "sph_smoothing_h_count")

    def smoothing_length_kth(self, k=50):
        """h = half the k-th smallest distance (self at 0), the reference's
        smoothing_length_mpi (libsx.py:777-800) for k = 50."""
        self._chk(self._L.sph_smoothing_length_kth(self._h, int(k)), "sph_smoothing_length_kth")

    def neighbours(self):
        self._chk(self._L.sph_neighbours(self._h), "sph_neighbours")

    def neighbour_lists(self):
        """Canonical CSR over storage order, rows sorted ascending."""
        off = np.zeros(self.n + 1, np.int64)
        self._chk(self._L.sph_get_neighbours(self._h, _ptr(off), None, 0, 1), "ngb count")
        lst = np.zeros(max(int(off[-1]), 1), np.int32)
        self._chk(self._L.sph_get_neighbours(self._h, _ptr(off), _ptr(lst), len(lst), 1),
                  "ngb lists")
        return off, lst[: off[-1]]

    def density(self):
        self._chk(self._L.sph_density(self._h), "sph_density")

    def divcurl(self):
        self._chk(self._L.sph_divcurl(self._h), "sph_divcurl")

    def forces(self):
        self._chk(self._L.sph_forces(self._h), "sph_forces")

    def dudt(self):
        self._chk(self._L.sph_dudt(self._h), "sph_dudt")

    def gravity(self):
        self._chk(self._L.sph_gravity(self._h), "sph_gravity")

    def gravity_direct(self, targets):
        """FP64 Plummer direct sum onto storage indices -> (acc[n,3], pot[n])."""
        t = np.ascontiguousarray(targets, dtype=np.int32)
        out = np.zeros(4 * len(t))
        self._chk(self._L.sph_gravity_direct(self._h, len(t), _ptr(t), _ptr(out), 1),
                  "gravity_direct")
        out = out.reshape(-1, 4)
        return out[:, :3].copy(), out[:, 3].copy()

    def gravity_direct_spline(self, eps, targets):
        t = np.ascontiguousarray(targets, dtype=np.int32)
        e = _f64(eps)
        out = np.zeros(3 * len(t))
        self._chk(self._L.sph_gravity_direct_spline(self._h, _ptr(e), len(t), _ptr(t), _ptr(out), 1),
                  "gravity_direct_spline")
        return out.reshape(-1, 3)

    def gravity_direct_spline_rows(self, eps, nbeg, nend):
        """The reference's partial field of rows [nbeg, nend) (original order,
        (n, 3)); fields of a partition of the rows sum to the full field."""
        e = _f64(eps)
        out = np.zeros((self.n, 3))
        self._chk(self._L.sph_gravity_direct_spline_rows(self._h, _ptr(e), int(nbeg), int(nend),
                                                         _ptr(out), 1),
                  "gravity_direct_spline_rows")
        return out

    def counters(self):
        out = np.zeros(2, np.int64)
        self._chk(self._L.sph_get_counters(self._h, _ptr(out)), "counters")
        far = np.zeros(1, np.int64)
        self._chk(self._L.sph_get_far_cells(self._h, _ptr(far)), "far cells")
        sg = np.zeros(2, np.int64)
        self._chk(self._L.sph_get_supergroup_stats(self._h, _ptr(sg)), "super-group stats")
        return {"cells": int(out[0]), "particles": int(out[1]), "far_cells": int(far[0]),
                "sg_far_cells": int(sg[0]), "sg_fallback": int(sg[1])}

    def kick(self, fac=0.5):
        self._chk(self._L.sph_kick(self._h, fac), "sph_kick")

    def drift(self):
        self._chk(self._L.sph_drift(self._h), "sph_drift")

    def update_u(self, first=False):
        self._chk(self._L.sph_update_u(self._h, int(first)), "sph_update_u")

    def cfl_dt(self):
        out = np.zeros(max(self.n_clouds, 1))
        self._chk(self._L.sph_cfl_dt(self._h, _ptr(out)), "sph_cfl_dt")
        return out

    def dt_individual(self) -> dict:
        """Per-particle steps of the reference's six criteria over the
        neighbour lists (dt_array_indiv_dt, hfvCLibs_v7_hfv_v2.h:999-1078),
        dh/dt and power-of-two bins, in original order; the per-cloud minimum
        becomes the next step."""
        n = self.n
        dt, dh = np.zeros(n), np.zeros(n)
        b = np.zeros(n, np.int32)
        self._chk(self._L.sph_dt_individual(self._h, _ptr(dt), _ptr(dh), _ptr(b), 1),
                  "sph_dt_individual")
        return {"dt": dt, "dhdt": dh, "bin": b}

    def outflow_inject(self, mdot, v_in, m_particle, u_inject, r_max=1e-3, h_first=1e-3,
                       seed=0, leftover=0.0, cloud=None):
        """Spawn mdot * dt + leftover as outflow pairs (outflow_injector2,
        hfvCLibs_v7_hfv_v2.h:1094-1210); returns (particles added, leftover
        mass).  The new particles get the next original ids."""
        p = L.SphOutflowParams(mdot=mdot, v_in=v_in, m_particle=m_particle, u_inject=u_inject,
                               r_max=r_max, h_first=h_first, seed=int(seed),
                               cloud=self.n_clouds - 1 if cloud is None else int(cloud))
        left = C.c_double(leftover)
        added = C.c_int32(0)
        self._chk(self._L.sph_outflow_inject(self._h, C.byref(p), C.byref(left), C.byref(added)),
                  "sph_outflow_inject")
        return int(added.value), float(left.value)

    def energies(self) -> dict:
        out = np.zeros(10)
        self._chk(self._L.sph_energies(self._h, _ptr(out)), "sph_energies")
        keys = ["KE", "U", "PE", "px", "py", "pz", "Lx", "Ly", "Lz", "M"]
        return dict(zip(keys, out.tolist()))

    def prologue(self):
        self._chk(self._L.sph_prologue(self._h), "sph_prologue")

    def step(self, nsteps=1):
        self._chk(self._L.sph_step(self._h, nsteps), "sph_step")

    def debug_array(self, which: str) -> np.ndarray:
        k = {"cand_cnt": 0, "ngb_cnt": 1, "retry": 2, "hcand": 3, "p0_h": 4, "p1_m": 5,
             "tree_search": 6}[which]
        out = np.zeros(self.n + (k == 6), np.float64 if 3 <= k <= 5 else np.int32)
        self._chk(self._L.sph_debug_copy(self._h, k, _ptr(out), 1), "debug_copy")
        return out

    def phase_times(self) -> dict:
        ms = (C.c_float * 12)()
        rc = self._L.sph_get_phase_times(self._h, ms)
        if rc < 0:
            L.check(rc, "phase_times", self._h)
        return dict(zip(L.PHASES, [float(v) for v in ms]))

    def time_steps(self, nsteps) -> float:
        """Device time in ms of nsteps of sph_step (CUDA events on the
        context's stream)."""
        ms = C.c_float()
        self._chk(self._L.sph_time_steps(self._h, int(nsteps), C.byref(ms)), "sph_time_steps")
        return float(ms.value)

    def graph_kernel_count(self) -> int:
        c = C.c_int32()
        self._chk(self._L.sph_graph_kernel_count(self._h, C.byref(c)), "graph_kernel_count")
        return int(c.value)

    def graph_kernels_launched(self, reset=False) -> int:
        """Kernel nodes of the step graphs launched since the last reset."""
        c = C.c_int64(0)
        self._chk(self._L.sph_graph_kernels_launched(self._h, C.byref(c), int(bool(reset))),
                  "graph_kernels_launched")
        return int(c.value)

    def rows_kept(self):
        """Particles whose candidate row the last h iteration kept instead of
        searching again."""
        c = C.c_int64(0)
        self._chk(self._L.sph_rows_kept(self._h, C.byref(c)), "rows_kept")
        return int(c.value)

    def fp32_peak_tflops(self) -> float:
        v = C.c_double()
        self._chk(self._L.sph_measure_fp32_peak(self._h, C.byref(v)), "fp32 peak")
        return float(v.value)

    def sync(self):
        self._chk(self._L.sph_sync(self._h), "sph_sync")

    def set_stream(self, stream_handle: int):
        """Queue all work on an existing CUDA stream (e.g. a torch stream's
        ``cuda_stream``); the library stops using its own stream."""
        self._chk(self._L.sph_set_stream(self._h, C.c_void_p(stream_handle)), "sph_set_stream")

    # -- cooling --------------------------------------------------------------
    def cooling_setup(self, params: dict, log_lambda):
        p = L.SphCoolingParams()
        for k, v in params.items():
            setattr(p, k, v)
        ll = _f64(log_lambda)
        self._chk(self._L.sph_cooling_setup(self._h, C.byref(p), _ptr(ll)), "cooling_setup")

    def cooling_exact(self):
        self._chk(self._L.sph_cooling_exact(self._h), "cooling_exact")

    def cooling_mlp(self):
        self._chk(self._L.sph_cooling_mlp(self._h), "cooling_mlp")

    def cooling_table_load(self, path, **params):
        """Read a heating/cooling grid file in the layout of the reference's
        coolHeatGridNew.bin (see sph_2_b200.cooling.write_table_file)."""
        p = L.SphCoolTableParams(unit_rho=1.0, unit_u=1.0, unit_t=1.0, unit_length=1.0,
                                 kpc_cm=3.086e21, XH=0.70, mH=1.6726e-24, z_row=1)
        for k, v in params.items():
            setattr(p, k, v)
        self._chk(self._L.sph_cooling_table_load(self._h, str(path).encode(), C.byref(p)),
                  "sph_cooling_table_load")

    def cooling_table(self):
        self._chk(self._L.sph_cooling_table(self._h), "sph_cooling_table")

    def ion_frac(self, n_species) -> np.ndarray:
        out = np.zeros((self.n, n_species), np.float32)
        self._chk(self._L.sph_get_ion_frac(self._h, _ptr(out), 1), "sph_get_ion_frac")
        return out

    # -- cooling surrogate ----------------------------------------------------
    def mlp_set(self, params, norm):
        p = np.ascontiguousarray(params, np.float32)
        nm = np.ascontiguousarray(norm, np.float32)
        self._chk(self._L.sph_mlp_set(self._h, _ptr(p), _ptr(nm), 1), "mlp_set")

    def mlp_get(self):
        p = np.zeros(L.MLP_NPARAM, np.float32)
        nm = np.zeros(8, np.float32)
        self._chk(self._L.sph_mlp_get(self._h, _ptr(p), _ptr(nm), 1), "mlp_get")
        return p, nm

    def mlp_forward(self, X):
        X = np.ascontiguousarray(X, np.float32)
        y = np.zeros(len(X), np.float32)
        self._chk(self._L.sph_mlp_forward(self._h, len(X), _ptr(X), _ptr(y), 1), "mlp_forward")
        return y

    def mlp_grad(self, X, t):
        X = np.ascontiguousarray(X, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(L.MLP_NPARAM, np.float32)
        loss = np.zeros(1, np.float32)
        self._chk(self._L.sph_mlp_grad(self._h, len(t), _ptr(X), _ptr(t), _ptr(g), _ptr(loss), 1),
                  "mlp_grad")
        return g, float(loss[0])

    def cool_solve_mlp(self, rho, u_old, dt):
        """Surrogate + Newton polish + exact fallback on device copies of the
        arrays (cgs); returns (u_new, fell_back)."""
        import torch
        d = {k: torch.as_tensor(np.array(v, np.float64), device="cuda")
             for k, v in (("rho", rho), ("u", u_old), ("dt", np.broadcast_to(dt, np.shape(rho))))}
        out = torch.empty_like(d["u"])
        fb = torch.empty(len(out), dtype=torch.int32, device="cuda")
        self._chk(self._L.sph_cool_solve_mlp(self._h, len(out), C.c_void_p(d["rho"].data_ptr()),
                                             C.c_void_p(d["u"].data_ptr()),
                                             C.c_void_p(d["dt"].data_ptr()),
                                             C.c_void_p(out.data_ptr()),
                                             C.c_void_p(fb.data_ptr())), "cool_solve_mlp")
        self.sync()
        return out.cpu().numpy(), fb.cpu().numpy()

    def cool_solve(self, rho, u_old, dt):
        rho, u_old = _f64(rho), _f64(u_old)
        dt = _f64(np.broadcast_to(dt, rho.shape))
        out = np.zeros_like(rho)
        it = np.zeros(len(rho), np.int32)
        self._chk(self._L.sph_cool_solve(self._h, len(rho), _ptr(rho), _ptr(u_old), _ptr(dt),
                                         _ptr(out), _ptr(it), 1), "cool_solve")
        return out, it
