"""ctypes binding of libsphb200.so (declarations in include/sph_b200.h).

The library is built in-tree by ``python -m sph_2_b200.build`` (or
``__graft_entry__.build()``).  There is no fallback: if the shared library is
missing or no CUDA device is present, the calls fail with an exception.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsphb200.so")

# ---- constants mirrored from include/sph_b200.h ----
SPH_OK = 0
ERRORS = {
    -1: "SPH_ERR_ARG", -2: "SPH_ERR_CUDA", -3: "SPH_ERR_CAPACITY", -4: "SPH_ERR_NOCONV",
    -5: "SPH_ERR_OVERFLOW", -6: "SPH_ERR_NONFINITE", -7: "SPH_ERR_STATE", -8: "SPH_ERR_NOMEM",
    -9: "SPH_ERR_IO",
}
PREC = {"fp64": 0, "mixed": 1}
AV = {"mg83": 0, "gadget": 1}
DT_MODE = {"courant": 0, "individual": 1}
FIELDS = ["x", "y", "z", "vx", "vy", "vz", "m", "h", "u", "rho", "P", "c", "divV", "curlV",
          "ax_sph", "ay_sph", "az_sph", "ax_grav", "ay_grav", "az_grav", "dudt", "vsig", "pot",
          "dudt_prev", "u_prev"]
FIELD = {name: k for k, name in enumerate(FIELDS)}
STATUS = ["h_noconv", "ngb_overflow", "stack_overflow", "h_retry", "cool_noconv", "mlp_fallback",
          "nonfinite", "walk_stack_max", "wait_timeout"]
FLAG_DUDT_FUSED = 1
FLAG_COOLING = 2
FLAG_COOLING_MLP = 4
FLAG_NO_GRAPH = 8
FLAG_POTENTIAL = 16
FLAG_TIMING = 32
FLAG_COOLING_TABLE = 64
FLAG_STATIC_GRID = 128
FLAG_MLP_WARP_MMA = 256
FLAG_NO_ROW_REUSE = 512
PHASES = ["kick_drift", "sort", "tree", "smoothing_h", "neighbours", "density", "divcurl",
          "forces", "wait_kick", "dudt", "update_dt", "gravity"]
MLP_NPARAM = 3 * 64 + 64 + 64 * 64 + 64 + 64 + 1
NOALLOC_MAX_N = 262144


class SphConfig(C.Structure):
    _fields_ = [
        ("n_max", C.c_int32), ("n_cloud_max", C.c_int32), ("precision", C.c_int32),
        ("av_mode", C.c_int32), ("balsara", C.c_int32), ("leaf_size", C.c_int32),
        ("ngb_lanes", C.c_int32), ("block_size", C.c_int32), ("max_ngb", C.c_int32),
        ("h_max_iter", C.c_int32), ("flags", C.c_int32), ("walk_blocks", C.c_int32),
        ("n_ngb", C.c_double), ("h_tol", C.c_double), ("gamma", C.c_double),
        ("alpha", C.c_double), ("beta", C.c_double), ("eta", C.c_double), ("G", C.c_double),
        ("eps", C.c_double), ("theta", C.c_double), ("courant", C.c_double),
        ("dt_max", C.c_double), ("dt_fixed", C.c_double), ("theta_local", C.c_double),
        ("theta_small", C.c_double), ("small_cell", C.c_int32), ("dt_mode", C.c_int32),
        ("ext_sigma", C.c_double), ("rebuild_every", C.c_int32), ("reserved", C.c_int32),
    ]


class SphCoolTableParams(C.Structure):
    _fields_ = [
        ("unit_rho", C.c_double), ("unit_u", C.c_double), ("unit_t", C.c_double),
        ("unit_length", C.c_double), ("kpc_cm", C.c_double), ("XH", C.c_double),
        ("mH", C.c_double), ("z_row", C.c_int32), ("reserved", C.c_int32),
    ]


class SphOutflowParams(C.Structure):
    _fields_ = [
        ("mdot", C.c_double), ("v_in", C.c_double), ("m_particle", C.c_double),
        ("u_inject", C.c_double), ("r_max", C.c_double), ("h_first", C.c_double),
        ("seed", C.c_uint64), ("cloud", C.c_int32), ("reserved", C.c_int32),
    ]


class SphCoolingParams(C.Structure):
    _fields_ = [
        ("n_bins", C.c_int32), ("max_iter", C.c_int32), ("logT0", C.c_double),
        ("logT1", C.c_double), ("mu", C.c_double), ("gamma", C.c_double), ("XH", C.c_double),
        ("gamma_heat", C.c_double), ("tol", C.c_double), ("unit_rho", C.c_double),
        ("unit_u", C.c_double), ("unit_t", C.c_double), ("mlp_err_tol", C.c_double),
    ]


# (name, restype, argtypes) of every exported entry point
_P = C.c_void_p
_I = C.c_int32
_D = C.c_double
_F = C.c_float
SIGNATURES = [
    ("sph_default_config", C.c_int, [C.POINTER(SphConfig)]),
    ("sph_ctx_create", C.c_int, [C.POINTER(SphConfig), C.POINTER(_P)]),
    ("sph_ctx_destroy", None, [_P]),
    ("sph_set_stream", C.c_int, [_P, _P]),
    ("sph_sync", C.c_int, [_P]),
    ("sph_last_error", C.c_char_p, [_P]),
    ("sph_get_config", C.c_int, [_P, C.POINTER(SphConfig)]),
    ("sph_set_params", C.c_int, [_P, C.POINTER(SphConfig)]),
    ("sph_device_bytes", C.c_int64, [_P]),
    ("sph_load", C.c_int, [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I]),
    ("sph_count", C.c_int32, [_P]),
    ("sph_cloud_count", C.c_int32, [_P]),
    ("sph_get_field", C.c_int, [_P, _I, _P, _I, _I]),
    ("sph_set_field", C.c_int, [_P, _I, _P, _I, _I]),
    ("sph_set_fields", C.c_int, [_P, _I, _P, _P, _I, _I]),
    ("sph_get_fields", C.c_int, [_P, _I, _P, _P, _I, _I]),
    ("sph_step_io", C.c_int, [_P, _I, _P, _P, _I, _P, _P]),
    ("sph_get_ids", C.c_int, [_P, _P, _I]),
    ("sph_get_status", C.c_int, [_P, _P, _I]),
    ("sph_get_dt", C.c_int, [_P, _P]),
    ("sph_set_dt", C.c_int, [_P, _P]),
    ("sph_sort", C.c_int, [_P]),
    ("sph_get_sort", C.c_int, [_P, _P, _P, _I]),
    ("sph_build_tree", C.c_int, [_P]),
    ("sph_get_tree", C.c_int, [_P, _P, _P, _P, _P, _P, _P, _I]),
    ("sph_get_groups", C.c_int, [_P, _P, _P, _P, _I]),
    ("sph_smoothing_h", C.c_int, [_P]),
    ("sph_smoothing_h_count", C.c_int, [_P, _I, _I, _D, _I]),
    ("sph_smoothing_length_kth", C.c_int, [_P, _I]),
    ("sph_neighbours", C.c_int, [_P]),
    ("sph_get_neighbours", C.c_int, [_P, _P, _P, C.c_int64, _I]),
    ("sph_density", C.c_int, [_P]),
    ("sph_divcurl", C.c_int, [_P]),
    ("sph_forces", C.c_int, [_P]),
    ("sph_dudt", C.c_int, [_P]),
    ("sph_gravity", C.c_int, [_P]),
    ("sph_gravity_direct", C.c_int, [_P, _I, _P, _P, _I]),
    ("sph_gravity_direct_spline", C.c_int, [_P, _P, _I, _P, _P, _I]),
    ("sph_gravity_direct_spline_rows", C.c_int, [_P, _P, _I, _I, _P, _I]),
    ("sph_kick", C.c_int, [_P, _D]),
    ("sph_drift", C.c_int, [_P]),
    ("sph_update_u", C.c_int, [_P, _I]),
    ("sph_cfl_dt", C.c_int, [_P, _P]),
    ("sph_dt_individual", C.c_int, [_P, _P, _P, _P, _I]),
    ("sph_outflow_inject", C.c_int, [_P, C.POINTER(SphOutflowParams), _P, _P]),
    ("sph_energies", C.c_int, [_P, _P]),
    ("sph_get_far_cells", C.c_int, [_P, _P]),
    ("sph_get_supergroup_stats", C.c_int, [_P, _P]),
    ("sph_get_counters", C.c_int, [_P, _P]),
    ("sph_cooling_setup", C.c_int, [_P, C.POINTER(SphCoolingParams), _P]),
    ("sph_cooling_exact", C.c_int, [_P]),
    ("sph_cooling_mlp", C.c_int, [_P]),
    ("sph_cool_solve", C.c_int, [_P, _I, _P, _P, _P, _P, _P, _I]),
    ("sph_cooling_table_dims", C.c_int, [C.c_char_p, _P]),
    ("sph_cooling_table_load", C.c_int, [_P, C.c_char_p, C.POINTER(SphCoolTableParams)]),
    ("sph_cooling_table", C.c_int, [_P]),
    ("sph_get_ion_frac", C.c_int, [_P, _P, _I]),
    ("sph_mlp_set", C.c_int, [_P, _P, _P, _I]),
    ("sph_mlp_get", C.c_int, [_P, _P, _P, _I]),
    ("sph_mlp_forward", C.c_int, [_P, _I, _P, _P, _I]),
    ("sph_mlp_grad", C.c_int, [_P, _I, _P, _P, _P, _P, _I]),
    ("sph_mlp_train", C.c_int, [_P, _I, _P, _P, _I, _I, _F, _P]),
    ("sph_cool_solve_mlp", C.c_int, [_P, _I, _P, _P, _P, _P, _P]),
    ("sph_debug_copy", C.c_int, [_P, _I, _P, _I]),
    ("sph_get_phase_times", C.c_int, [_P, _P]),
    ("sph_time_steps", C.c_int, [_P, _I, _P]),
    ("sph_graph_kernel_count", C.c_int, [_P, _P]),
    ("sph_graph_kernels_launched", C.c_int, [_P, _P, _I]),
    ("sph_rows_kept", C.c_int, [_P, _P]),
    ("sph_measure_fp32_peak", C.c_int, [_P, _P]),
    ("sph_morton_sort_noalloc", C.c_int, [_P, _P, _P, _I, _P, _P, _P]),
    ("sph_ic_count", C.c_int, [C.c_char_p, _P]),
    ("sph_load_ic", C.c_int, [_P, C.c_char_p, _P]),
    ("sph_write_ic", C.c_int, [_P, C.c_char_p, _P]),
    ("sph_write_snapshot", C.c_int, [_P, C.c_char_p, _P, _I]),
    ("sph_write_restart", C.c_int, [_P, C.c_char_p]),
    ("sph_read_restart", C.c_int, [_P, C.c_char_p]),
    ("sph_prologue", C.c_int, [_P]),
    ("sph_step", C.c_int, [_P, _I]),
]

_lib = None


def load():
    """Load libsphb200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} not found: build it with `python -m sph_2_b200.build` "
            "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class SphError(RuntimeError):
    def __init__(self, code, where, detail=""):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)} {detail}".strip())


def check(rc, where, ctx=None):
    if rc != SPH_OK:
        detail = ""
        if ctx is not None and rc == -2:
            detail = load().sph_last_error(ctx).decode(errors="replace")
        raise SphError(rc, where, detail)
    return rc
