"""Benchmark of the per-step hot path: particle-steps/s of the Evrard collapse
at N = 1,000,000 on one B200, mixed precision (FP32 walk and SPH sums with
Kahan compensation, FP64 positions / integration / h convergence) beside the
plain FP64 step on the same GPU, with the acceleration error of each against
an FP64 direct-summation oracle on a seeded 10k-particle subset.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  Multi-GPU (torchrun): every rank advances its
own replica of the workload (the single sphere does not shard without a halo
exchange), timing is the max over ranks, value is the whole-job
throughput.  --impl reference times the reference's CPU implementation of the
step (the oracle's C restatement of MPI_sph/sph_code/libsx.py + shear.py, the
reference's all-pairs loops with its row-range decomposition) on the host
cores, on a bounded row sample per step, extrapolated to the full N.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at N=1M Evrard (mixed vs FP64 plain, same B200) at <=1e-4 accel err"
UNIT = "particle-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--theta", type=float, default=0.35, help="opening angle, mixed arm")
    ap.add_argument("--theta-fp64", type=float, default=0.38, help="opening angle, FP64 plain arm")
    ap.add_argument("--theta-local", type=float, default=0.28,
                    help="mixed walk: far cells through group Taylor expansions (0: off)")
    ap.add_argument("--theta-small", type=float, default=0.45,
                    help="mixed walk: opening angle of the cells of at most --small-cell particles")
    ap.add_argument("--small-cell", type=int, default=128)
    ap.add_argument("--no-row-reuse", action="store_true",
                    help="search every particle in each h iteration (no kept candidate rows)")
    ap.add_argument("--leaf", type=int, default=8)
    ap.add_argument("--lanes", type=int, default=4)
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 plain arm")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--err-subset", type=int, default=10_000)
    ap.add_argument("--workload", default="evrard", choices=["evrard", "ensemble", "cooling", "large"],
                    help="evrard: the headline line; ensemble / cooling / large: extra workloads")
    ap.add_argument("--clouds", type=int, default=64)
    ap.add_argument("--tune", action="store_true",
                    help="run the autotuner before timing the headline (the ensemble is always tuned)")
    ap.add_argument("--no-tune", action="store_true", help="do not tune the ensemble either")
    ap.add_argument("--no-theta-table", action="store_true")
    ap.add_argument("--arm", default="mixed", choices=["mixed", "fp64"],
                    help="precision of the timed headline arm (fp64: profile the plain step)")
    ap.add_argument("--static-grid", action="store_true",
                    help="group kernels on a grid over the groups instead of the work queue")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-cooling", action="store_true", help="skip the 2M cooling-cloud key")
    ap.add_argument("--no-large", action="store_true", help="skip the 16M Evrard key")
    ap.add_argument("--large-steps", type=int, default=50)
    ap.add_argument("--rebuild-every", type=int, default=4,
                    help="sort and split the tree every k-th step, refit it between (both arms)")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", str(self.index), "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ CPU sample ----
def cpu_reference_sample(n, rows_per_thread=64, seed=42):
    """One step of the reference's CPU path (oracle restatement of
    h_smooth_fast_mpi, getDensity_mpi, getAcc_g_smth_mimj_mpi, div_curlVel_mpi,
    getAcc_sph_shear_mpi, get_dU_shear_mpi -- sph_mpi4_v4.py:278-416) on a
    contiguous row slice of size rows_per_thread * threads against all n
    sources, extrapolated by n/rows.  Returns (seconds per full step, info)."""
    from oracle import oracle as O
    from sph_2_b200 import ic
    d = ic.evrard(n, seed=seed)
    pos = np.ascontiguousarray(d["pos"])
    m, u, h = d["m"], d["u"], d["h"]
    r = np.linalg.norm(pos, axis=1)
    rho = 1.0 / (2.0 * np.pi * np.maximum(r, 1e-3))          # analytic profile for j-data
    P = (5 / 3 - 1) * rho * u
    c = np.sqrt(5 / 3 * (5 / 3 - 1) * u)
    v = np.zeros_like(pos)
    zero = np.zeros(n)
    eps = np.full(n, 1e-2)
    thr = O.num_threads()
    rows = min(n, rows_per_thread * thr)
    nb = n // 2 - rows // 2
    ne = nb + rows
    # steady state of the reference's h iteration: h of the previous step is
    # already converged, so converge the sample rows once (untimed)
    hs = h.copy()
    hs[nb:ne] = O.ref_h_smooth_fast(nb, ne, pos, h)
    t = {}
    t0 = time.perf_counter(); O.ref_h_smooth_fast(nb, ne, pos, hs); t["h_smooth_fast"] = time.perf_counter() - t0
    t0 = time.perf_counter(); O.ref_getDensity(nb, ne, pos, m, hs); t["density"] = time.perf_counter() - t0
    t0 = time.perf_counter(); O.ref_getAcc_g_smth_mimj(nb, ne, pos, m, 1.0, eps); t["gravity"] = time.perf_counter() - t0
    t0 = time.perf_counter(); O.ref_div_curlVel(nb, ne, pos, v, rho, m, hs); t["divcurl"] = time.perf_counter() - t0
    t0 = time.perf_counter(); O.ref_getAcc_sph(nb, ne, pos, v, rho, P, c, hs, m, zero, zero, 1.0); t["acc_sph"] = time.perf_counter() - t0
    t0 = time.perf_counter(); O.ref_get_dU(nb, ne, pos, v, rho, P, c, hs, m, zero, zero, 1.0); t["dudt"] = time.perf_counter() - t0
    scale = n / rows
    step_s = sum(t.values()) * scale
    return step_s, dict(rows=rows, threads=thr, phase_s={k: round(v * scale, 3) for k, v in t.items()},
                        sample_s=round(sum(t.values()), 3))


def cpu_reference_full_step(n=10_000, seed=42, steps=3):
    """Every row of the reference's CPU step at N = 10,000 (the plain FP64
    Evrard configuration): h_smooth_fast_mpi, getDensity_mpi,
    getAcc_g_smth_mimj_mpi, div_curlVel_mpi, getAcc_sph_shear_mpi,
    get_dU_shear_mpi and the KDK updates of sph_mpi4_v4.py:278-416, through
    the oracle's C restatement on all host threads; measured, not
    extrapolated.  Returns (mean seconds per step, phase seconds)."""
    from oracle import oracle as O
    from sph_2_b200 import ic
    d = ic.evrard(n, seed=seed)
    pos = np.ascontiguousarray(d["pos"])
    m, u = d["m"], d["u"].copy()
    v = np.zeros_like(pos)
    eps = np.full(n, 1e-2)
    gama, dt = 5.0 / 3.0, 1e-3
    h = O.ref_h_smooth_fast(0, n, pos, d["h"])          # converged start (untimed)
    acc = np.zeros_like(pos)
    times, phases = [], {}
    for _ in range(steps):
        t = {}
        t0 = time.perf_counter()
        v = v + 0.5 * dt * acc
        pos = pos + dt * v
        t["kick_drift"] = time.perf_counter() - t0
        t0 = time.perf_counter(); h = O.ref_h_smooth_fast(0, n, pos, h); t["h_smooth_fast"] = time.perf_counter() - t0
        t0 = time.perf_counter(); rho = O.ref_getDensity(0, n, pos, m, h); t["density"] = time.perf_counter() - t0
        t0 = time.perf_counter(); ag = O.ref_getAcc_g_smth_mimj(0, n, pos, m, 1.0, eps); t["gravity"] = time.perf_counter() - t0
        P = (gama - 1.0) * rho * u
        c = np.sqrt(gama * (gama - 1.0) * u)
        t0 = time.perf_counter(); dv, cv = O.ref_div_curlVel(0, n, pos, v, rho, m, h); t["divcurl"] = time.perf_counter() - t0
        t0 = time.perf_counter(); asph = O.ref_getAcc_sph(0, n, pos, v, rho, P, c, h, m, dv, cv, 1.0); t["acc_sph"] = time.perf_counter() - t0
        acc = ag + asph
        v = v + 0.5 * dt * acc
        t0 = time.perf_counter(); du = O.ref_get_dU(0, n, pos, v, rho, P, c, h, m, dv, cv, 1.0); t["dudt"] = time.perf_counter() - t0
        u = u + dt * du
        times.append(sum(t.values()))
        for k, val in t.items():
            phases[k] = phases.get(k, 0.0) + val / steps
    return float(np.mean(times)), {k: round(val, 4) for k, val in phases.items()}


def reference_arm(a, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    thr = O.num_threads()
    rpt = 32
    full_s, full_phases = cpu_reference_full_step()
    for _ in range(a.warmup):
        cpu_reference_sample(a.n, rpt)
    steps = []
    info = None
    for _ in range(a.steps):
        s, info = cpu_reference_sample(a.n, rpt)
        steps.append(s)
    step_s = float(np.mean(steps))
    value = a.n / step_s
    sample = (f"{info['rows']} rows x {a.n} sources per phase per step (contiguous slice at N/2), "
              f"6 phases, extrapolated x{a.n / info['rows']:.0f}; oracle C restatement of the "
              "reference numba step, OpenMP over rows")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": step_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Evrard sphere)",
        "config": {"workload": f"evrard_n{a.n}_reference_cpu_step", "n": a.n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "phase_s_extrapolated": info["phase_s"],
        "cfg0_measured": {"n": 10_000, "s_per_step": full_s,
                          "particle_steps_per_s": 10_000 / full_s, "threads": thr,
                          "phase_s": full_phases,
                          "what": "every row of the reference CPU step at N = 10,000, 3 steps, "
                                  "oracle C restatement, measured (not extrapolated)"},
    }
    print(json.dumps(line))


# ------------------------------------------------------------------ ours ----
# compulsory bytes per particle of each SPH-side phase (FP64 arrays; neighbour
# j-data re-reads that hit L1/L2 are not counted), the figures the per-phase
# roofline fractions use
PHASE_BYTES = {"sort": 416, "smoothing_h": 312, "neighbours": 288, "density_divcurl": 344,
               "forces": 392, "dudt": 392}


def hbm_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def phase_roofline(ctx, n, stream, reps=3):
    """Each phase run alone through the C ABI on the context's current state,
    timed with CUDA events on its stream: ms per call, and for the SPH-side
    phases the compulsory bytes per particle / time against the HBM peak (the
    walk's FP32 figure is in the roofline object)."""
    import torch
    calls = [("sort", ctx.sort), ("tree", ctx.build_tree), ("smoothing_h", ctx.smoothing_h),
             ("neighbours", ctx.neighbours), ("density_divcurl", lambda: (ctx.density(), ctx.divcurl())),
             ("forces", ctx.forces), ("dudt", ctx.dudt), ("gravity", ctx.gravity)]
    peak, src = hbm_peak_gbs()
    out = {}
    for name, fn in calls:
        fn()
        ctx.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        row = {"ms": ms}
        if name in PHASE_BYTES:
            gbs = PHASE_BYTES[name] * n / (ms * 1e-3) / 1e9
            row.update(bytes_per_particle=PHASE_BYTES[name], achieved_gbs=gbs, frac_hbm=gbs / peak)
        out[name] = row
    out["peak_gbs"] = peak
    out["peak_source"] = src
    return out


def rms_rel(a, b):
    num = np.sum((a - b) ** 2, axis=1)
    den = np.sum(b * b, axis=1) + 1e-300
    return float(np.sqrt(np.mean(num / den)))


def walk_kw(a, precision):
    """Opening-angle settings of one arm: the mixed arm with its group
    expansions and small-cell angle, the FP64 plain arm with theta alone."""
    if precision == "mixed":
        return dict(theta=a.theta, theta_local=a.theta_local, theta_small=a.theta_small,
                    small_cell=a.small_cell)
    return dict(theta=a.theta_fp64)


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        reference_arm(a, rank)
        return
    if a.workload != "evrard":
        extra_workload(a, world, rank, local)
        return

    import torch
    import torch.distributed as dist
    from sph_2_b200 import Config, Context, ic
    from sph_2_b200 import _lib as L

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = a.n
    d = ic.evrard(n, seed=42 + rank)
    # high priority for the SPH passes; the library runs gravity on its own
    # low-priority stream beside them
    stream = torch.cuda.Stream(priority=-10)

    def make(precision, flags=0, vel=None, walk=None):
        if a.static_grid:
            flags |= L.FLAG_STATIC_GRID
        if a.no_row_reuse:
            flags |= L.FLAG_NO_ROW_REUSE
        cfg = Config(n_max=n, precision=precision, leaf_size=a.leaf, ngb_lanes=a.lanes,
                     flags=flags, rebuild_every=a.rebuild_every, **(walk or walk_kw(a, precision)))
        c = Context(cfg)
        c.set_stream(stream.cuda_stream)
        c.load(d["pos"], d["vel"] if vel is None else vel, d["m"], d["h"], d["u"])
        c.prologue()
        return c

    def timed_steps(ctx, steps, warmup):
        ctx.step(warmup)
        ctx.sync()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record()
            ctx.step(steps)
            e1.record()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    # ---- mixed precision arm (the headline) ----
    ctx = make(a.arm, L.FLAG_TIMING)
    sampler = ClockSampler(local)
    ctx.step(a.warmup)
    ctx.sync()
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.graph_kernels_launched(reset=True)
    with torch.cuda.stream(stream):
        e0.record()
        ctx.step(a.steps)
        e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches_timed = ctx.graph_kernels_launched()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * n * a.steps / (ms * 1e-3)
    phases = ctx.phase_times()
    status = ctx.status()

    # ---- roofline of the dominant kernel (the gravity walk) ----
    reps = 5
    ctx.gravity()
    ctx.sync()
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        w0.record()
        for _ in range(reps):
            ctx.gravity()
        w1.record()
    torch.cuda.synchronize()
    walk_ms = w0.elapsed_time(w1) / reps
    cnt = ctx.counters()
    # far cells: 190 flop each (35 Taylor coefficients), once per group or
    # super-group; 115 per particle to evaluate each expansion (the group's
    # and its super-group's)
    flops = 60.0 * cnt["cells"] + 20.0 * cnt["particles"] + 190.0 * cnt["far_cells"] + \
        (115.0 * n if cnt["far_cells"] else 0.0) + (115.0 * n if cnt.get("sg_far_cells") else 0.0)
    fp32_peak = ctx.fp32_peak_tflops()
    achieved = flops / (walk_ms * 1e-3) / 1e12
    roofline = {"kernel": "k_sg_walk + k_walk<float> (gravity walk)", "bound": "fp32",
                "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "traffic": None,
                "peak_source": ("FP32 FMA-chain kernels, scalar and packed f32x2, the larger, "
                                "measured in this run (MEASURED_PEAKS.json has no FP32 figure)"),
                "algorithmic": ("60 flop per quadrupole cell + 20 per particle interaction "
                                "+ 190 per far cell (once per group or super-group) + 115 per "
                                "particle for each of the group and super-group expansions"),
                "interactions_per_particle": {"cells": cnt["cells"] / n,
                                              "particles": cnt["particles"] / n,
                                              "far_cells_per_particle_equiv": cnt["far_cells"] / n,
                                              "supergroup_far_cells_per_particle_equiv":
                                                  cnt.get("sg_far_cells", 0) / n},
                "walk_ms": walk_ms}
    try:
        with open(os.path.join(ROOT, "profiles", "walk_traffic.json")) as f:
            tr = json.load(f)
        roofline["traffic"] = tr["dram_bytes_per_interaction"] * (cnt["cells"] + cnt["particles"])
        roofline["traffic_source"] = tr["source"]
    except (OSError, KeyError, ValueError):
        pass

    # ---- each phase alone (the step overlaps the walk with the SPH passes) ----
    phases_alone = phase_roofline(ctx, n, stream)

    # ---- accuracy at the common initial state (mixed vs FP64 oracle) ----
    err = {}
    ctx64 = None
    if not a.no_fp64:
        # the accuracy pair starts from the seeded sphere with a seeded
        # infall-plus-noise velocity field: at rest du/dt is identically zero
        # and the viscosity terms are idle, so the SPH error columns would
        # test nothing
        rng = np.random.default_rng(11)
        vel_chk = -0.3 * d["pos"] + 0.05 * rng.normal(size=d["pos"].shape)
        ctx64 = make("fp64", vel=vel_chk)
        sub = np.random.default_rng(7).choice(n, min(a.err_subset, n), replace=False)
        # both prologues ran on the same state; compare in original order
        ctx_m = make("mixed", vel=vel_chk)
        ids64 = ctx64.ids()
        inv = np.empty(n, np.int64)
        inv[ids64] = np.arange(n)
        tg = inv[sub].astype(np.int32)                       # storage indices in ctx64
        ad, _ = ctx64.gravity_direct(tg)                     # FP64 direct sum
        ag_m = ctx_m.get_acc("grav")[sub]
        ag_64 = ctx64.get_acc("grav")[sub]
        as_m = ctx_m.get_acc("sph")[sub]
        as_64 = ctx64.get_acc("sph")[sub]
        err = {"grav_mixed_vs_direct_fp64": rms_rel(ag_m, ad),
               "grav_fp64tree_vs_direct_fp64": rms_rel(ag_64, ad),
               "sph_mixed_vs_fp64": rms_rel(as_m, as_64),
               "total_mixed_vs_fp64_oracle": rms_rel(ag_m + as_m, ad + as_64),
               "rho_mixed_vs_fp64": float(np.max(np.abs(ctx_m.get("rho")[sub] / ctx64.get("rho")[sub] - 1))),
               "dudt_mixed_vs_fp64": float(np.sqrt(np.mean((ctx_m.get("dudt")[sub] - ctx64.get("dudt")[sub]) ** 2)) /
                                           np.sqrt(np.mean(ctx64.get("dudt")[sub] ** 2))),
               "subset": len(sub), "definition": "RMS over the subset of |a-a_ref|/|a_ref|",
               "state": "seeded sphere, v = -0.3 r + N(0, 0.05) (seed 11); the prologue's a and du/dt"}
        if a.rebuild_every > 1:
            # the walk on a refitted tree: the mixed context after the steps
            # that keep the last sort's topology, against the FP64 direct sum
            # on its own positions
            ctx_m.step(a.rebuild_every - 1)
            ctx_m.gravity()
            inv_m = np.empty(n, np.int64)
            inv_m[ctx_m.ids()] = np.arange(n)
            tg_m = inv_m[sub].astype(np.int32)
            ad_m, _ = ctx_m.gravity_direct(tg_m)
            err["grav_mixed_vs_direct_fp64_refit_tree"] = rms_rel(ctx_m.get_acc("grav", True)[tg_m], ad_m)
            err["refit_steps_before_that_check"] = a.rebuild_every - 1
        ctx_m.close()
        ctx64.close()
        ctx64 = make("fp64", L.FLAG_TIMING)
        ms64 = timed_steps(ctx64, max(2, a.steps // 2), a.warmup)
        k64 = max(2, a.steps // 2)
        fp64 = {"value": world * n * k64 / (ms64 * 1e-3), "ms_per_step": ms64 / k64, "steps": k64,
                "phases_ms": ctx64.phase_times(), "walk": walk_kw(a, "fp64")}
        ctx64.close()
        # the same step in mixed precision with the FP64 arm's walk (theta
        # alone, no expansions, super-groups or small-cell angle): the
        # precision's own gain, algorithm for algorithm
        ctx_s = make("mixed", L.FLAG_TIMING, walk=walk_kw(a, "fp64"))
        ms_s = timed_steps(ctx_s, k64, a.warmup)
        same_walk = {"value": world * n * k64 / (ms_s * 1e-3), "ms_per_step": ms_s / k64,
                     "steps": k64, "phases_ms": ctx_s.phase_times(), "walk": walk_kw(a, "fp64")}
        ctx_s.close()
    else:
        fp64 = same_walk = None

    # ---- opening angles theta in {0.4, 0.5, 0.7} at N = 1M: both precisions
    # with the plain walk, time per step and gravity error against the FP64
    # direct sum on the seeded subset ----
    theta_rows = []
    if not a.no_fp64 and not a.no_theta_table:
        sub = np.random.default_rng(7).choice(n, min(a.err_subset, n), replace=False)
        ref = make("fp64")
        inv = np.empty(n, np.int64)
        inv[ref.ids()] = np.arange(n)
        ad, _ = ref.gravity_direct(inv[sub].astype(np.int32))
        ref.close()
        kt = max(2, a.steps // 5)
        for th in (0.4, 0.5, 0.7):
            row = {"theta": th}
            for prec in ("mixed", "fp64"):
                c = make(prec, walk=dict(theta=th))
                row[f"grav_err_{prec}"] = rms_rel(c.get_acc("grav")[sub], ad)
                msx = timed_steps(c, kt, max(2, a.warmup // 2))
                row[f"ms_per_step_{prec}"] = msx / kt
                row[f"value_{prec}"] = world * n * kt / (msx * 1e-3)
                c.close()
            row["mixed_over_fp64"] = row["value_mixed"] / row["value_fp64"]
            theta_rows.append(row)

    # ---- the 64-cloud ensemble (log-uniform 20k-500k particles per cloud),
    # one launch per phase over every cloud ----
    ens = None
    if not a.no_ensemble:
        ens = ensemble_run(a, stream, timed_steps)

    # ---- the cooling cloud (N = 2M) and the large Evrard run (N = 16M,
    # learned cooling, 50 steps beside the FP64 plain path) ----
    cool = large = None
    if not a.no_cooling:
        cool = cooling_run(a, stream, timed_steps)
    if not a.no_large:
        from types import SimpleNamespace
        big = SimpleNamespace(**{**vars(a), "steps": a.large_steps, "warmup": 3})
        large = large_evrard(big, stream, timed_steps)

    # ---- energy and momentum drift over 100 steps, N = 10,000 Evrard (the
    # plain FP64 method's own configuration: theta 0.5, Courant 0.25) ----
    conservation = {}
    if not a.no_fp64:
        n0 = 10_000
        d0 = ic.evrard(n0, seed=42)
        for prec in ("fp64", "mixed"):
            c0 = Context(Config(n_max=n0, precision=prec, theta=0.5, leaf_size=a.leaf,
                                ngb_lanes=a.lanes, flags=L.FLAG_POTENTIAL))
            c0.set_stream(stream.cuda_stream)
            c0.load(d0["pos"], d0["vel"], d0["m"], d0["h"], d0["u"])
            c0.prologue()
            e0 = c0.energies()
            c0.step(100)
            c0.sync()
            e1 = c0.energies()
            E0 = e0["KE"] + e0["U"] + e0["PE"]
            E1 = e1["KE"] + e1["U"] + e1["PE"]
            v = np.stack([c0.get("vx"), c0.get("vy"), c0.get("vz")], 1)
            pscale = float(np.sum(d0["m"] * np.linalg.norm(v, axis=1)))
            p1 = float(np.linalg.norm([e1["px"], e1["py"], e1["pz"]]))
            conservation[prec] = {"E0": E0, "E100": E1, "rel_energy_drift": abs(E1 - E0) / abs(E0),
                                  "momentum_100": p1, "momentum_rel": p1 / pscale if pscale > 0 else None,
                                  "KE100": e1["KE"], "status": c0.status()}
            c0.close()
        conservation["definition"] = ("E = KE + U + PE (PE from the tree walk's potential), "
                                      "drift |E100 - E0| / |E0|; momentum |sum m v| after 100 steps, "
                                      "relative to sum m |v|")

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e = None
    if not a.no_e2e:
        fields = ["x", "y", "z", "vx", "vy", "vz", "u", "h"]
        pinned = {f: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for f in fields}
        for f in fields:
            pinned[f][:] = ctx.get(f)
        ctx.step_io(pinned, pinned)   # first call: staging buffer and copy stream
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            ctx.step_io(pinned, pinned)
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(time.perf_counter() - t0)
        # the same loop through the three separate calls, for comparison
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            ctx.set_fields(pinned)
            ctx.step(1)
            ctx.get_fields(fields, out=pinned)
        torch.cuda.synchronize()
        t_sep = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": world * n * a.steps / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": 8 * n * len(fields), "d2h_bytes_per_step": 8 * n * len(fields),
               "api": "sph_step_io per step: 8 fields copied in from pinned host memory, one step, "
                      "the same 8 fields copied back into it (each as soon as the step has "
                      "written it, beside the rest of the step)",
               "separate_calls": {"value": world * n * a.steps / t_sep,
                                  "api": "sph_set_fields + sph_step + sph_get_fields per step"}}

    # ---- CPU baseline (rank 0, one GPU only) ----
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        step_s, info = cpu_reference_sample(n, 64)
        cpu = {"value": n / step_s, "unit": UNIT, "cores": info["threads"], "kind": "port",
               "sample": (f"{info['rows']} rows x {n} sources per phase (6 phases of the reference "
                          f"CPU step), extrapolated x{n / info['rows']:.0f}; {info['sample_s']} s "
                          "of CPU work"),
               "phase_s_extrapolated": info["phase_s"]}

    final_status = ctx.status()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64 (mixed)",
        "data": "synthetic (seeded Evrard sphere, numpy default_rng)",
        "config": {"workload": "evrard_1M_mixed" if n == 1_000_000 else f"evrard_{n}_mixed",
                   "n": n, "theta_mixed": a.theta, "theta_fp64": a.theta_fp64,
                   "theta_local_mixed": a.theta_local, "theta_small_mixed": a.theta_small,
                   "small_cell_mixed": a.small_cell,
                   "leaf_size": a.leaf, "ngb_lanes": a.lanes,
                   "n_ngb": 64, "eps": 1e-2, "av": "monaghan-gingold alpha=1 beta=2",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "working set > L2 (neighbour rows ~0.3 GB + tree ~0.5 GB per step)",
                   "graph": "CUDA graph per step",
                   "rebuild_every": a.rebuild_every,
                   "kept_candidate_rows": not a.no_row_reuse},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches_timed,
        "clocks": clocks,
        "fp64_plain": fp64,
        "mixed_same_walk": same_walk,
        "mixed_over_fp64": (same_walk["value"] / fp64["value"]) if fp64 else None,
        "mixed_over_fp64_definition": ("same algorithm: the mixed step with the FP64 arm's "
                                       "walk settings over the FP64 plain step"),
        "mixed_over_fp64_tuned_walk": (value / fp64["value"]) if fp64 else None,
        "theta_table_1M": theta_rows,
        "ensemble": ens,
        "cooling_cloud_2M": cool,
        "large_16M": large,
        "accel_err": err,
        "conservation_100_steps_n10k": conservation,
        "phases_ms": phases,
        "phases_alone": phases_alone,
        "status": final_status,
        "device_gb": ctx.device_bytes() / 1e9,
    }
    ctx.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def ensemble_run(a, stream, timed, rank=0, world=1):
    """The batched ensemble of a.clouds independent Evrard spheres (counts
    log-uniform in [20k, 500k], mass, radius and u0 jittered by 20 %), each
    with its own tree and time step, all advanced by the same launches;
    clouds sharded over the ranks by LPT when world > 1."""
    from sph_2_b200 import Config, Context, ic
    from sph_2_b200.distributed import local_ensemble, shard_clouds
    e = ic.ensemble(n_clouds=a.clouds, seed=42)
    owner = shard_clouds(e["counts"], world)
    mine = local_ensemble(e, owner, rank)
    n = len(mine["m"])
    ctx = Context(Config(n_max=n, n_cloud_max=len(mine["counts"]), precision="mixed",
                         leaf_size=a.leaf, ngb_lanes=a.lanes, rebuild_every=a.rebuild_every,
                         **walk_kw(a, "mixed")))
    ctx.set_stream(stream.cuda_stream)
    ctx.load(mine["pos"], mine["vel"], mine["m"], mine["h"], mine["u"], cloud=mine["cloud"])
    ctx.prologue()
    tuned = None
    if not a.no_tune:
        from sph_2_b200.autotune import tune
        best, res = tune(ctx, use_cache=False)
        tuned = {"choice": best, "candidates_ms_per_step": [[ms, p] for ms, p in res]}
    k = max(2, a.steps // 4)
    ms = timed(ctx, k, a.warmup)
    total = int(e["counts"].sum())
    out = {"value": total * k / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / k, "steps": k,
           "workload": f"ensemble_{a.clouds}_clouds", "particles": total, "clouds": a.clouds,
           "per_rank_particles": n, "status": ctx.status(), "tuned": tuned,
           "launch_params": {"ngb_lanes": ctx.config.ngb_lanes, "block_size": ctx.config.block_size,
                             "leaf_size": ctx.config.leaf_size}}
    ctx.close()
    return out


def large_evrard(a, stream, timed):
    """Evrard collapse at N = 16M (default) in mixed precision with the learned
    cooling path, beside the plain FP64 method with the exact solve on the same
    GPU: throughput, device memory, per-phase times and roofline fractions,
    and energy / momentum after the warm-up and timed steps of both."""
    from sph_2_b200 import Config, Context, cooling, ic
    from sph_2_b200 import _lib as L
    n = a.n if a.n != 1_000_000 else 16_000_000
    d = ic.evrard(n, seed=42)
    # physical scale: a 100 cm^-3 mean-density sphere whose u = 0.05 is 1e6 K
    # (mu = 1.22): the gas cools through the table's 1e5 K peak towards the
    # 1e4 K cut-off while it falls in
    kb, mh, gcgs, mu, gam = 1.380649e-16, 1.6726e-24, 6.674e-8, 1.22, 5.0 / 3.0
    unit_u = kb * 1e6 / ((gam - 1.0) * mu * mh) / 0.05
    rho_mean = 100.0 * mu * mh
    R = (3.0 * unit_u / gcgs / (4.0 * np.pi * rho_mean)) ** 0.5
    M = unit_u * R / gcgs
    units = {"unit_rho": M / R ** 3, "unit_u": unit_u, "unit_t": (R ** 3 / (gcgs * M)) ** 0.5}
    res = {}
    for arm, prec, mlp in (("mixed_mlp", "mixed", True), ("fp64_exact", "fp64", False)):
        flags = L.FLAG_COOLING | L.FLAG_TIMING | L.FLAG_POTENTIAL | (L.FLAG_COOLING_MLP if mlp else 0)
        ctx = Context(Config(n_max=n, precision=prec, leaf_size=a.leaf, ngb_lanes=a.lanes,
                             flags=flags, rebuild_every=a.rebuild_every, **walk_kw(a, prec)))
        ctx.set_stream(stream.cuda_stream)
        cooling.setup(ctx, units)
        if mlp:
            Xn, yn, norm, _ = cooling.training_set(
                ctx, n=5_000_000, seed=7,
                ranges=dict(log_rho=(-23.0, -17.0), log_T=(1.5, 6.5), log_dt=(9.5, 13.5)))
            ctx.mlp_set(cooling.init_params(seed=0), norm)
            cooling.train(ctx, Xn, yn, steps=4000, batch=4096, lr=2e-3)
        ctx.load(d["pos"], d["vel"], d["m"], d["h"], d["u"])
        ctx.prologue()
        e0 = ctx.energies()
        ms = timed(ctx, a.steps, a.warmup)
        e1 = ctx.energies()
        row = {"value": n * a.steps / (ms * 1e-3), "ms_per_step": ms / a.steps,
               "device_gb": ctx.device_bytes() / 1e9, "phases_ms": ctx.phase_times(),
               "E_start": e0["KE"] + e0["U"] + e0["PE"], "E_end": e1["KE"] + e1["U"] + e1["PE"],
               "p_end": float(np.linalg.norm([e1["px"], e1["py"], e1["pz"]])),
               "status": ctx.status()}
        if mlp:
            row["phases_alone"] = phase_roofline(ctx, n, stream)
        res[arm] = row
        ctx.close()
    mx, fp = res["mixed_mlp"], res["fp64_exact"]
    return {"value": mx["value"], "ms_per_step": mx["ms_per_step"],
            "config": {"workload": f"evrard_{n}_mixed_mlp_cooling", "n": n, "theta": a.theta,
                       "units_cgs": units, "steps_advanced": a.warmup + a.steps},
            "memory": {"device_gb_mixed": mx["device_gb"], "device_gb_fp64": fp["device_gb"],
                       "neighbour_rows_gb": 4 * 256 * n / 1e9,
                       "candidate_rows_gb": 4 * 256 * n / 1e9},
            "mixed_over_fp64": mx["value"] / fp["value"],
            "energy_vs_fp64": abs(mx["E_end"] - fp["E_end"]) / abs(fp["E_end"]),
            "momentum_end": {"mixed": mx["p_end"], "fp64": fp["p_end"]},
            "arms": res}


def cooling_run(a, stream, timed, n=2_000_000):
    """The cooling cloud collapse: N = 2M uniform sphere at n = 100 cm^-3, T =
    1e4 K, Mach 2 turbulence (k^-4), the synthetic 128-bin Lambda(T) table;
    the step with the exact implicit solve, then with the MLP surrogate
    (trained on the GPU on 5M exact-solver samples) and its exact fallback.
    The cooling phase is the u update + cooling solve + dt commit of a step."""
    from sph_2_b200 import Config, Context, cooling, ic
    from sph_2_b200 import _lib as L
    d = ic.cooling_cloud(n, seed=42)
    res = {}
    for mode in ("exact", "mlp"):
        flags = L.FLAG_COOLING | (L.FLAG_COOLING_MLP if mode == "mlp" else 0) | L.FLAG_TIMING
        ctx = Context(Config(n_max=n, precision="mixed", leaf_size=a.leaf, flags=flags,
                             rebuild_every=a.rebuild_every, **walk_kw(a, "mixed")))
        ctx.set_stream(stream.cuda_stream)
        cooling.setup(ctx, d["units"])
        if mode == "mlp":
            Xn, yn, norm, _ = cooling.training_set(ctx, n=5_000_000, seed=7)
            ctx.mlp_set(cooling.init_params(seed=0), norm)
            cooling.train(ctx, Xn, yn, steps=4000, batch=4096, lr=2e-3)
        ctx.load(d["pos"], d["vel"], d["m"], d["h"], d["u"])
        ctx.prologue()
        k = max(2, a.steps // 2)
        ms = timed(ctx, k, a.warmup)
        ph = ctx.phase_times()
        res[mode] = {"value": n * k / (ms * 1e-3), "ms_per_step": ms / k, "steps": k,
                     "cooling_phase_ms": ph["update_dt"], "status": ctx.status()}
        ctx.close()
    return {"value": res["mlp"]["value"], "ms_per_step": res["mlp"]["ms_per_step"],
            "config": {"workload": f"cooling_cloud_{n}", "n": n, "theta": a.theta, "mach": 2,
                       "n_cgs": 100, "T": 1e4, "training_samples": 5_000_000,
                       "cooling_phase": "u update + cooling solve + dt commit of the last step",
                       "mlp_inference": "tcgen05.mma, TMEM accumulator, 128-row tiles"},
            "exact": res["exact"], "mlp": res["mlp"],
            "cooling_phase_mlp_over_exact": res["mlp"]["cooling_phase_ms"] /
            res["exact"]["cooling_phase_ms"]}


def extra_workload(a, world, rank, local):
    """The batched 64-cloud ensemble (clouds sharded over the ranks) or the
    2M-particle turbulent cooling cloud (exact implicit cooling vs the MLP
    surrogate path).  Same timing rules as the headline line."""
    import torch
    import torch.distributed as dist
    from sph_2_b200 import Config, Context, cooling, ic
    from sph_2_b200 import _lib as L

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    stream = torch.cuda.Stream(priority=-10)

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(ctx, steps, warmup):
        ctx.step(warmup)
        ctx.sync()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record()
            ctx.step(steps)
            e1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    out = {"metric": METRIC, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "fp32+fp64 (mixed)", "data": "synthetic"}
    if a.workload == "ensemble":
        r = ensemble_run(a, stream, timed, rank, world)
        out.update(value=r["value"], ms_per_step=r["ms_per_step"],
                   config={"workload": r["workload"], "particles": r["particles"],
                           "clouds": a.clouds, "theta": a.theta,
                           "parallelism": f"clouds sharded over {world} ranks (LPT)",
                           "per_rank_particles": r["per_rank_particles"]},
                   status=r["status"], tuned=r["tuned"], launch_params=r["launch_params"])
    elif a.workload == "large":
        out.update(large_evrard(a, stream, timed))
    else:
        out.update(cooling_run(a, stream, timed, a.n if a.n != 1_000_000 else 2_000_000))
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
