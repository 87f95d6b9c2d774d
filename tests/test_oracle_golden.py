"""The CPU oracle against golden vectors from the reference's own code.

The fixtures in tests/golden/ were produced by running the reference's numba
functions (MPI_sph/sph_code/libsx.py, shear.py) and its compiled cooling solver
(GPU_sph/With_cooling/Model_C/myPhotoLibsGPU.h); see make_golden.py.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

G = os.path.join(os.path.dirname(__file__), "golden")
GAMA, ALPHA, BETA, ETA = 5.0 / 3.0, 1.0, 2.0, 0.1


def load(name):
    return dict(np.load(os.path.join(G, name)))


def close(a, b, rtol=1e-11):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = np.max(np.abs(b)) + 1e-300
    assert np.max(np.abs(a - b)) <= rtol * scale, np.max(np.abs(a - b)) / scale


@pytest.fixture(scope="module", params=["ref_sph_evrard_n600.npz", "ref_sph_ragged_n64.npz"])
def case(request):
    return load(request.param)


def test_smoothing_length(case):
    n = len(case["m"])
    close(O.ref_smoothing_length(0, n, case["pos"]), case["h0"], 1e-14)


def test_h_smooth_fast(case):
    n = len(case["m"])
    close(O.ref_h_smooth_fast(0, n, case["pos"], case["h0"]), case["h"], 1e-13)


def test_density(case):
    n = len(case["m"])
    close(O.ref_getDensity(0, n, case["pos"], case["m"], case["h"]), case["rho"])
    # row split = the reference's MPI decomposition (sph_mpi4_v4.py:57-65)
    a = O.ref_getDensity(0, n // 3, case["pos"], case["m"], case["h"])
    b = O.ref_getDensity(n // 3, n, case["pos"], case["m"], case["h"])
    close(np.concatenate([a, b]), case["rho"])


def test_div_curl(case):
    n = len(case["m"])
    d, c = O.ref_div_curlVel(0, n, case["pos"], case["v"], case["rho"], case["m"], case["h"])
    close(d, case["divV"])
    close(c, case["curlV"])


@pytest.mark.parametrize("mode,bal,ka,kd", [(1, 1, "acc_shear", "du_shear"), (0, 0, "acc_mg", "du_mg")])
def test_forces(case, mode, bal, ka, kd):
    n = len(case["m"])
    args = (case["pos"], case["v"], case["rho"], case["P"], case["c"], case["h"], case["m"],
            case["divV"], case["curlV"], ALPHA, BETA, ETA, mode, bal)
    close(O.ref_getAcc_sph(0, n, *args), case[ka])
    close(O.ref_get_dU(0, n, *args), case[kd])


def test_gravity_and_energies(case):
    n = len(case["m"])
    close(O.ref_getKE(case["v"], case["m"]), case["ke"])
    if int(case["grav_raises"]):
        # coincident particles: the reference raises ZeroDivisionError; the
        # project's Plummer direct sum stays finite there
        acc, pot = O.grav_direct(*case["pos"].T.copy(), case["m"], 1.0, 1e-2, np.arange(n))
        assert np.isfinite(acc).all() and np.isfinite(pot).all()
        return
    close(O.ref_getAcc_g_smth_mimj(0, n, case["pos"], case["m"], 1.0, case["eps"]), case["acc_g"])
    close(O.ref_getAcc_g_smth_mimj(0, n // 2, case["pos"], case["m"], 1.0, case["eps"]),
          case["acc_g_half"])
    close(O.ref_getPE(case["pos"], case["m"], 1.0, case["eps"]), case["pe"])


def test_reference_step_sequence():
    """Two steps of sph_mpi4_v4.py:278-416 restated with the oracle."""
    c = load("ref_sph_evrard_n600.npz")
    n, m, eps, dt = len(c["m"]), c["m"], c["eps"], 0.001
    r, v, u, h = c["pos"].copy(), np.zeros((n, 3)), np.full(n, 0.05), c["h"].copy()

    def forces(r, v, u, h):
        rho = O.ref_getDensity(0, n, r, m, h)
        ag = O.ref_getAcc_g_smth_mimj(0, n, r, m, 1.0, eps)
        P, cs = O.ref_pressure(rho, u, GAMA), O.ref_sound_speed(u, GAMA)
        dv, cv = O.ref_div_curlVel(0, n, r, v, rho, m, h)
        a = ag + O.ref_getAcc_sph(0, n, r, v, rho, P, cs, h, m, dv, cv, ALPHA)
        return rho, P, cs, dv, cv, a

    rho, P, cs, dv, cv, acc = forces(r, v, u, h)
    ut = O.ref_get_dU(0, n, r, v, rho, P, cs, h, m, dv, cv, ALPHA)
    u = u + ut * dt
    u_prev, ut_prev = u.copy(), ut.copy()
    for _ in range(2):
        v = v + acc * dt / 2
        r = r + v * dt
        h = O.ref_h_smooth_fast(0, n, r, h)
        rho, P, cs, dv, cv, acc = forces(r, v, u, h)
        v = v + acc * dt / 2
        ut = O.ref_get_dU(0, n, r, v, rho, P, cs, h, m, dv, cv, ALPHA)
        u = u_prev + 0.5 * dt * (ut + ut_prev)
        u_prev, ut_prev = u.copy(), ut.copy()
    for k, a in [("step_r", r), ("step_v", v), ("step_u", u), ("step_h", h), ("step_rho", rho),
                 ("step_acc", acc)]:
        close(a, c[k], 1e-9)


def test_list_sums_equal_all_pairs(case):
    """The project's exact neighbour lists give the same sums as the
    reference's all-pairs loops (W = 0 outside q <= 2)."""
    x, y, z = (case["pos"][:, k].copy() for k in range(3))
    v = case["v"]
    off, lst = O.neighbours(x, y, z, case["h"])
    close(O.density_list(x, y, z, case["m"], case["h"], off, lst), case["rho"])
    d, c = O.divcurl_list(x, y, z, *v.T.copy(), case["rho"], case["m"], case["h"], off, lst)
    close(d, case["divV"], 1e-10)
    close(c, case["curlV"], 1e-10)
    for mode, bal, ka, kd in [(1, 1, "acc_shear", "du_shear"), (0, 0, "acc_mg", "du_mg")]:
        a, du, vs = O.force_list(x, y, z, *v.T.copy(), case["rho"], case["P"], case["c"],
                                 case["h"], case["m"], case["divV"], case["curlV"], ALPHA, BETA,
                                 ETA, mode, bal, off, lst)
        close(a, case[ka], 1e-10)
        close(du, case[kd], 1e-10)
        assert (vs >= 2 * case["c"] - 1e-12).all()


def test_docooling_structure_pinned():
    """FP32 restatement of DoCooling over the reference's own rate function
    reproduces the reference solver bit for bit."""
    if O.ref_cooling_lib() is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    g = load("ref_docooling_f32.npz")
    out = np.array([O.do_cooling_f32_with_ref_rate(float(a), float(b), float(c), float(g["XH"]))
                    for a, b, c in zip(g["rho"], g["u_old"], g["dt"])], np.float32)
    assert np.array_equal(out.view(np.uint32), g["u_new"].view(np.uint32))


def test_dt_individual_oracle_equals_all_pairs_form():
    """With every pair inside the lists (h large enough), the oracle's
    list-restricted individual step equals dt_array_indiv_dt's all-pairs form
    (hfvCLibs_v7_hfv_v2.h:999-1078, written out here in NumPy, FP64)."""
    rng = np.random.default_rng(4)
    n = 40
    pos = rng.random((n, 3))
    v = rng.normal(size=(n, 3))
    m = np.full(n, 1.0 / n)
    h = np.full(n, 2.0)                       # every |r_ij| <= h_i + h_j
    c = 0.2 + rng.random(n)
    asph, agrav = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    x, y, z = (pos[:, k].copy() for k in range(3))
    off, lst = O.neighbours(x, y, z, h)
    assert off[-1] == n * n
    rho = O.density_list(x, y, z, m, h, off, lst)
    eps, C, alpha = 1e-2, 0.25, 1.0
    dt, dh = O.dt_individual(x, y, z, v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy(), m, h, rho, c,
                             asph, agrav, eps, C, alpha, off, lst)
    d = pos[:, None, :] - pos[None, :, :]
    rr = np.sqrt(np.sum(d * d, axis=2))
    u = v[:, None, :] - v[None, :, :]
    vr = np.sum(u * d, axis=2)
    vsig = np.maximum(0.0, np.max(c[:, None] + c[None, :] - 3.0 * vr / (rr + 1e-5), axis=1))
    # signed divergence with the M4 kernel gradient at h_ij
    hij = 0.5 * (h[:, None] + h[None, :])
    q = rr / hij
    nW = np.where(q <= 1.0, (1 / np.pi) / hij ** 5 * (-3.0 + 2.25 * q),
                  np.where(q <= 2.0, -0.75 / np.pi / hij ** 5 * (2.0 - q) ** 2 / (q + 1e-20), 0.0))
    div = -np.sum(m[None, :] * nW * vr, axis=1) / rho
    at = np.linalg.norm(asph + agrav, axis=1)
    ag = np.linalg.norm(agrav, axis=1)
    va = np.linalg.norm(v, axis=1)
    est = np.stack([C * h / vsig, C * h / (h * np.abs(div) + np.maximum(c, va) * (1 + 0.6 * alpha)),
                    0.4 * np.sqrt(eps / at), 0.4 * eps / va, np.sqrt(h / ag), np.sqrt(h / at)], 1)
    assert np.allclose(dt, est.min(axis=1), rtol=1e-12, atol=0)
    assert np.allclose(dh, h * div / 3.0, rtol=1e-10, atol=1e-14)
