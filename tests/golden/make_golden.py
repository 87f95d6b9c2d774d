"""Generate golden vectors by running the reference's own CPU implementation.

Run here (where the reference tree is mounted), never on the GPU box:

    python tests/golden/make_golden.py

It imports the reference's numba functions from
``11_Dec_2022/MPI_sph/sph_code/{libsx,shear}.py`` and calls them on seeded
inputs, and it calls the reference's compiled implicit cooling solver
(``oracle/_ref/libphcool.so``, built from
``GPU_sph/With_cooling/Model_C/myPhotoLibsGPU.h`` by ``oracle/Makefile``).
The outputs are committed as small ``.npz`` fixtures next to this script.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's 11_Dec_2022 directory ($SPH2_REFERENCE, else its place here)
REF = os.path.join(os.environ.get("SPH2_REFERENCE", "/root/reference/11_Dec_2022"),
                   "MPI_sph", "sph_code")


def evrard_positions(n, seed):
    """Seeded uniform ball stretched r -> r^{3/2} (rho ~ 1/r)."""
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.random(n))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    return d * r[:, None], rng


def sph_case(n, seed, duplicate=False):
    sys.path.insert(0, REF)
    import libsx  # noqa: E402  (the reference module)
    import shear  # noqa: E402

    pos, rng = evrard_positions(n, seed)
    if duplicate:
        pos[1] = pos[0]          # two particles at the same place
        pos[3, 0] = pos[2, 0]    # equal x only
    v = rng.normal(scale=0.1, size=(n, 3))
    m = np.full(n, 1.0 / n) * (1.0 + 0.2 * rng.random(n))
    u = 0.05 * (1.0 + 0.5 * rng.random(n))
    eps = np.full(n, 0.1)
    gama, alpha, beta, eta, G = 5.0 / 3.0, 1.0, 2.0, 0.1, 1.0

    h0 = libsx.smoothing_length_mpi(0, n, pos)
    h = libsx.h_smooth_fast_mpi(0, n, pos, h0)
    rho = libsx.getDensity_mpi(0, n, pos, m, h)
    P = libsx.getPressure(rho, u, gama)
    c = np.sqrt(gama * (gama - 1.0) * u)
    divV, curlV = shear.div_curlVel_mpi(0, n, pos, v, rho, m, h)
    acc_shear = shear.getAcc_sph_shear_mpi(0, n, pos, v, rho, P, c, h, m, divV, curlV, alpha)
    du_shear = shear.get_dU_shear_mpi(0, n, pos, v, rho, P, c, h, m, divV, curlV, alpha)
    acc_mg = libsx.getAcc_sph_mpiXXX(0, n, pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
    du_mg = libsx.get_dU_mpiXXXX(0, n, pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
    # the reference's spline gravity divides by r^3 before the softening test
    # (libsx.py:922), so coincident particles raise ZeroDivisionError there
    try:
        acc_g = libsx.getAcc_g_smth_mimj_mpi(0, n, pos, m, G, eps)
        acc_g_half = libsx.getAcc_g_smth_mimj_mpi(0, n // 2, pos, m, G, eps)
        pe = libsx.getPE(pos, m, G, eps)
        grav_raises = 0
    except ZeroDivisionError:
        acc_g = acc_g_half = np.full((n, 3), np.nan)
        pe = np.nan
        grav_raises = 1
    ke = libsx.getKE(v, m)
    if grav_raises:
        return dict(pos=pos, v=v, m=m, u=u, eps=eps, h0=h0, h=h, rho=rho, P=P, c=c, divV=divV,
                    curlV=curlV, acc_shear=acc_shear, du_shear=du_shear, acc_mg=acc_mg,
                    du_mg=du_mg, ke=ke, grav_raises=grav_raises)

    # two steps of the reference loop, sph_mpi4_v4.py:278-416, same call order
    dt = 0.001
    r = pos.copy()
    vv = np.zeros_like(r)
    uu = np.full(n, 0.05)
    hh = h.copy()
    rho_s = libsx.getDensity_mpi(0, n, r, m, hh)
    acc = libsx.getAcc_g_smth_mimj_mpi(0, n, r, m, G, eps)
    P_s = libsx.getPressure(rho_s, uu, gama)
    c_s = np.sqrt(gama * (gama - 1.0) * uu)
    dv, cv = shear.div_curlVel_mpi(0, n, r, vv, rho_s, m, hh)
    acc = acc + shear.getAcc_sph_shear_mpi(0, n, r, vv, rho_s, P_s, c_s, hh, m, dv, cv, alpha)
    ut = shear.get_dU_shear_mpi(0, n, r, vv, rho_s, P_s, c_s, hh, m, dv, cv, alpha)
    uu = uu + ut * dt
    u_prev, ut_prev = uu.copy(), ut.copy()
    for _ in range(2):
        vv = vv + acc * dt / 2.0
        r = r + vv * dt
        hh = libsx.h_smooth_fast_mpi(0, n, r, hh)
        rho_s = libsx.getDensity_mpi(0, n, r, m, hh)
        acc_g_s = libsx.getAcc_g_smth_mimj_mpi(0, n, r, m, G, eps)
        P_s = libsx.getPressure(rho_s, uu, gama)
        c_s = np.sqrt(gama * (gama - 1.0) * uu)
        dv, cv = shear.div_curlVel_mpi(0, n, r, vv, rho_s, m, hh)
        acc = acc_g_s + shear.getAcc_sph_shear_mpi(0, n, r, vv, rho_s, P_s, c_s, hh, m, dv, cv, alpha)
        vv = vv + acc * dt / 2.0
        ut = shear.get_dU_shear_mpi(0, n, r, vv, rho_s, P_s, c_s, hh, m, dv, cv, alpha)
        uu = u_prev + 0.5 * dt * (ut + ut_prev)
        u_prev, ut_prev = uu.copy(), ut.copy()

    return dict(pos=pos, v=v, m=m, u=u, eps=eps, h0=h0, h=h, rho=rho, P=P, c=c, divV=divV,
                curlV=curlV, acc_shear=acc_shear, du_shear=du_shear, acc_mg=acc_mg, du_mg=du_mg,
                acc_g=acc_g, acc_g_half=acc_g_half, ke=ke, pe=pe, grav_raises=grav_raises,
                step_r=r, step_v=vv, step_u=uu, step_h=hh, step_rho=rho_s, step_acc=acc)


def cooling_case(n, seed):
    sys.path.insert(0, os.path.join(HERE, "..", ".."))
    from oracle import oracle as O

    R = O.ref_cooling_lib()
    if R is None:
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    rng = np.random.default_rng(seed)
    rho = (10.0 ** rng.uniform(-24, -21, n)).astype(np.float32)
    u = (10.0 ** rng.uniform(11.5, 13.5, n)).astype(np.float32)
    dt = (10.0 ** rng.uniform(9, 13, n)).astype(np.float32)
    XH = np.float32(0.7)
    out = np.array([R.ref_DoCooling(float(a), float(b), float(c), float(XH))
                    for a, b, c in zip(rho, u, dt)], np.float32)
    return dict(rho=rho, u_old=u, dt=dt, XH=np.float32(XH), u_new=out)


def main():
    np.savez_compressed(os.path.join(HERE, "ref_sph_evrard_n600.npz"), **sph_case(600, 42))
    np.savez_compressed(os.path.join(HERE, "ref_sph_ragged_n64.npz"), **sph_case(64, 7, duplicate=True))
    np.savez_compressed(os.path.join(HERE, "ref_docooling_f32.npz"), **cooling_case(256, 11))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
