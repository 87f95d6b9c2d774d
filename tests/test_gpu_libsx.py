"""The reference-named drop-in functions (sph_2_b200.libsx) against the
numbers the reference's own numba functions produced on the same inputs
(tests/golden/ref_sph_evrard_n600.npz, written by tests/golden/make_golden.py
from MPI_sph/sph_code/libsx.py and shear.py)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from sph_2_b200 import libsx as X

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


@pytest.fixture(scope="module")
def g():
    X.precision("fp64")
    yield dict(np.load(os.path.join(GOLD, "ref_sph_evrard_n600.npz")))
    X.release()


def test_density_and_rows(g):
    n = len(g["m"])
    assert rel(X.getDensity_mpi(0, n, g["pos"], g["m"], g["h"]), g["rho"]) < 1e-12
    part = X.getDensity_mpi(100, 400, g["pos"], g["m"], g["h"])
    assert part.shape == (300,) and rel(part, g["rho"][100:400]) < 1e-12
    assert rel(X.getDensity(g["pos"], g["m"], g["h"]), g["rho"]) < 1e-12
    assert rel(X.getPressure(g["rho"], g["u"], 5.0 / 3.0), g["P"]) < 1e-15


def test_div_curl(g):
    n = len(g["m"])
    d, c = X.div_curlVel_mpi(0, n, g["pos"], g["v"], g["rho"], g["m"], g["h"])
    assert rel(d, g["divV"]) < 1e-11 and rel(c, g["curlV"]) < 1e-11


def test_viscosity_forms(g):
    n = len(g["m"])
    a = (g["pos"], g["v"], g["rho"], g["P"], g["c"], g["h"], g["m"])
    acc = X.getAcc_sph_shear_mpi(0, n, *a, g["divV"], g["curlV"], 1.0)
    assert acc.shape == (n, 3) and rel(acc, g["acc_shear"]) < 1e-11
    assert rel(X.get_dU_shear_mpi(0, n, *a, g["divV"], g["curlV"], 1.0), g["du_shear"]) < 1e-11
    acc = X.getAcc_sph_mpiXXX(0, n, *a, 5.0 / 3.0, 0.1, 1.0, 2.0)
    assert rel(acc, g["acc_mg"]) < 1e-11
    assert rel(X.get_dU_mpiXXXX(0, n, *a, 5.0 / 3.0, 0.1, 1.0, 2.0), g["du_mg"]) < 1e-11
    sub = X.getAcc_sph_mpiXXX(50, 70, *a, 5.0 / 3.0, 0.1, 1.0, 2.0)
    assert sub.shape == (20, 3) and rel(sub, g["acc_mg"][50:70]) < 1e-11
    # signal velocity without the switch (libsx.py:270) == the oracle's form
    acc = X.getAcc_sph_mpi(0, n, *a, 5.0 / 3.0, 0.1, 1.0, 2.0)
    ao = O.ref_getAcc_sph(0, n, *a, g["divV"], g["curlV"], 1.0, mode=1, balsara=0)
    assert rel(acc, ao) < 1e-11
    du = X.get_dU_mpi(0, n, *a, 5.0 / 3.0, 0.1, 1.0, 2.0)
    assert rel(du, O.ref_get_dU(0, n, *a, g["divV"], g["curlV"], 1.0, mode=1, balsara=0)) < 1e-11


def test_gravity_and_energies(g):
    n = len(g["m"])
    acc = X.getAcc_g_smth_mimj_mpi(0, n, g["pos"], g["m"], 1.0, g["eps"])
    assert rel(acc, g["acc_g"]) < 1e-12
    # the reference's partial field of a row range (its MPI decomposition),
    # and the sum over a partition of the rows is the whole field
    half = X.getAcc_g_smth_mimj_mpi(0, n // 2, g["pos"], g["m"], 1.0, g["eps"])
    assert rel(half, g["acc_g_half"]) < 1e-12
    rest = X.getAcc_g_smth_mimj_mpi(n // 2, n, g["pos"], g["m"], 1.0, g["eps"])
    assert rel(half + rest, g["acc_g"]) < 1e-12
    assert abs(X.getKE(g["v"], g["m"]) / float(g["ke"]) - 1) < 1e-13
    pe = X.getPE(g["pos"], g["m"], 1.0, np.full(n, 1e-2))
    x, y, z = (g["pos"][:, k].copy() for k in range(3))
    _, po = O.grav_direct(x, y, z, g["m"], 1.0, 1e-2, np.arange(n))
    assert abs(pe / (0.5 * np.sum(g["m"] * po)) - 1) < 1e-3    # tree potential vs direct


def test_smoothing_length(g):
    n = len(g["m"])
    # the reference's count iteration, from its own start: its output bit for bit
    h = X.h_smooth_fast_mpi(0, n, g["pos"], g["h0"])
    assert np.array_equal(h, g["h"])
    assert np.array_equal(X.h_smooth_fast_mpi(100, 300, g["pos"], g["h0"]), g["h"][100:300])
    # the project's Newton h under its own name
    hn = X.h_newton_mpi(0, n, g["pos"], g["h"], m=g["m"])
    x, y, z = (g["pos"][:, k].copy() for k in range(3))
    ho, _, bad = O.newton_h(x, y, z, g["m"], g["h"], n_ngb=50.0)
    assert bad == 0 and np.max(np.abs(hn / ho - 1)) < 2e-3
    # the reference's starting h: half the 50th-neighbour distance
    assert np.array_equal(X.smoothing_length_mpi(0, n, g["pos"]), g["h0"])
    assert np.array_equal(X.smoothing_length_mpi(17, 99, g["pos"]), g["h0"][17:99])


def test_torch_cuda_tensors(g):
    torch = pytest.importorskip("torch")
    n = len(g["m"])
    tp, tm, th = (torch.tensor(g[k], device="cuda") for k in ("pos", "m", "h"))
    rho = X.getDensity_mpi(0, n, tp, tm, th)
    assert rho.is_cuda and rel(rho.cpu().numpy(), g["rho"]) < 1e-12
    tv, tr, tP, tc, td, tcu = (torch.tensor(g[k], device="cuda")
                               for k in ("v", "rho", "P", "c", "divV", "curlV"))
    acc = X.getAcc_sph_shear_mpi(0, n, tp, tv, tr, tP, tc, th, tm, td, tcu, 1.0)
    assert acc.is_cuda and acc.shape == (n, 3) and rel(acc.cpu().numpy(), g["acc_shear"]) < 1e-11
