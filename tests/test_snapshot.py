"""The reference's binary IC / snapshot layouts and params.txt, on the host.

Byte layouts are built independently with `struct` in the order the
reference's own readers use (readVectorsFromFile, hfvCLibs_v7_hfv_v2.h:59-101;
singlex_gpu_data.py:55-72) and compared with this package's writers and
readers.  sph_ic_count is the library's own header check and needs no GPU.
"""
import ctypes as C
import struct

import numpy as np
import pytest

from sph_2_b200 import snapshot as S
from sph_2_b200 import _lib as L


def _cols(n, seed=0):
    rng = np.random.default_rng(seed)
    return {k: rng.normal(size=n).astype(np.float32) for k in S.IC_FIELDS}


def test_ic_layout_matches_reference_reader(tmp_path):
    n = 7
    c = _cols(n)
    p = tmp_path / "ic.bin"
    S.write_ic(p, c["x"], c["y"], c["z"], c["vx"], c["vy"], c["vz"], c["u"], c["h"], c["mass"],
               eps=c["eps"])
    want = struct.pack("<i", n) + struct.pack(f"<{n}i", *([0] * n))
    for k in ("x", "y", "z", "vx", "vy", "vz", "u", "h", "eps", "mass"):
        want += struct.pack(f"<{n}f", *c[k].tolist())
    assert p.read_bytes() == want
    r = S.read_ic(p)
    assert r["N"] == n and (r["Typ"] == 0).all()
    for k in S.IC_FIELDS:
        assert np.array_equal(r[k], c[k])


def test_ic_eps_defaults_to_h(tmp_path):
    c = _cols(5, 1)
    p = tmp_path / "ic.bin"
    S.write_ic(p, c["x"], c["y"], c["z"], c["vx"], c["vy"], c["vz"], c["u"], c["h"], c["mass"])
    assert np.array_equal(S.read_ic(p)["eps"], c["h"])


def test_snapshot_reader_on_reference_layout(tmp_path):
    n, nion = 4, 6
    rng = np.random.default_rng(3)
    cols = {k: rng.normal(size=n).astype(np.float32) for k in S.SNAP_FIELDS}
    ion = rng.random(nion).astype(np.float32)
    dbg = np.arange(n, dtype=np.int32) + 60
    raw = struct.pack("<ii", n, nion) + struct.pack(f"<{n}i", *([0] * n))
    for k in ("x", "y", "z", "vx", "vy", "vz", "rho", "h", "u", "mass"):
        raw += struct.pack(f"<{n}f", *cols[k].tolist())
    raw += struct.pack(f"<{nion}f", *ion.tolist()) + struct.pack(f"<{n}i", *dbg.tolist())
    p = tmp_path / "G-0.1.bin"
    p.write_bytes(raw)
    r = S.read_snapshot(p)
    assert r["N"] == n and r["N_ionFrac"] == nion
    for k in S.SNAP_FIELDS:
        assert np.array_equal(r[k], cols[k])
    assert np.array_equal(r["ionFrac"], ion) and np.array_equal(r["debug"], dbg)
    p.write_bytes(raw[:-1])
    with pytest.raises(ValueError):
        S.read_snapshot(p)


def test_params_round_trip(tmp_path):
    p = tmp_path / "params.txt"
    S.write_params(p, "IC_Evrard_1472.bin", 1472, G=1.0, unitLength_in_cm=3.086e18)
    lines = p.read_text().splitlines()
    assert lines[0] == "IC_Evrard_1472.bin" and len(lines) == 14
    r = S.read_params(p)
    assert r["filename"] == "IC_Evrard_1472.bin" and r["N_tot"] == 1472 and r["ndx_BH"] == 1472
    assert r["unitLength_in_cm"] == pytest.approx(3.086e18) and r["sigma_in_code_unit"] == 1.0


def test_library_header_check(tmp_path):
    from sph_2_b200.core import ic_count
    c = _cols(9, 2)
    p = tmp_path / "ic.bin"
    S.write_ic(p, c["x"], c["y"], c["z"], c["vx"], c["vy"], c["vz"], c["u"], c["h"], c["mass"])
    assert ic_count(p) == 9
    raw = p.read_bytes()
    (tmp_path / "short.bin").write_bytes(raw[:-4])
    with pytest.raises(L.SphError) as e:
        ic_count(tmp_path / "short.bin")
    assert e.value.code == -9
    with pytest.raises(L.SphError):
        ic_count(tmp_path / "missing.bin")


def test_cooling_table_file_layout(tmp_path):
    """The grid file of the table backend: written in the reference's
    coolHeatGridNew.bin layout, its header and size checked by the library
    without a GPU, and read back unchanged."""
    from sph_2_b200 import cooling
    t = cooling.synthetic_table(seed=1, n_kpc=2, n_nH=5, n_Z=3, n_T=7, n_M=2, n_time=4)
    p = tmp_path / "grid.bin"
    cooling.write_table_file(p, **t)
    dims = np.zeros(6, np.int32)
    lib = L.load()
    assert lib.sph_cooling_table_dims(str(p).encode(), dims.ctypes.data_as(C.c_void_p)) == 0
    assert dims.tolist() == [2, 5, 3, 7, 2, 4]
    r = cooling.read_table_file(p)
    for k in ("kpc", "nH", "T", "time_s", "u_evol", "frac"):
        assert np.array_equal(r[k], np.asarray(t[k], np.float32)), k
    raw = p.read_bytes()
    (tmp_path / "short.bin").write_bytes(raw[:-4])
    assert lib.sph_cooling_table_dims(str(tmp_path / "short.bin").encode(),
                                      dims.ctypes.data_as(C.c_void_p)) == -9
