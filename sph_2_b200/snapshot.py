"""The reference's file formats on the host side: binary IC files, snapshots
and the line-oriented params.txt, read and written with NumPy.

* IC file -- Particles_in_BH_Tree_II/Evrard_test/IC_evrard4.cu:245-260 writes
  it, hfvCLibs_v7_hfv_v2.h:59-101 (readVectorsFromFile) reads it:
  int32 N, int32 Typ[N], float32 x, y, z, vx, vy, vz, u, h, eps, mass [N each].
* snapshot -- hfvCLibs_v7_hfv_v2.h:107-143 (saveArraysToBinary) writes it,
  Evrard_test/singlex_gpu_data.py:55-72 reads it: int32 N, int32 N_ionFrac,
  int32 Typ[N], float32 x, y, z, vx, vy, vz, rho, h, u, mass [N each],
  float32 ionFrac[N_ionFrac], int32 debug[N].
* params.txt -- IC_evrard4.cu:277-295 writes it, hfvCLibs_v7_hfv_v2.h:21-50
  (readParams) reads it: the IC file name on the first line, then N_tot,
  ndx_BH, G, L_AGN, M_dot_in, v_in, u_for_10K_Temp, m_sph_high_res, sigma,
  UnitDensity_in_cgs, Unit_u_in_cgs, unitTime_in_s, unitLength_in_cm.

The GPU context reads and writes the binary files itself
(Context.load_ic / write_ic / write_snapshot, native code); these functions
are for scripts that prepare inputs or analyse outputs without a GPU.
"""
from __future__ import annotations

import numpy as np

IC_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "u", "h", "eps", "mass")
SNAP_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "rho", "h", "u", "mass")
PARAMS = ("N_tot", "ndx_BH", "G", "L_AGN_code_unit", "M_dot_in_code_unit", "vin_in_code_unit",
          "u_for_10K_Temp", "m_sph_high_res", "sigma_in_code_unit", "UnitDensity_in_cgs",
          "Unit_u_in_cgs", "unitTime_in_s", "unitLength_in_cm")


def _read_exact(f, dtype, count):
    a = np.fromfile(f, dtype=dtype, count=count)
    if a.size != count:
        raise ValueError(f"file ends early: wanted {count} {np.dtype(dtype).name}, got {a.size}")
    return a


def read_ic(path) -> dict:
    """IC file -> dict of Typ (int32) and the ten float32 columns."""
    with open(path, "rb") as f:
        n = int(_read_exact(f, "<i4", 1)[0])
        if n < 0:
            raise ValueError(f"negative particle count {n}")
        out = {"N": n, "Typ": _read_exact(f, "<i4", n)}
        for k in IC_FIELDS:
            out[k] = _read_exact(f, "<f4", n)
        if f.read(1):
            raise ValueError("trailing bytes after the IC columns")
    return out


def write_ic(path, x, y, z, vx, vy, vz, u, h, mass, eps=None, typ=None):
    """Write an IC file; eps defaults to h (IC_evrard4.cu:224-229), Typ to 0."""
    n = len(x)
    cols = {"x": x, "y": y, "z": z, "vx": vx, "vy": vy, "vz": vz, "u": u, "h": h,
            "eps": h if eps is None else eps, "mass": mass}
    with open(path, "wb") as f:
        np.asarray([n], "<i4").tofile(f)
        np.asarray(np.zeros(n) if typ is None else typ, "<i4").tofile(f)
        for k in IC_FIELDS:
            a = np.asarray(cols[k], dtype="<f4")
            if a.shape != (n,):
                raise ValueError(f"column {k} has shape {a.shape}, expected ({n},)")
            a.tofile(f)


def read_snapshot(path) -> dict:
    """Snapshot -> dict of Typ, the ten float32 columns, ionFrac and debug."""
    with open(path, "rb") as f:
        n, nion = (int(v) for v in _read_exact(f, "<i4", 2))
        out = {"N": n, "N_ionFrac": nion, "Typ": _read_exact(f, "<i4", n)}
        for k in SNAP_FIELDS:
            out[k] = _read_exact(f, "<f4", n)
        out["ionFrac"] = _read_exact(f, "<f4", nion)
        out["debug"] = _read_exact(f, "<i4", n)
        if f.read(1):
            raise ValueError("trailing bytes after the snapshot")
    return out


def write_params(path, ic_filename, n_tot, **kw):
    """params.txt in the reference's order; quantities not given are 1.0 and
    ndx_BH is N_tot (no black hole), as IC_evrard4.cu writes them."""
    vals = {"N_tot": int(n_tot), "ndx_BH": int(kw.pop("ndx_BH", n_tot))}
    for k in PARAMS[2:]:
        vals[k] = float(kw.pop(k, 1.0))
    if kw:
        raise ValueError(f"unknown params {sorted(kw)}")
    with open(path, "w") as f:
        f.write(f"{ic_filename}\n")
        for k in PARAMS:
            f.write(f"{vals[k]}\n")


def read_params(path) -> dict:
    """params.txt -> dict (file name, two ints, eleven floats)."""
    with open(path) as f:
        name = f.readline().rstrip("\n")
        tok = f.read().split()
    if len(tok) < len(PARAMS):
        raise ValueError(f"params file has {len(tok)} values, expected {len(PARAMS)}")
    out = {"filename": name}
    for k, t in zip(PARAMS, tok):
        out[k] = int(t) if k in ("N_tot", "ndx_BH") else float(t)
    return out
