"""The C-ABI library loads and exports every entry point include/sph_b200.h
declares, and the ctypes mirror of the structs matches the header.  No
compute calls: this runs without a GPU."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sph_b200.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sph_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from sph_2_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from sph_2_b200 import build
        build.build()
    return C.CDLL(_lib.LIB_PATH)


def test_exports_every_declared_symbol(lib):
    names = declared()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from sph_2_b200 import _lib
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(declared()) <= bound, set(declared()) - bound


def test_struct_layout_matches_header():
    from sph_2_b200 import _lib
    txt = open(HEADER).read()
    body = re.search(r"typedef struct sph_config \{(.*?)\} sph_config;", txt, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for typ, decl in re.findall(r"(int32_t|double)\s+([^;]+);", body):
        names += [d.strip() for d in decl.split(",")]
    assert [f[0] for f in _lib.SphConfig._fields_] == names
    body = re.search(r"typedef struct sph_cooling_params \{(.*?)\} sph_cooling_params;", txt,
                     re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for typ, decl in re.findall(r"(int32_t|double)\s+([^;]+);", body):
        names += [d.strip() for d in decl.split(",")]
    assert [f[0] for f in _lib.SphCoolingParams._fields_] == names


def test_context_create_fails_loudly_without_gpu(lib):
    """On a machine without a CUDA device the library reports an error code
    instead of falling back to anything."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from sph_2_b200 import _lib
    L = _lib.load()
    cfg = _lib.SphConfig()
    assert L.sph_default_config(C.byref(cfg)) == 0
    h = C.c_void_p()
    assert L.sph_ctx_create(C.byref(cfg), C.byref(h)) != 0


def test_python_config_defaults_match_the_library():
    """Config() and sph_default_config give the same sph_config, field by
    field (host-only call, no GPU); the walk's optional settings default
    to off."""
    from sph_2_b200 import Config, _lib
    L = _lib.load()
    c = _lib.SphConfig()
    assert L.sph_default_config(C.byref(c)) == 0
    py = Config().to_c()
    for name, _ in _lib.SphConfig._fields_:
        assert getattr(py, name) == getattr(c, name), name
    assert c.theta_local == 0.0 and c.theta_small == 0.0 and c.small_cell == 0
    on = Config(theta_local=0.28, theta_small=0.45, small_cell=128).to_c()
    assert (on.theta_local, on.theta_small, on.small_cell) == (0.28, 0.45, 128)
