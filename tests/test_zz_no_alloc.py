"""The allocation-free Morton-order entry point against the context path.

sph_morton_sort_noalloc exists for callers that must not allocate device
memory (for instance when another framework's caching allocator owns the
device memory, or where cudaMalloc's implicit synchronisation is not
acceptable): it uses a fixed scratch array compiled into the library instead.
This file runs last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from sph_2_b200 import Config, Context, ic
from sph_2_b200 import _lib as L

pytestmark = pytest.mark.gpu


def context_keys_perm(pos):
    """Keys (input order) and stable permutation from the existing entry points
    (sph_load + sph_sort + sph_get_sort)."""
    n = len(pos)
    with Context(Config(n_max=n, precision="fp64")) as ctx:
        ctx.load(pos)
        ctx.sort()
        return ctx.sort_info()


def noalloc_keys_perm(pos, stream=None, free_bytes=None):
    """Run the entry point on device copies of pos, on `stream` (default: the
    current torch stream).  free_bytes: a list that receives the device's free
    memory just before and just after the call."""
    import torch
    lib = L.load()
    dev = torch.device("cuda:0")
    x, y, z = (torch.tensor(np.ascontiguousarray(pos[:, k]), dtype=torch.float64, device=dev)
               for k in range(3))
    n = len(pos)
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    stream = stream or torch.cuda.current_stream()
    torch.cuda.synchronize()
    if free_bytes is not None:
        free_bytes.append(torch.cuda.mem_get_info()[0])
    rc = lib.sph_morton_sort_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                     C.c_void_p(z.data_ptr()), n, C.c_void_p(keys.data_ptr()),
                                     C.c_void_p(perm.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    if free_bytes is not None:
        free_bytes.append(torch.cuda.mem_get_info()[0])
    return keys.cpu().numpy().view(np.uint64), perm.cpu().numpy()


def test_noalloc_matches_context_sort_on_two_calls_in_a_row():
    a = ic.evrard(50_000, seed=3)["pos"]
    b = ic.evrard(L.NOALLOC_MAX_N, seed=4)["pos"]
    b[17] = b[5]                      # equal keys must keep their input order
    for pos in (a, b):                # two calls in a row share the scratch array
        k_ref, p_ref = context_keys_perm(pos)
        k, p = noalloc_keys_perm(pos)
        assert np.array_equal(k, k_ref)
        assert np.array_equal(p, p_ref)


def test_noalloc_takes_no_device_memory_and_runs_on_any_stream():
    """A repeated call leaves the device's free memory unchanged, and a call
    queued on a non-default stream gives the same order."""
    import torch
    pos = ic.evrard(100_000, seed=6)["pos"]
    k_ref, p_ref = context_keys_perm(pos)
    noalloc_keys_perm(pos)                         # first call on the device: set-up
    free = []
    k, p = noalloc_keys_perm(pos, free_bytes=free)
    assert free[0] == free[1], f"free device memory changed by {free[0] - free[1]} bytes"
    assert np.array_equal(k, k_ref) and np.array_equal(p, p_ref)
    side = torch.cuda.Stream()
    k2, p2 = noalloc_keys_perm(pos, stream=side)
    assert np.array_equal(k2, k_ref) and np.array_equal(p2, p_ref)


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = L.load()
    dummy = C.c_void_p(1)
    rc = lib.sph_morton_sort_noalloc(dummy, dummy, dummy, L.NOALLOC_MAX_N + 1, dummy, dummy, None)
    assert rc == -3                   # SPH_ERR_CAPACITY, nothing launched
    assert lib.sph_morton_sort_noalloc(None, None, None, 10, None, None, None) == -1
    assert lib.sph_morton_sort_noalloc(None, None, None, 0, None, None, None) == 0
