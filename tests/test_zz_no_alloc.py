"""mtd_factor_noalloc: the factorisation entry point for callers that cannot allocate
device memory.

Callers whose device memory belongs entirely to a pool allocator (PyTorch's caching
allocator, RMM) and latency-critical request paths cannot call cudaMalloc.
mtd_factor_noalloc keeps all of its device scratch in one fixed 24 MiB array inside the
library instead.  These tests call
it through the C ABI and check that it gives what the allocating entry points
(mtd_tiled_cholesky / mtd_tiled_lu) give, within the FP64 parity tolerance of the other
tests, on consecutive calls that reuse the same array -- including a call after a larger
problem of the other kind left its own contents there -- and that a warm call leaves the
device's free memory exactly as it found it.  This file runs last in the
suite (pytest orders files by name), after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from oracle import gen
from tests.gpu_util import from_dev, rel_diff, to_dev

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _noalloc(mtd, kind, d, tile):
    lib = mtd.lib()
    info = ctypes.c_int(-1)
    n = d.shape[0]
    rc = lib.mtd_factor_noalloc(kind, ctypes.c_void_p(d.data_ptr()), n, d.stride(1), tile, None, ctypes.byref(info))
    return rc, info.value


def _allocating(mtd, kind, d, tile):
    lib = mtd.lib()
    info = ctypes.c_int(-1)
    fn = lib.mtd_tiled_cholesky if kind == mtd.KIND_CHOLESKY else lib.mtd_tiled_lu
    rc = fn(ctypes.c_void_p(d.data_ptr()), d.shape[0], d.stride(1), tile, None, ctypes.byref(info))
    return rc, info.value


def _compare(mtd, kind, a, tile):
    import torch
    ref = to_dev(a)
    assert _allocating(mtd, kind, ref, tile) == (0, 0)
    want = from_dev(ref)
    for _ in range(2):  # two calls in a row on fresh copies share the one scratch array
        d = to_dev(a)
        assert _noalloc(mtd, kind, d, tile) == (0, 0)
        torch.cuda.synchronize()
        got = from_dev(d)
        if kind == mtd.KIND_CHOLESKY:
            assert rel_diff(np.tril(got), np.tril(want)) <= TOL
            assert np.array_equal(np.triu(got, 1), np.triu(a, 1))
        else:
            assert rel_diff(got, want) <= TOL


@pytest.mark.parametrize("kind_name,n,tile", [("chol", 2048, 512), ("lu", 2048, 512),
                                              ("chol", 1500, 384), ("lu", 1030, 256)])
def test_noalloc_matches_allocating_entry_point(mtd, kind_name, n, tile):
    kind = mtd.KIND_CHOLESKY if kind_name == "chol" else mtd.KIND_LU
    a = gen.spd_input(n, 31) if kind_name == "chol" else gen.lu_input(n, 31)
    _compare(mtd, kind, a, tile)


def test_noalloc_after_a_larger_call_of_the_other_kind(mtd):
    # a large LU fills more of the array (more tasks, queue slots, both inverse
    # workspaces); a smaller Cholesky right after must not see any of it
    _compare(mtd, mtd.KIND_LU, gen.lu_input(4000, 7), 1000)
    _compare(mtd, mtd.KIND_CHOLESKY, gen.spd_input(600, 7), 300)


def test_noalloc_rejects_problems_beyond_its_scratch(mtd):
    import torch
    d = torch.empty((8, 8), dtype=torch.float64, device="cuda").t()
    lib = mtd.lib()
    info = ctypes.c_int(0)
    # n above the 16384 limit: rejected before any device work
    rc = lib.mtd_factor_noalloc(mtd.KIND_CHOLESKY, ctypes.c_void_p(d.data_ptr()), 20000, 20000, 512, None,
                                ctypes.byref(info))
    assert rc == 11  # MTD_ERR_TOO_LARGE
    # n within the limit but a tile so small that the task graph exceeds the task table
    rc = lib.mtd_factor_noalloc(mtd.KIND_LU, ctypes.c_void_p(d.data_ptr()), 16000, 16000, 128, None,
                                ctypes.byref(info))
    assert rc == 11
    assert b"scratch" in lib.mtd_strerror(rc)
    # a tiny tile (2000 x 2000 tiles, ~2.7e9 tasks) is rejected from the closed-form task
    # count, before any task list is built
    import time
    t0 = time.perf_counter()
    rc = lib.mtd_factor_noalloc(mtd.KIND_LU, ctypes.c_void_p(d.data_ptr()), 16000, 16000, 8, None,
                                ctypes.byref(info))
    assert rc == 11 and time.perf_counter() - t0 < 1.0


def test_noalloc_allocates_no_device_memory(mtd):
    import torch
    a = gen.spd_input(2048, 5)
    d1, d2 = to_dev(a), to_dev(a)
    assert _noalloc(mtd, mtd.KIND_CHOLESKY, d1, 512) == (0, 0)  # warm: per-device set-up done
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert _noalloc(mtd, mtd.KIND_CHOLESKY, d2, 512) == (0, 0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(from_dev(d1), from_dev(d2))


def test_noalloc_reports_non_spd_info(mtd):
    a = gen.spd_input(700, 3)
    a[500, 500] = -5.0
    d = to_dev(a)
    rc, info = _noalloc(mtd, mtd.KIND_CHOLESKY, d, 256)
    assert rc == 5 and info == 501
    # and the next call is clean
    b = gen.spd_input(700, 3)
    _compare(mtd, mtd.KIND_CHOLESKY, b, 256)
