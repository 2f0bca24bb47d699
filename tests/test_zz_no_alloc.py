"""GPU: ocu_grid_reduce_noalloc, the reduction entry point that performs no device allocation.

It serves callers that may not allocate device memory at the moment they need a norm (their
host or framework owns the device memory, or the code path must stay off the allocator); its
scratch is a static array inside the library.  Called through the C ABI, it must return the
same value as ocu_grid_reduce, bit for bit, on two calls in a row -- the second call reuses the
array the first one left behind.  This file is collected last so that a run stopping at the
first failure has already run every other test; it also passes when run on its own.
"""
import ctypes as C

import numpy as np
import pytest

import opencurrent_b200 as ocu
from opencurrent_b200 import _capi

pytestmark = pytest.mark.gpu

OPS = [_capi.REDUCE_MAXABS, _capi.REDUCE_MAX, _capi.REDUCE_MIN, _capi.REDUCE_SUM, _capi.REDUCE_SQRSUM,
       _capi.REDUCE_CHECKNAN]


def _grid(dtype, shape, seed):
    g = ocu.Grid3DDevice(dtype)
    g.init(*shape)
    rng = np.random.default_rng(seed)
    host = rng.uniform(-2.0, 2.0, int(g.layout.allocated)).astype(np.float64 if dtype == ocu.F64 else np.float32)
    g.copy_from_host(host)
    return g


def _reduce(fn, g, op):
    r = C.c_double(np.nan)
    st = fn(g.handle, op, C.byref(r), None)
    assert st == _capi.OK, ocu.load().ocu_last_error()
    return r.value


@pytest.mark.parametrize("dtype", [ocu.F32, ocu.F64])
@pytest.mark.parametrize("shape", [(64, 64, 64), (33, 70, 45), (256, 256, 40), (1024, 1024, 2)])
def test_noalloc_matches_allocating_reduce_twice(dtype, shape):
    lib = ocu.load()
    g = _grid(dtype, shape, seed=sum(shape))
    for op in OPS:
        ref = _reduce(lib.ocu_grid_reduce, g, op)
        first = _reduce(lib.ocu_grid_reduce_noalloc, g, op)
        second = _reduce(lib.ocu_grid_reduce_noalloc, g, op)
        assert first == ref and second == ref, (op, ref, first, second)


def test_noalloc_allocates_nothing():
    """After the first call (which only looks up the static array's address), calls leave the
    device's free memory unchanged; an allocation of any size would take at least one 2 MB
    page from it."""
    import torch

    lib = ocu.load()
    g = _grid(ocu.F64, (128, 96, 40), seed=4)
    _reduce(lib.ocu_grid_reduce_noalloc, g, _capi.REDUCE_SQRSUM)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for op in OPS:
        _reduce(lib.ocu_grid_reduce_noalloc, g, op)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_back_to_back_different_grids():
    """Consecutive calls on different grids: the shared scratch carries no state across calls."""
    lib = ocu.load()
    a = _grid(ocu.F32, (128, 128, 32), seed=1)
    b = _grid(ocu.F64, (16, 8, 70), seed=2)
    for _ in range(2):
        for g in (a, b):
            assert _reduce(lib.ocu_grid_reduce_noalloc, g, _capi.REDUCE_SQRSUM) == \
                _reduce(lib.ocu_grid_reduce, g, _capi.REDUCE_SQRSUM)


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    lib = ocu.load()
    rows_max = 256 * 4096
    g = ocu.Grid3DDevice(ocu.F32)
    g.init(1025, 1024, 1)  # nx*ny = rows_max + 1024
    assert 1025 * 1024 > rows_max
    r = C.c_double(0)
    st = lib.ocu_grid_reduce_noalloc(g.handle, _capi.REDUCE_SUM, C.byref(r), None)
    assert st == _capi.ERR_INVALID_VALUE
    assert b"static scratch" in lib.ocu_last_error()
