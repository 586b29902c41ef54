"""The allocation-free Gaussian filter entry point.

gpk_gaussian_filter_3d_noalloc serves callers that cannot call cudaMalloc
(device memory owned by another allocator or a fixed budget, loops that must
not allocate, hosts that only link the library): it keeps its scratch in a
static device array instead.  Its result must equal the allocating
gpk_gaussian_filter_3d's bit for bit, including on a second call in a row,
when the static array still holds the first call's data.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from gpk_b200 import lib
from gpk_b200._lib import GPKError, check

pytestmark = pytest.mark.gpu


def _taps(sigma):
    r = int(np.ceil(3.5 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float32)
    w = np.exp(-x * x / np.float32(2 * sigma * sigma)).astype(np.float32)
    return (w / w.sum(dtype=np.float32)).astype(np.float32), r


def _call(fn, field, taps, r):
    out = np.empty_like(field)
    Nz, Ny, Nx = field.shape
    check(fn(field.ctypes.data, out.ctypes.data, Nz, Ny, Nx, taps.ctypes.data, r))
    return out


@pytest.mark.parametrize("shape,sigma", [((1, 96, 80), 2.0), ((20, 24, 28), 1.5), ((128, 128, 128), 5.0)])
def test_noalloc_filter_matches_allocating_filter_twice(shape, sigma):
    L = lib()
    check(L.gpk_device_init(0))
    taps, r = _taps(sigma)
    rng = np.random.default_rng(7)
    for call in range(2):
        field = rng.random(shape, dtype=np.float32)
        want = _call(L.gpk_gaussian_filter_3d, field, taps, r)
        got = _call(L.gpk_gaussian_filter_3d_noalloc, field, taps, r)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"call {call}"


def test_noalloc_filter_rejects_grids_beyond_its_scratch():
    L = lib()
    check(L.gpk_device_init(0))
    taps, r = _taps(1.0)
    big = np.zeros((1, 1, (1 << 21) + 1), dtype=np.float32)
    out = np.empty_like(big)
    rc = L.gpk_gaussian_filter_3d_noalloc(big.ctypes.data, out.ctypes.data, 1, 1, big.shape[2],
                                          taps.ctypes.data, r)
    assert rc == 1
    assert b"static scratch" in L.gpk_last_error()


def test_noalloc_filter_after_a_larger_call():
    """A small 3-D grid and a 2-D grid (whose result lands in the other half
    of the array) right after a 128^3 call has filled both field regions:
    stale data from the larger call must not reach the result."""
    L = lib()
    check(L.gpk_device_init(0))
    rng = np.random.default_rng(11)
    for shape, sigma in [((128, 128, 128), 5.0), ((1, 70, 90), 2.0), ((12, 18, 10), 1.5), ((1, 33, 17), 0.8)]:
        taps, r = _taps(sigma)
        field = rng.random(shape, dtype=np.float32)
        want = _call(L.gpk_gaussian_filter_3d, field, taps, r)
        got = _call(L.gpk_gaussian_filter_3d_noalloc, field, taps, r)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), shape


def test_noalloc_filter_tap_limit():
    """511 taps (radius 255, the largest accepted; its passes are too wide
    for a shared-memory tile and run one thread per output) equal the
    allocating filter; 513 taps are rejected."""
    L = lib()
    check(L.gpk_device_init(0))
    rng = np.random.default_rng(12)
    field = rng.random((8, 8, 8), dtype=np.float32)
    w = rng.random(511, dtype=np.float32)
    taps = (w / w.sum(dtype=np.float32)).astype(np.float32)
    want = _call(L.gpk_gaussian_filter_3d, field, taps, 255)
    got = _call(L.gpk_gaussian_filter_3d_noalloc, field, taps, 255)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    big = np.ones(513, dtype=np.float32) / 513
    out = np.empty_like(field)
    rc = L.gpk_gaussian_filter_3d_noalloc(field.ctypes.data, out.ctypes.data, 8, 8, 8, big.ctypes.data, 256)
    assert rc == 1
    assert b"static scratch" in L.gpk_last_error()
