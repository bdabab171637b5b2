"""The allocation-free shift (``ob_shift_noalloc``) against the allocating one (``ob_shift``).

``ob_shift_noalloc`` exists for callers that cannot let the library allocate device memory (a
host runtime that owns every byte of the device, or a latency-critical loop); it keeps its
scratch in a static device array instead. This file is collected last, so a run that stops at
its first failure has run every other test before it.
"""

from __future__ import annotations

import numpy as np
import pytest

from ordito_b200 import _lib
from ordito_b200.device import DeviceArray

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the two folds sum the same terms in a different block order


def shift_both(phi: np.ndarray, sources: np.ndarray, offsets: np.ndarray | None, k: int):
    n = phi.shape[0]
    a = DeviceArray.from_host(phi.reshape(-1))
    b = DeviceArray.from_host(phi.reshape(-1))
    src = DeviceArray.from_host(sources.astype(np.int32))
    off = DeviceArray.from_host(offsets.astype(np.int32)) if offsets is not None else None
    off_ptr = off.ptr if off is not None else None
    _lib.call("ob_shift", a.ptr, n, src.ptr, src.size, off_ptr, k, 1, None)
    _lib.call("ob_shift_noalloc", b.ptr, n, src.ptr, src.size, off_ptr, k, 1, None)
    return a.numpy().reshape(n, k), b.numpy().reshape(n, k)


def test_no_alloc_shift_matches_the_allocating_one(gpu) -> None:
    rng = np.random.default_rng(11)
    n = 40_000
    # Two calls in a row through the shared static scratch, several columns with ragged sources.
    for k in (7, 7):
        phi = rng.normal(size=(n, k)) + 3.0
        counts = rng.integers(1, 9, size=k)
        offsets = np.concatenate(([0], np.cumsum(counts)))
        sources = rng.integers(0, n, size=int(offsets[-1]))
        expected, got = shift_both(phi, sources, offsets, k)
        np.testing.assert_allclose(got, expected, rtol=RTOL, atol=RTOL * np.abs(expected).max())
    # One column with no offsets, and a field whose orientation flips.
    for sign in (1.0, -1.0):
        phi = sign * rng.random(size=(n, 1))
        sources = rng.integers(0, n, size=3)
        expected, got = shift_both(phi, sources, None, 1)
        np.testing.assert_allclose(got, expected, rtol=RTOL, atol=RTOL * np.abs(expected).max())


def test_no_alloc_shift_takes_nothing_from_the_pool(gpu) -> None:
    # Its promise: a call allocates nothing. Read the device pool's used and reserved bytes
    # around a run of calls made on their own (after one warm-up call), with every input made
    # beforehand; neither may move.
    from cuda.bindings import driver

    from ordito_b200.device import synchronize

    assert driver.cuInit(0)[0] == driver.CUresult.CUDA_SUCCESS
    rng = np.random.default_rng(5)
    n, k = 50_000, 16
    phi = DeviceArray.from_host((rng.normal(size=(n, k)) + 2.0).reshape(-1))
    counts = rng.integers(1, 5, size=k)
    offsets = DeviceArray.from_host(np.concatenate(([0], np.cumsum(counts))).astype(np.int32))
    sources = DeviceArray.from_host(rng.integers(0, n, size=int(counts.sum())).astype(np.int32))

    def pool() -> tuple[int, int]:
        synchronize()
        err, device = driver.cuCtxGetDevice()
        assert err == driver.CUresult.CUDA_SUCCESS
        err, handle = driver.cuDeviceGetDefaultMemPool(device)
        assert err == driver.CUresult.CUDA_SUCCESS
        attr = driver.CUmemPool_attribute
        used = int(driver.cuMemPoolGetAttribute(handle, attr.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)[1])
        reserved = int(driver.cuMemPoolGetAttribute(handle, attr.CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT)[1])
        return used, reserved

    def call() -> None:
        _lib.call("ob_shift_noalloc", phi.ptr, n, sources.ptr, sources.size, offsets.ptr, k, 1, None)

    call()
    before = pool()
    for _ in range(20):
        call()
    assert pool() == before


def test_no_alloc_shift_rejects_too_many_columns(gpu) -> None:
    phi = DeviceArray.zeros(10 * 65, np.float64)
    src = DeviceArray.from_host(np.zeros(65, dtype=np.int32))
    offsets = DeviceArray.from_host(np.arange(66, dtype=np.int32))
    status = _lib.lib.ob_shift_noalloc(phi.ptr, 10, src.ptr, 65, offsets.ptr, 65, 1, None)
    assert status == _lib.OB_ERR_INVALID
    assert b"n_columns" in _lib.lib.ob_last_error()
