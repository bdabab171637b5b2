"""The C-ABI library loads on a machine without a GPU and exports every declared symbol."""

from __future__ import annotations

import ctypes
import os
import re

import pytest

from ordito_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "ordito_b200.h")


def declared_functions() -> list[str]:
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(ob_\w+)\(", text, re.M)))


def test_library_is_built() -> None:
    assert _lib.LIBRARY_PATH.exists(), "run python -m ordito_b200.build"


def test_every_declared_symbol_is_exported_and_bound() -> None:
    lib = ctypes.CDLL(str(_lib.LIBRARY_PATH))
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_errors_cross_the_boundary_as_status_codes() -> None:
    # A null output pointer is rejected on the host before any CUDA call.
    status = _lib.lib.ob_pattern_workspace(10, 10, None)
    assert status == _lib.OB_ERR_INVALID
    assert b"null" in _lib.lib.ob_last_error()
    with pytest.raises(ValueError):
        _lib.check(status)


def test_a_call_without_a_device_returns_a_status() -> None:
    # The sort's workspace query asks the device for its properties: without one it must come
    # back as a CUDA status with a message, never a crash.
    size = ctypes.c_size_t(0)
    status = _lib.lib.ob_pattern_workspace(1000, 2000, ctypes.byref(size))
    if _lib.device_count() > 0:
        assert status == _lib.OB_OK and size.value > 8 * (6 * 2000 + 1000)
    else:
        assert status == _lib.OB_ERR_CUDA
        assert _lib.lib.ob_last_error()


@pytest.mark.parametrize("chunk", [17, 20, 12, 4100])
def test_split_chunk_must_keep_copies_aligned(chunk: int) -> None:
    # A split tile starts its inner range at a multiple of chunk and the tile kernels read from
    # there in 16-byte pieces, so only multiples of 8 doubles in [16, 4096] (or 0) pass. The
    # arguments are checked before the handle is touched, so a placeholder handle is enough.
    status = _lib.lib.ob_chol_tile(ctypes.c_void_p(1), chunk, 2, None)
    assert status == _lib.OB_ERR_INVALID
    assert b"chunk" in _lib.lib.ob_last_error()
