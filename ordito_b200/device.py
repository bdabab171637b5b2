"""Device arrays: the library's own buffers, exchanged zero-copy through ``__cuda_array_interface__``.

A ``DeviceArray`` is a pool allocation made through the C ABI (``ob_malloc``), freed when the
last reference to it goes. Every public function of this package accepts, for an array argument,
a ``DeviceArray``, any object exposing ``__cuda_array_interface__`` (a Warp array, a PyTorch CUDA
tensor, a CuPy array -- read in place, no copy), or a host NumPy array (uploaded once).
"""

from __future__ import annotations

import ctypes
from typing import Any

import numpy as np

from ordito_b200 import _lib

_TYPESTR = {
    np.dtype(np.float32): "<f4",
    np.dtype(np.float64): "<f8",
    np.dtype(np.int32): "<i4",
    np.dtype(np.uint64): "<u8",
    np.dtype(np.int64): "<i8",
    np.dtype(np.uint32): "<u4",
    np.dtype(np.uint8): "|u1",
}
_FROM_TYPESTR = {v: k for k, v in _TYPESTR.items()}

# The stream every wrapper enqueues on unless told otherwise: the legacy default stream, which
# PyTorch's default stream also is, so buffers shared with it need no extra synchronisation.
DEFAULT_STREAM = None


class DeviceArray:
    """A contiguous device buffer with a shape and a NumPy dtype."""

    __slots__ = ("ptr", "shape", "dtype", "_owned", "_base", "__weakref__")

    def __init__(self, ptr: int, shape: tuple[int, ...], dtype: Any, *, owned: bool, base: Any = None):
        self.ptr = int(ptr or 0)
        self.shape = tuple(int(s) for s in shape)
        self.dtype = np.dtype(dtype)
        self._owned = owned
        self._base = base

    # -- construction ------------------------------------------------------------------------
    @classmethod
    def empty(cls, shape: int | tuple[int, ...], dtype: Any = np.float64) -> "DeviceArray":
        shape = (shape,) if isinstance(shape, (int, np.integer)) else tuple(shape)
        nbytes = int(np.prod(shape, dtype=np.int64)) * np.dtype(dtype).itemsize
        ptr = ctypes.c_void_p(0)
        if nbytes > 0:
            _lib.call("ob_malloc", nbytes, ctypes.byref(ptr), DEFAULT_STREAM)
        return cls(ptr.value or 0, shape, dtype, owned=nbytes > 0)

    @classmethod
    def zeros(cls, shape: int | tuple[int, ...], dtype: Any = np.float64) -> "DeviceArray":
        out = cls.empty(shape, dtype)
        out.fill_zero()
        return out

    @classmethod
    def from_host(cls, array: np.ndarray, dtype: Any = None) -> "DeviceArray":
        host = np.ascontiguousarray(array, dtype=dtype)
        out = cls.empty(host.shape, host.dtype)
        if host.nbytes:
            _lib.call("ob_memcpy", out.ptr, host.ctypes.data, host.nbytes, 0, DEFAULT_STREAM, 1)
        return out

    def __del__(self) -> None:
        if self._owned and self.ptr:
            try:
                _lib.lib.ob_free(self.ptr, DEFAULT_STREAM)
            except Exception:  # interpreter shutdown: the process is going anyway
                pass
            self.ptr = 0

    # -- properties --------------------------------------------------------------------------
    @property
    def size(self) -> int:
        return int(np.prod(self.shape, dtype=np.int64))

    @property
    def nbytes(self) -> int:
        return self.size * self.dtype.itemsize

    @property
    def ndim(self) -> int:
        return len(self.shape)

    def __len__(self) -> int:
        return self.shape[0] if self.shape else 0

    @property
    def __cuda_array_interface__(self) -> dict[str, Any]:
        return {
            "shape": self.shape,
            "typestr": _TYPESTR[self.dtype],
            "data": (self.ptr, False),
            "strides": None,
            "version": 3,
        }

    def __repr__(self) -> str:
        return f"DeviceArray(shape={self.shape}, dtype={self.dtype})"

    # -- operations --------------------------------------------------------------------------
    def numpy(self) -> np.ndarray:
        """Copy to the host (waits for the stream)."""
        host = np.empty(self.shape, dtype=self.dtype)
        if host.nbytes:
            _lib.call("ob_memcpy", host.ctypes.data, self.ptr, host.nbytes, 1, DEFAULT_STREAM, 1)
        return host

    def fill_zero(self) -> "DeviceArray":
        if self.nbytes:
            _lib.call("ob_memset", self.ptr, 0, self.nbytes, DEFAULT_STREAM)
        return self

    def copy_from(self, other: Any) -> "DeviceArray":
        src, keep = device_pointer(other, self.dtype, self.size)
        if self.nbytes:
            _lib.call("ob_memcpy", self.ptr, src, self.nbytes, 2, DEFAULT_STREAM, 0)
        del keep
        return self

    def copy(self) -> "DeviceArray":
        return DeviceArray.empty(self.shape, self.dtype).copy_from(self)

    def view(self, start: int, stop: int, shape: tuple[int, ...] | None = None) -> "DeviceArray":
        """Elements ``[start, stop)`` of the flat buffer, sharing its memory."""
        count = stop - start
        return DeviceArray(
            self.ptr + start * self.dtype.itemsize if count else 0,
            shape or (count,),
            self.dtype,
            owned=False,
            base=self,
        )

    def reshape(self, *shape: int) -> "DeviceArray":
        shape = shape[0] if len(shape) == 1 and isinstance(shape[0], tuple) else shape
        shape = tuple(int(s) for s in shape)
        if -1 in shape:
            known = int(np.prod([s for s in shape if s != -1]))
            shape = tuple(self.size // known if s == -1 else s for s in shape)
        if int(np.prod(shape)) != self.size:
            raise ValueError(f"cannot reshape {self.shape} to {shape}")
        return DeviceArray(self.ptr, shape, self.dtype, owned=False, base=self)

    def flatten(self) -> "DeviceArray":
        return self.reshape(self.size)


class PinnedArray:
    """Page-locked host memory viewed as a NumPy array (fast device<->host copies)."""

    def __init__(self, shape: int | tuple[int, ...], dtype: Any = np.float64) -> None:
        shape = (shape,) if isinstance(shape, (int, np.integer)) else tuple(shape)
        dtype = np.dtype(dtype)
        nbytes = max(int(np.prod(shape, dtype=np.int64)) * dtype.itemsize, 1)
        ptr = ctypes.c_void_p(0)
        _lib.call("ob_host_alloc", nbytes, ctypes.byref(ptr))
        self.ptr = int(ptr.value)
        buffer = (ctypes.c_byte * nbytes).from_address(self.ptr)
        self.array = np.frombuffer(buffer, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def __del__(self) -> None:
        if getattr(self, "ptr", 0):
            try:
                _lib.lib.ob_host_free(self.ptr)
            except Exception:
                pass
            self.ptr = 0

    def copy_from_device(self, device: "DeviceArray", sync: bool = True) -> np.ndarray:
        if device.nbytes > self.array.nbytes:
            raise ValueError("pinned buffer too small")
        _lib.call("ob_memcpy", self.ptr, device.ptr, device.nbytes, 1, DEFAULT_STREAM, int(sync))
        return self.array

    def upload(self, sync: bool = False) -> "DeviceArray":
        out = DeviceArray.empty(self.array.shape, self.array.dtype)
        _lib.call("ob_memcpy", out.ptr, self.ptr, self.array.nbytes, 0, DEFAULT_STREAM, int(sync))
        return out


def interface_of(obj: Any) -> dict[str, Any] | None:
    return getattr(obj, "__cuda_array_interface__", None)


def device_pointer(obj: Any, dtype: Any, size: int | None = None) -> tuple[int, Any]:
    """Return ``(pointer, keepalive)`` for ``obj`` as a contiguous device buffer of ``dtype``.

    A device object must already have the dtype (no silent conversion of a device array); a host
    array is converted and uploaded. ``size``, when given, is the element count required.
    """
    dtype = np.dtype(dtype)
    if obj is None:
        return 0, None
    iface = interface_of(obj)
    if iface is not None:
        typestr = iface["typestr"]
        have = _FROM_TYPESTR.get(typestr)
        if have is None or have != dtype:
            raise ValueError(f"expected a {dtype} device array, got typestr {typestr!r}")
        shape = tuple(iface["shape"])
        strides = iface.get("strides")
        if strides is not None:
            expected = []
            step = dtype.itemsize
            for extent in reversed(shape):
                expected.append(step)
                step *= extent
            if tuple(reversed(expected)) != tuple(strides) and int(np.prod(shape)) > 1:
                raise ValueError("device arrays must be C-contiguous")
        n = int(np.prod(shape, dtype=np.int64))
        if size is not None and n != size:
            raise ValueError(f"expected {size} elements, got {n} (shape {shape})")
        return int(iface["data"][0] or 0), obj
    host = np.ascontiguousarray(np.asarray(obj), dtype=dtype)
    if size is not None and host.size != size:
        raise ValueError(f"expected {size} elements, got {host.size}")
    uploaded = DeviceArray.from_host(host)
    return uploaded.ptr, uploaded


def as_device(obj: Any, dtype: Any) -> DeviceArray:
    """``obj`` as a ``DeviceArray`` of ``dtype`` (a zero-copy wrapper of a device object)."""
    if isinstance(obj, DeviceArray):
        if obj.dtype != np.dtype(dtype):
            raise ValueError(f"expected {np.dtype(dtype)}, got {obj.dtype}")
        return obj
    iface = interface_of(obj)
    if iface is not None:
        ptr, keep = device_pointer(obj, dtype)
        return DeviceArray(ptr, tuple(iface["shape"]), dtype, owned=False, base=keep)
    return DeviceArray.from_host(np.asarray(obj), dtype=dtype)


def element_count(obj: Any) -> int:
    if isinstance(obj, DeviceArray):
        return obj.size
    iface = interface_of(obj)
    if iface is not None:
        return int(np.prod(iface["shape"], dtype=np.int64))
    return int(np.asarray(obj).size)


def synchronize() -> None:
    """Wait for all of the library's work on the current device, on every stream (the served and
    batched passes run on created non-blocking streams, which the legacy default stream does not
    wait for)."""
    _lib.call("ob_device_synchronize")


def trim_pool(keep_bytes: int = 0) -> None:
    """Hand the device memory the library keeps for reuse back to the driver, all but
    ``keep_bytes`` of it (after a device-wide synchronise)."""
    _lib.call("ob_mem_trim", int(keep_bytes))
