"""Sparse containers: the CSR matrix the operators are returned as (ordito/array.py bsr_from_csr).

ordito returns ``warp.sparse.BsrMatrix`` with 1x1 blocks; this build returns ``CsrMatrix``, which
exposes the same fields (``nrow``, ``ncol``, ``nnz``, ``offsets``, ``columns``, ``values``,
``shape``, ``scalar_type``) over device arrays; each array exposes ``__cuda_array_interface__``,
so a caller wraps them zero-copy in its own framework.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from ordito_b200.device import DeviceArray


class CsrMatrix:
    """A square or rectangular CSR matrix over device arrays (values float64 or float32)."""

    def __init__(self, nrow: int, ncol: int, offsets: DeviceArray, columns: DeviceArray,
                 values: DeviceArray, nnz: int | None = None) -> None:
        self.nrow = int(nrow)
        self.ncol = int(ncol)
        self.offsets = offsets
        self.columns = columns
        self.values = values
        self._nnz = nnz
        # Native solver states kept for this operator's lifetime (linalg._solver).
        self._solvers: dict[Any, Any] = {}
        self._factorization: Any = None

    @classmethod
    def from_host(cls, offsets: Any, columns: Any, values: Any, shape: tuple[int, int]) -> "CsrMatrix":
        """Upload host CSR arrays (int32 offsets/columns, float64 values)."""
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        return cls(int(shape[0]), int(shape[1]), DeviceArray.from_host(offsets),
                   DeviceArray.from_host(np.ascontiguousarray(columns, dtype=np.int32)),
                   DeviceArray.from_host(np.ascontiguousarray(values, dtype=np.float64)),
                   int(offsets[-1]) if offsets.size else 0)

    @property
    def nnz(self) -> int:
        """Stored entries (``offsets[nrow]``; read back once)."""
        if self._nnz is None:
            self._nnz = int(self.offsets.view(self.nrow, self.nrow + 1).numpy()[0]) if self.nrow else 0
        return self._nnz

    @property
    def shape(self) -> tuple[int, int]:
        return (self.nrow, self.ncol)

    @property
    def scalar_type(self) -> np.dtype:
        return self.values.dtype

    def with_values(self, values: DeviceArray) -> "CsrMatrix":
        """The same pattern (shared ``offsets``/``columns``) over other values."""
        return CsrMatrix(self.nrow, self.ncol, self.offsets, self.columns, values, self._nnz)

    def to_scipy(self):
        """Host copy as ``scipy.sparse.csr_matrix`` (for inspection and tests)."""
        import scipy.sparse as sp

        offsets = self.offsets.numpy()
        nnz = int(offsets[-1]) if offsets.size else 0
        columns = self.columns.numpy()[:nnz]
        values = self.values.numpy()[:nnz]
        return sp.csr_matrix((values, columns, offsets), shape=self.shape)

    def release(self) -> None:
        """Drop the native solver states (kept by shape for the next operator of this shape) and
        the factorization kept for this operator."""
        if self._solvers:
            from ordito_b200.linalg import retire_solver  # noqa: PLC0415

            for solver in self._solvers.values():
                retire_solver(solver)
        self._solvers.clear()
        if self._factorization is not None:
            self._factorization.close()
            self._factorization = None

    def __del__(self) -> None:
        try:
            self.release()
        except Exception:
            pass
