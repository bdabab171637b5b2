"""Sparse Cholesky of the heat path's systems (``ordito.cholesky`` / ``linalg.OperatorFactorization``).

``sparse_cholesky(matrix, coordinates)`` (ordito/cholesky.py:538) returns a ``SparseCholesky`` whose
``solve(rhs, solution, *, tol, componentwise, refine)`` (:427) solves by the factor on the device;
``OperatorFactorization(matrix, coordinates)`` (ordito/linalg.py:2191) is the caller-owned slot a
``HeatSolver`` keeps per system: ``factor()`` builds the factorization (``False`` when it cannot --
over ``CHOLESKY_MEMORY_BUDGET``, or not positive definite), ``solve(rhs, solution)`` solves by it.

The ordering is a nested dissection of the operator's graph (geometric, from the vertex positions
when given) and the supernodes are the dissection tree's nodes; the analysis runs on the host
(``ob_chol_analyse``), the numeric factorisation on the device (``ob_chol_factor``: multifrontal,
level by level, float64 tensor-core products), and the triangular solves on the device, level by
level, as batched dense products over all right-hand sides at once (``ob_chol_solve``). A singular
operator (the Poisson system ``-L``) has one vertex per connected component pinned, so its
solution is the consistent system's up to a constant per component (ordito/cholesky.py:17-20).
"""

from __future__ import annotations

import ctypes
from typing import Any

import numpy as np

from ordito_b200 import _lib, config
from ordito_b200.array import CsrMatrix
from ordito_b200.device import DEFAULT_STREAM, DeviceArray, device_pointer, element_count

CHOLESKY_MEMORY_BUDGET = 4 << 30  # ordito/cholesky.py:74
CHOLESKY_REFINE_ROUNDS = 12  # :72
# Vertices a nested-dissection leaf holds (ordito's CHOLESKY_LEAF_ROWS, :65, is 32 for its own
# supernodes); each leaf is one dense front of the factor.
CHOLESKY_LEAF_ROWS = 64


class NotPositiveDefiniteError(ValueError):
    """A factorization met a non-positive pivot (ordito/cholesky.py:90)."""


class CholeskyAnalysis:
    """The ordering and symbolic structure of one pattern, shareable by every operator on it."""

    def __init__(self, matrix: CsrMatrix, coordinates: Any = None, leaf_size: int | None = None,
                 block: int = 1) -> None:
        """``block`` > 1: the rows come in groups of ``block``, one group a vertex of
        ``coordinates`` (the vector heat system's two tangent components a vertex); each vertex's
        rows stay consecutive in the ordering."""
        if leaf_size is None:
            leaf_size = CHOLESKY_LEAF_ROWS
        handle = ctypes.c_void_p(0)
        xyz = 0
        keep = None
        if coordinates is not None:
            xyz, keep = device_pointer(coordinates, np.float32, 3 * (matrix.nrow // block))
        _lib.call("ob_chol_analyse_blocked", matrix.nrow, int(block), matrix.offsets.ptr,
                  matrix.columns.ptr, xyz, int(leaf_size), ctypes.byref(handle), DEFAULT_STREAM)
        del keep
        self.handle = handle
        info = (ctypes.c_longlong * 5)()
        _lib.call("ob_chol_analysis_info", handle, info)
        self.n, self.supernodes, self.levels, self.factor_entries, self.widest_front = map(int, info)
        self.offsets = matrix.offsets
        self.columns = matrix.columns

    @property
    def factor_bytes(self) -> int:
        return 8 * self.factor_entries

    def close(self) -> None:
        if self.handle and self.handle.value:
            _lib.lib.ob_chol_analysis_destroy(self.handle)
            self.handle = ctypes.c_void_p(0)

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


# ob_chol_factor's singular modes: pin nothing, pin every component, pin the zero-sum ones.
_PIN_NONE, _PIN_ALL, _PIN_ZERO_SUM = 0, 1, 2
# Rows whose diagonal ``sparse_cholesky(negated=None)`` sums to choose the sign it tries first
# (ordito/cholesky.py:78).
_SIGN_PROBE_ROWS = 64


class SparseCholesky:
    """A device-resident factor of one operator (ordito/cholesky.py:121).

    ``singular``: ``False`` pins nothing, ``True`` pins one vertex of every connected component,
    ``None`` pins it on the components whose rows all sum to zero (the reference's rule,
    ordito/cholesky.py:76). ``negated`` factors ``-matrix``; solves still answer ``matrix x = rhs``.
    """

    def __init__(self, matrix: CsrMatrix, analysis: CholeskyAnalysis, *, singular: bool | None = None,
                 negated: bool = False) -> None:
        if analysis.n != matrix.nrow:
            raise ValueError("analysis was built for another operator size")
        mode = _PIN_ZERO_SUM if singular is None else (_PIN_ALL if singular else _PIN_NONE)
        handle = ctypes.c_void_p(0)
        status = _lib.lib.ob_chol_factor(analysis.handle, matrix.values.ptr, mode, int(bool(negated)),
                                         ctypes.byref(handle), DEFAULT_STREAM)
        if status == _lib.OB_ERR_INDEFINITE:
            raise NotPositiveDefiniteError("sparse_cholesky: the operator is not positive definite")
        _lib.check(status, "ob_chol_factor")
        self.handle = handle
        self.matrix = matrix
        self.analysis = analysis
        self.singular = singular is not False
        self.negated = bool(negated)
        # The determinism setting in force when the factorization is built (ordito_b200.config).
        self.deterministic = config.is_deterministic()
        if self.deterministic:
            _lib.call("ob_chol_set_deterministic", handle, 1, DEFAULT_STREAM)

    @property
    def n(self) -> int:
        """Rows of the factored operator."""
        return self.matrix.nrow

    @property
    def nbytes(self) -> int:
        size = ctypes.c_size_t(0)
        _lib.call("ob_chol_nbytes", self.handle, ctypes.byref(size))
        return int(size.value)

    def buffers(self, n_columns: int) -> tuple[int, int]:
        """Device pointers of the factor's own right-hand-side and solution buffers ([n][k])."""
        rhs, sol = ctypes.c_void_p(0), ctypes.c_void_p(0)
        _lib.call("ob_chol_buffers", self.handle, int(n_columns), ctypes.byref(rhs),
                  ctypes.byref(sol), DEFAULT_STREAM)
        return int(rhs.value), int(sol.value)

    def work(self, n_columns: int, stream: Any = None, work_set: int = 0) -> tuple[int, int, int, int, int]:
        """``(B, X, stride, iperm, pinned)`` device pointers of the factor's own buffers (of work
        set ``work_set``, 0 to 2) in its numbering (``ob_chol_work_set``), for pipelines that stay
        in it."""
        b, x, iperm, pinned = (ctypes.c_void_p(0) for _ in range(4))
        stride = ctypes.c_int(0)
        _lib.call("ob_chol_work_set", self.handle, int(work_set), int(n_columns), ctypes.byref(b),
                  ctypes.byref(x), ctypes.byref(stride), ctypes.byref(iperm), ctypes.byref(pinned),
                  stream if stream is not None else DEFAULT_STREAM)
        return int(b.value), int(x.value), int(stride.value), int(iperm.value), int(pinned.value)

    @property
    def generation(self) -> int:
        """Changes whenever the buffers ``work`` points at are reallocated (``ob_chol_work_generation``)."""
        return self.work_generation(0)

    def work_generation(self, work_set: int) -> int:
        value = ctypes.c_longlong(0)
        _lib.call("ob_chol_work_generation_set", self.handle, int(work_set), ctypes.byref(value))
        return int(value.value)

    def solve_in_place(self, n_columns: int, stream: Any = None, work_set: int = 0) -> None:
        """``X = A^-1 B`` on the factor's own buffers (work set ``work_set``), in its numbering
        (no read-back)."""
        _lib.call("ob_chol_solve_in_place_set", self.handle, int(work_set), int(n_columns),
                  stream if stream is not None else DEFAULT_STREAM)

    def solve_in_place_sources(self, n_columns: int, sources: Any, source_offsets: Any,
                               stream: Any = None, work_set: int = 0) -> None:
        """``solve_in_place`` for a right-hand side of source indicators (``ob_seed_permuted`` of
        the same device ``sources`` / ``source_offsets``): the forward pass runs only the
        supernodes the sources reach (``ob_chol_solve_in_place_sources``)."""
        _lib.call("ob_chol_solve_in_place_sources", self.handle, int(work_set), int(n_columns),
                  sources.ptr, source_offsets.ptr, stream if stream is not None else DEFAULT_STREAM)

    def solve_pointers(self, rhs: int, x: int, n_columns: int, refine: int, stream: Any = None) -> None:
        """``x = A^-1 rhs`` for ``n_columns`` interleaved columns ([n][n_columns]) plus ``refine``
        float64 refinement steps, all enqueued on the device (no read-back)."""
        m = self.matrix
        _lib.call("ob_chol_solve", self.handle, rhs, x, int(n_columns), int(refine), m.offsets.ptr,
                  m.columns.ptr, m.values.ptr, stream if stream is not None else DEFAULT_STREAM)

    def solve(self, rhs: Any, solution: Any, *, tol: float = 1e-12, componentwise: bool = False,
              refine: bool = True) -> None:
        """Solve into ``solution``; with ``refine`` iterate ``x += A^-1 (b - A x)`` until the
        componentwise backward error is within ``tol`` (at most ``CHOLESKY_REFINE_ROUNDS``), or
        one step when ``componentwise`` is off (ordito/cholesky.py:427)."""
        n = self.matrix.nrow
        count = element_count(rhs)
        if count % n or element_count(solution) != count:
            raise ValueError("rhs and solution must hold n_columns * n entries of one shape")
        k = count // n
        rhs_ptr, keep_rhs = device_pointer(rhs, np.float64)
        x_ptr, keep_x = device_pointer(solution, np.float64)
        self.solve_pointers(rhs_ptr, x_ptr, k, 1 if refine else 0)
        if refine and componentwise and not self.singular:
            flag = DeviceArray.empty(1, np.int32)
            m = self.matrix
            for _ in range(CHOLESKY_REFINE_ROUNDS):
                _lib.call("ob_backward_error", n, m.offsets.ptr, m.columns.ptr, m.values.ptr,
                          x_ptr, rhs_ptr, k, float(tol), flag.ptr, DEFAULT_STREAM)
                if int(flag.numpy()[0]) == 0:
                    break
                # One more correction: x += A^-1 (b - A x) (the refinement kernel's own form).
                self._refine_once(rhs_ptr, x_ptr, k)
        if isinstance(keep_x, DeviceArray) and not hasattr(solution, "__cuda_array_interface__"):
            np.copyto(solution, keep_x.numpy().reshape(np.shape(solution)))
        del keep_rhs

    def _refine_once(self, rhs_ptr: int, x_ptr: int, k: int) -> None:
        m = self.matrix
        n = m.nrow
        residual = DeviceArray.empty(n * k, np.float64)
        correction = DeviceArray.empty(n * k, np.float64)
        _lib.call("ob_spmv", n, m.offsets.ptr, m.columns.ptr, m.values.ptr, x_ptr, residual.ptr, k,
                  DEFAULT_STREAM)
        _lib.call("ob_axpby", n * k, 1.0, rhs_ptr, -1.0, residual.ptr, residual.ptr, DEFAULT_STREAM)
        self.solve_pointers(residual.ptr, correction.ptr, k, 0)
        _lib.call("ob_axpby", n * k, 1.0, x_ptr, 1.0, correction.ptr, x_ptr, DEFAULT_STREAM)

    def close(self) -> None:
        if self.handle and self.handle.value:
            _lib.lib.ob_chol_destroy(self.handle)
            self.handle = ctypes.c_void_p(0)

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


def _leading_diagonal_negative(matrix: CsrMatrix) -> bool:
    """Whether the diagonal of the first ``_SIGN_PROBE_ROWS`` rows sums below zero
    (ordito/cholesky.py:642-660 tries that sign first)."""
    rows = min(matrix.nrow, _SIGN_PROBE_ROWS)
    if rows == 0:
        return False
    offsets = matrix.offsets.view(0, rows + 1).numpy()
    end = int(offsets[-1])
    columns = matrix.columns.view(0, end).numpy()
    values = matrix.values.view(0, end).numpy()
    total = 0.0
    for r in range(rows):
        span = slice(int(offsets[r]), int(offsets[r + 1]))
        total += float(values[span][columns[span] == r].sum())
    return total < 0.0


def sparse_cholesky(matrix: CsrMatrix, coordinates: Any = None, *, negated: bool | None = False,
                    expandable: bool = False) -> SparseCholesky:
    """Factor ``matrix`` on the device (ordito/cholesky.py:538).

    ``negated`` factors ``-matrix`` (a negative semi-definite operator such as a cotangent
    Laplacian); solves still answer ``matrix x = rhs``. ``negated=None`` factors whichever sign
    is positive definite over one analysis, the sign of the leading diagonal first. A component
    whose rows all sum to zero is solved up to a constant (one of its vertices pinned).
    ``expandable`` orders with leaves of half ``CHOLESKY_LEAF_ROWS`` rows (ordito orders so for a
    later 2 x 2 block expansion of the operator; here it only changes the leaf size).
    Raises ``NotPositiveDefiniteError`` when the operator (with ``negated=None``: either sign) is
    not positive definite."""
    if matrix.nrow != matrix.ncol:
        raise ValueError("sparse_cholesky: matrix must be square")
    if np.dtype(matrix.scalar_type) != np.float64:
        raise ValueError("sparse_cholesky: matrix must hold float64 values")
    leaf = CHOLESKY_LEAF_ROWS // 2 if expandable else CHOLESKY_LEAF_ROWS
    analysis = CholeskyAnalysis(matrix, coordinates, leaf_size=leaf)
    if negated is not None:
        return SparseCholesky(matrix, analysis, singular=None, negated=bool(negated))
    first = _leading_diagonal_negative(matrix)
    try:
        return SparseCholesky(matrix, analysis, singular=None, negated=first)
    except NotPositiveDefiniteError:
        pass
    return SparseCholesky(matrix, analysis, singular=None, negated=not first)


class OperatorFactorization:
    """The factorization slot of one operator (ordito/linalg.py:2191)."""

    def __init__(self, matrix: CsrMatrix, coordinates: Any = None, *, singular: bool | None = None,
                 block: int = 1) -> None:
        self.matrix = matrix
        self.coordinates = coordinates
        self.singular = singular
        self.block = block
        self.factorization: SparseCholesky | None = None
        self.analysis: CholeskyAnalysis | None = None
        self.refused = False
        self.indefinite = False
        self.iterate_rejected = False

    def exceeds_budget(self) -> bool:
        """Whether the factor would exceed ``CHOLESKY_MEMORY_BUDGET`` (asks the analysis)."""
        if self.analysis is None:
            self.analysis = CholeskyAnalysis(self.matrix, self.coordinates, block=self.block)
        return self.analysis.factor_bytes > CHOLESKY_MEMORY_BUDGET

    def factor(self, sharing: "OperatorFactorization | None" = None) -> bool:
        """Build the factorization (reusing ``sharing``'s analysis when it has one)."""
        if self.factorization is not None:
            return True
        if self.refused:
            return False
        if self.analysis is None and sharing is not None and sharing.analysis is not None:
            self.analysis = sharing.analysis
        if self.exceeds_budget():
            self.refused = True
            return False
        try:
            # singular None: the components whose rows all sum to zero are pinned.
            self.factorization = SparseCholesky(self.matrix, self.analysis, singular=self.singular)
        except NotPositiveDefiniteError:
            self.indefinite = True
            self.refused = True
            return False
        return True

    def solve(self, rhs: Any, solution: Any, *, tol: float = 1e-12, componentwise: bool = False) -> None:
        if self.factorization is None:
            raise RuntimeError("OperatorFactorization.solve: no factorization is held")
        self.factorization.solve(rhs, solution, tol=tol, componentwise=componentwise)

    def release(self) -> None:
        if self.factorization is not None:
            self.factorization.close()
            self.factorization = None

    def close(self) -> None:
        self.release()

    @property
    def nbytes(self) -> int:
        return 0 if self.factorization is None else self.factorization.nbytes
