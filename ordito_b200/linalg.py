"""Conjugate-gradient solves of the heat path (``ordito.linalg``'s path subset).

``solve_spd`` (ordito/linalg.py:1356), ``solve_spd_settled`` (:2490), ``jacobi_preconditioner``
(:1591), ``chebyshev_preconditioner`` (:5135) and ``multigrid_preconditioner`` (:5020) with the
reference's signatures and contracts: ``solution`` is the initial guess and is overwritten in
place; a solver state is kept per operator for its lifetime, so a later solve replays its recorded
device loop. The iteration runs in ``libordito_b200.so``: ob_pcg_* (Chronopoulos-Gear CG, loop and
stopping tests on the device) for the Jacobi and Chebyshev preconditioners, ob_amg_* (float32 CG
with the float32 smoothed-aggregation V-cycle inside float64 iterative refinement) for multigrid.
Several right-hand sides are laid out ``[n][n_columns]`` (one row's columns contiguous).
"""

from __future__ import annotations

import collections
import ctypes
import threading
import warnings
from typing import Any

import numpy as np

from ordito_b200 import _lib
from ordito_b200.array import CsrMatrix
from ordito_b200.device import DEFAULT_STREAM, DeviceArray, device_pointer, element_count

CG_TOLERANCE = 1e-8
CG_MAXITER_FACTOR = 10  # ordito/linalg.py:172
SETTLE_BACKWARD_ERROR = 1e-6  # :178
SETTLE_DIRECT_TOLERANCE = 1e-12  # :181

_KINDS = {"diag": 0, "chebyshev": 1}

# The mixed-precision multigrid solve: float64 refinement rounds at most, and the relative residual
# each float32 inner CG solve reaches before the next float64 residual is formed.
AMG_MAX_OUTER = 20
AMG_INNER_TOLERANCE = 1e-4
AMG_MAX_INNER = 500


class Preconditioner:
    """A preconditioner this module builds for one operator: Jacobi or Jacobi-Chebyshev.

    Stands in for the ``warp.optim.linear.LinearOperator`` ordito returns; ``solve_spd`` accepts
    it only for the matrix it was built for, as the reference does (linalg.py:1500-1530).
    """

    def __init__(self, matrix: CsrMatrix, kind: str, n_columns: int = 1) -> None:
        self.matrix = matrix
        self.kind = kind
        self.n_columns = n_columns
        self.shape = (matrix.nrow * n_columns, matrix.nrow * n_columns)


class MultigridPreconditioner(Preconditioner):
    """Smoothed-aggregation V-cycle of one operator (ordito/linalg.py:5020).

    The hierarchy (strength 0.05, distance-2 aggregation, l1-Jacobi smoothing with the damping from
    a power iteration, smoothed prolongation, Galerkin coarse operators, a dense pseudo-inverse at
    <= 384 rows) is built once (``ob_amg_setup``: its levels of 32 768 rows or more on the device,
    the rest on the host) and held on the device in float32.
    An operator that does not coarsen gets a Jacobi preconditioner in its place, as the reference
    returns one (ordito/linalg.py:5118-5119); ``grid`` then has a single level. ``matvec(x, y, z,
    1, 0)`` applies one cycle, ``z = M x``; other ``alpha``/``beta`` raise ``ValueError``.
    The matrix's arrays are borrowed and must stay alive (the preconditioner keeps a reference).
    """

    def __init__(self, matrix: CsrMatrix, n_columns: int = 1, *, seed: int = 0) -> None:
        super().__init__(matrix, "multigrid", n_columns)
        handle = ctypes.c_void_p(0)
        _lib.call(
            "ob_amg_setup", matrix.nrow, matrix.offsets.ptr, matrix.columns.ptr,
            matrix.values.ptr, int(seed) & 0xFFFFFFFF, ctypes.byref(handle), DEFAULT_STREAM,
        )  # fmt: skip
        self.handle = handle
        self.seed = seed

    @property
    def grid(self) -> list[int]:
        """Rows per level, coarsest last (one level: the Jacobi fallback)."""
        info = (ctypes.c_longlong * 4)()
        _lib.call("ob_amg_info", self.handle, info)
        levels = max(1, int(info[0]))
        rows = (ctypes.c_longlong * levels)()
        nnz = (ctypes.c_longlong * levels)()
        _lib.call("ob_amg_levels", self.handle, rows, nnz, levels)
        return [int(r) for r in rows]

    @property
    def stored_entries(self) -> int:
        """Stored entries of every level's operator together."""
        info = (ctypes.c_longlong * 4)()
        _lib.call("ob_amg_info", self.handle, info)
        return int(info[3])

    @property
    def is_jacobi(self) -> bool:
        info = (ctypes.c_longlong * 4)()
        _lib.call("ob_amg_info", self.handle, info)
        return int(info[0]) == 0

    def matvec(self, x: Any, y: Any, z: Any, alpha: float, beta: float) -> None:
        if alpha != 1.0 or beta != 0.0:
            raise ValueError(
                "multigrid_preconditioner's operator only implements z = M x "
                f"(got alpha={alpha}, beta={beta})"
            )
        n_columns = _columns(self.matrix, x, z)
        x_ptr, keep_x = device_pointer(x, np.float64)
        z_ptr, keep_z = device_pointer(z, np.float64)
        _lib.call("ob_amg_apply", self.handle, x_ptr, z_ptr, n_columns, n_columns, DEFAULT_STREAM)
        if isinstance(keep_z, DeviceArray) and not hasattr(z, "__cuda_array_interface__"):
            np.copyto(z, keep_z.numpy().reshape(np.shape(z)))
        del keep_x

    def solve(self, rhs: int, x: int, n_columns: int, tol: float, maxiter: int,
              inner_tol: float = AMG_INNER_TOLERANCE,
              max_outer: int = AMG_MAX_OUTER) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Mixed-precision solve of ``n_columns`` systems in place (``ob_amg_solve``)."""
        iters = (ctypes.c_int * n_columns)()
        residual = (ctypes.c_double * n_columns)()
        status = (ctypes.c_int * n_columns)()
        _lib.call(
            "ob_amg_solve", self.handle, rhs, x, n_columns, n_columns, float(tol), int(max_outer),
            int(max(1, min(maxiter, AMG_MAX_INNER))), float(inner_tol), iters, residual, status,
            DEFAULT_STREAM,
        )  # fmt: skip
        return (np.frombuffer(iters, dtype=np.int32).copy(), np.frombuffer(residual).copy(),
                np.frombuffer(status, dtype=np.int32).copy())

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.lib.ob_amg_destroy(self.handle)
            self.handle = ctypes.c_void_p(0)

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


def multigrid_preconditioner(matrix: CsrMatrix, n_columns: int = 1, *,
                             seed: int = 0) -> MultigridPreconditioner:
    """ordito/linalg.py:5020: the smoothed-aggregation V-cycle of ``matrix`` (see the class)."""
    return MultigridPreconditioner(matrix, n_columns, seed=seed)


def jacobi_preconditioner(matrix: CsrMatrix) -> Preconditioner:
    return Preconditioner(matrix, "diag")


def chebyshev_preconditioner(matrix: CsrMatrix, n_columns: int = 1) -> Preconditioner:
    """Degree-12 Jacobi-Chebyshev polynomial on ``[max(min(80/n, .5), 1-r), 1+r]``, ``r`` the
    rows' largest Gershgorin ratio (built on the device at the first solve)."""
    return Preconditioner(matrix, "chebyshev", n_columns)


class NativeSolver:
    """One ``ob_pcg_*`` solver state: its own copy of the operator, work vectors and recorded loop
    graphs. When its matrix is released the state goes back to a pool of kept states by shape,
    and the next operator of that shape is copied into it (``rebind``) and replays its loops."""

    def __init__(self, matrix: CsrMatrix, kind: str, narrow: bool, n_columns: int) -> None:
        handle = ctypes.c_void_p(0)
        _lib.call(
            "ob_pcg_create", matrix.nrow, matrix.offsets.ptr, matrix.columns.ptr,
            matrix.values.ptr, int(n_columns), _KINDS[kind], int(narrow), ctypes.byref(handle),
            DEFAULT_STREAM,
        )  # fmt: skip
        self.handle = handle
        self.n = matrix.nrow
        self.n_columns = n_columns
        self.shape_key = (matrix.nrow, matrix.nnz, kind, bool(narrow), int(n_columns))
        # In the pool of kept states: its finaliser must not close it (a dead matrix's objects
        # are collected as one cycle, whose finalisers all run, after the matrix retired it).
        self.pooled = False

    def rebind(self, matrix: CsrMatrix) -> None:
        _lib.call("ob_pcg_rebind", self.handle, matrix.offsets.ptr, matrix.columns.ptr,
                  matrix.values.ptr, matrix.nnz, DEFAULT_STREAM)

    def close(self) -> None:
        if self.handle and self.handle.value:
            _lib.lib.ob_pcg_destroy(self.handle)
            self.handle = ctypes.c_void_p(0)

    def __del__(self) -> None:
        if getattr(self, "pooled", False):
            return
        try:
            self.close()
        except Exception:
            pass

    def solve(self, rhs: int, x: int, tol: float, maxiter: int) -> tuple[np.ndarray, np.ndarray]:
        iters = (ctypes.c_int * self.n_columns)()
        residual = (ctypes.c_double * self.n_columns)()
        _lib.call("ob_pcg_solve", self.handle, rhs, x, float(tol), int(maxiter), iters, residual,
                  DEFAULT_STREAM)
        return np.frombuffer(iters, dtype=np.int32).copy(), np.frombuffer(residual).copy()

    def settle(self, rhs: int, x: int, check_rounds: int, change_tolerance: float,
               settle_rounds: int, maxiter: int) -> tuple[int, int]:
        rounds, status = ctypes.c_int(0), ctypes.c_int(0)
        _lib.call(
            "ob_pcg_settle", self.handle, rhs, x, int(check_rounds), float(change_tolerance),
            int(settle_rounds), int(maxiter), ctypes.byref(rounds), ctypes.byref(status),
            DEFAULT_STREAM,
        )  # fmt: skip
        return rounds.value, status.value


# Solver states whose matrix was released, kept by shape for the next operator of that shape.
_KEPT: "collections.OrderedDict[tuple, NativeSolver]" = collections.OrderedDict()
_KEPT_LIMIT = 16
_KEPT_LOCK = threading.Lock()


def _solver(matrix: CsrMatrix, kind: str, narrow: bool, n_columns: int) -> NativeSolver:
    key = (kind, bool(narrow), int(n_columns))
    solver = matrix._solvers.get(key)
    if solver is None:
        with _KEPT_LOCK:
            solver = _KEPT.pop((matrix.nrow, matrix.nnz) + key, None)
        if solver is not None:
            solver.pooled = False
            solver.rebind(matrix)
        else:
            solver = NativeSolver(matrix, kind, narrow, n_columns)
        matrix._solvers[key] = solver
    return solver


def retire_solver(solver: Any) -> None:
    """A released matrix's solver state: kept for the next operator of its shape (a bounded
    pool, least recently retired closed first), or closed."""
    if not isinstance(solver, NativeSolver) or not (solver.handle and solver.handle.value):
        return
    closing = []
    solver.pooled = True
    with _KEPT_LOCK:
        previous = _KEPT.pop(solver.shape_key, None)
        if previous is not None:
            closing.append(previous)
        _KEPT[solver.shape_key] = solver
        while len(_KEPT) > _KEPT_LIMIT:
            closing.append(_KEPT.popitem(last=False)[1])
    for old in closing:
        old.pooled = False
        old.close()


def _kind(matrix: CsrMatrix, preconditioner: Preconditioner | None) -> str:
    if preconditioner is None:
        return "diag"
    if not isinstance(preconditioner, Preconditioner) or preconditioner.matrix is not matrix:
        raise ValueError("preconditioner must be one this module built for matrix")
    return preconditioner.kind


def _columns(matrix: CsrMatrix, rhs: Any, solution: Any) -> int:
    n_rhs = element_count(rhs)
    if matrix.nrow == 0 or n_rhs % matrix.nrow or element_count(solution) != n_rhs:
        raise ValueError(
            f"rhs and solution must hold n_columns * {matrix.nrow} entries of one shape"
        )
    return n_rhs // matrix.nrow


def solve_spd(
    matrix: CsrMatrix,
    rhs: Any,
    solution: Any,
    *,
    tol: float = CG_TOLERANCE,
    maxiter: int | None = None,
    check_every: int = 10,
    preconditioner: Preconditioner | None = None,
    name: str = "solve_spd",
    narrow_values: bool = False,
) -> tuple[int, float, float]:
    """Solve one SPD (or consistent semi-definite) system by preconditioned CG, in place.

    Returns ``(iterations, residual, tol)`` with ``residual`` the relative residual |r|/|b|;
    warns (``UserWarning``) when the solve stops outside ``tol``, as ordito/linalg.py:7610 does.
    ``narrow_values`` iterates on float32 copies of the values (float64 vectors and dots). A
    ``multigrid_preconditioner`` runs the mixed-precision solve: float32 CG with the float32
    V-cycle inside float64 iterative refinement to the same relative residual ``tol``.
    """
    n_columns = _columns(matrix, rhs, solution)
    kind = _kind(matrix, preconditioner)
    cap = CG_MAXITER_FACTOR * matrix.nrow if maxiter is None else int(maxiter)
    rhs_ptr, keep_rhs = device_pointer(rhs, np.float64)
    x_ptr, keep_x = device_pointer(solution, np.float64)
    if kind == "multigrid":
        iters, residual, _ = preconditioner.solve(rhs_ptr, x_ptr, n_columns, tol, cap)
    else:
        solver = _solver(matrix, kind, narrow_values, n_columns)
        iters, residual = solver.solve(rhs_ptr, x_ptr, tol, cap)
    if isinstance(keep_x, DeviceArray) and keep_x is not solution and not hasattr(solution, "__cuda_array_interface__"):
        np.copyto(solution, keep_x.numpy().reshape(np.shape(solution)))
    worst = float(np.max(residual)) if residual.size else 0.0
    if check_every > 0 and not worst <= tol:
        warnings.warn(
            f"{name}: conjugate gradient stopped at relative residual {worst:.3g} "
            f"(tolerance {tol:.3g}) after {int(iters.max())} iterations",
            UserWarning,
            stacklevel=2,
        )
    del keep_rhs
    return int(iters.max()), worst, float(tol)


def march_settled(matrix: CsrMatrix, rhs: Any, solution: Any) -> int:
    """Solve ``matrix x = rhs`` band by band, every entry to its own precision (ordito/linalg.py:
    2765 ``_march_settled``; ``ob_march_solve``), into ``solution``, column by column for an
    ``[n][k]`` layout. Returns the band solves' CG rounds."""
    n_columns = _columns(matrix, rhs, solution)
    n = matrix.nrow
    rhs_ptr, keep_rhs = device_pointer(rhs, np.float64)
    x_ptr, keep_x = device_pointer(solution, np.float64)
    info = (ctypes.c_longlong * 3)()
    rounds = 0
    if n_columns == 1:
        _lib.call("ob_march_solve", n, matrix.offsets.ptr, matrix.columns.ptr, matrix.values.ptr,
                  rhs_ptr, x_ptr, info, DEFAULT_STREAM)
        rounds = int(info[1])
    else:
        # [n][k] -> [k][n]: each column contiguous for its march, then back.
        columns_in = DeviceArray.empty((n_columns, n), np.float64)
        columns_out = DeviceArray.empty((n_columns, n), np.float64)
        _lib.call("ob_transpose", n, n_columns, rhs_ptr, columns_in.ptr, DEFAULT_STREAM)
        for c in range(n_columns):
            _lib.call("ob_march_solve", n, matrix.offsets.ptr, matrix.columns.ptr,
                      matrix.values.ptr, columns_in.ptr + 8 * n * c,
                      columns_out.ptr + 8 * n * c, info, DEFAULT_STREAM)
            rounds += int(info[1])
        _lib.call("ob_transpose", n_columns, n, columns_out.ptr, x_ptr, DEFAULT_STREAM)
    if isinstance(keep_x, DeviceArray) and keep_x is not solution and not hasattr(solution, "__cuda_array_interface__"):
        np.copyto(solution, keep_x.numpy().reshape(np.shape(solution)))
    del keep_rhs
    return rounds


def solve_spd_settled(
    matrix: CsrMatrix,
    rhs: Any,
    solution: Any,
    *,
    check_rounds: int,
    change_tolerance: float,
    settle_rounds: int,
    maxiter: int | None = None,
    preconditioner: Preconditioner | None = None,
    factorization: Any = None,
    narrow_values: bool = True,
) -> DeviceArray:
    """Jacobi CG at zero tolerance until every entry has settled relative to itself.

    ordito/linalg.py:2490: a check every ``check_rounds`` rounds stops once no entry is newly
    non-zero and none moved by ``change_tolerance`` of itself, or ``settle_rounds`` rounds after the
    non-zero count last changed, or at ``maxiter``. The settled iterate is then verified by its
    componentwise backward error (``SETTLE_BACKWARD_ERROR``); where it fails and a
    ``factorization`` (``OperatorFactorization``) is given or can be built, the system is solved by
    the sparse Cholesky factorization instead. Returns the ``(1,)`` int32 device array of rounds.
    """
    n_columns = _columns(matrix, rhs, solution)
    if _kind(matrix, preconditioner) != "diag":
        raise ValueError("solve_spd_settled runs under its own Jacobi preconditioner")
    rhs_ptr, keep_rhs = device_pointer(rhs, np.float64)
    x_ptr, keep_x = device_pointer(solution, np.float64)
    if factorization is not None and getattr(factorization, "factorization", None) is not None:
        factorization.solve(rhs, solution, tol=SETTLE_DIRECT_TOLERANCE, componentwise=True)
        return DeviceArray.from_host(np.zeros(1, dtype=np.int32))
    cap = CG_MAXITER_FACTOR * matrix.nrow if maxiter is None else int(maxiter)
    solver = _solver(matrix, "diag", narrow_values, n_columns)
    rounds, status = solver.settle(rhs_ptr, x_ptr, check_rounds, change_tolerance, settle_rounds, cap)
    flag = DeviceArray.empty(1, np.int32)
    _lib.call(
        "ob_backward_error", matrix.nrow, matrix.offsets.ptr, matrix.columns.ptr, matrix.values.ptr,
        x_ptr, rhs_ptr, n_columns, SETTLE_BACKWARD_ERROR, flag.ptr, DEFAULT_STREAM,
    )  # fmt: skip
    verified = int(flag.numpy()[0]) == 0
    if not verified:
        fallback = factorization
        if fallback is None:
            from ordito_b200.cholesky import OperatorFactorization  # noqa: PLC0415

            fallback = OperatorFactorization(matrix)
        fallback.iterate_rejected = True
        if fallback.factor():
            DeviceArray(x_ptr, (matrix.nrow * n_columns,), np.float64, owned=False).fill_zero()
            fallback.solve(rhs, solution, tol=SETTLE_DIRECT_TOLERANCE, componentwise=True)
        else:
            # The factorisation is refused (over the budget): the band march reaches every entry
            # with its own precision (ordito/linalg.py:2574-2590).
            march_settled(matrix, rhs, solution)
    del keep_rhs, keep_x
    return DeviceArray.from_host(np.array([rounds], dtype=np.int32))
