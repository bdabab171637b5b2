"""Sparse Cholesky of the heat path's systems (``ordito.cholesky`` / ``linalg.OperatorFactorization``).

``OperatorFactorization(matrix, coordinates)`` is the caller-owned slot a ``HeatSolver`` keeps per
system (ordito/linalg.py:2191): ``factor()`` builds the factorization (False when it cannot:
over the memory budget, or not positive definite), ``solve(rhs, solution)`` solves by it.
"""

from __future__ import annotations

from typing import Any

from ordito_b200.array import CsrMatrix

CHOLESKY_MEMORY_BUDGET = 4 << 30  # ordito/cholesky.py:74


class NotPositiveDefiniteError(ValueError):
    """A factorization met a non-positive pivot (ordito/cholesky.py:90)."""


class OperatorFactorization:
    """The factorization slot of one operator."""

    def __init__(self, matrix: CsrMatrix, coordinates: Any = None) -> None:
        self.matrix = matrix
        self.coordinates = coordinates
        self.factorization: Any = None
        self.refused = True
        self.iterate_rejected = False

    def factor(self, sharing: "OperatorFactorization | None" = None) -> bool:
        """Build the factorization; returns whether one is held."""
        return False

    def solve(self, rhs: Any, solution: Any, *, tol: float = 1e-12,
              componentwise: bool = False) -> None:
        raise RuntimeError("OperatorFactorization.solve: no factorization is held")

    def release(self) -> None:
        self.factorization = None

    def close(self) -> None:
        self.release()

    @property
    def nbytes(self) -> int:
        return 0
