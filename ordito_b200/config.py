"""Runtime configuration: whether the factored solves repeat bit for bit (ordito/config.py).

``set_deterministic(True)`` makes every factorization built from then on (and kept by a
``HeatSolver`` or ``PackedMeshes`` built then) take deterministic passes: no split tiles and no
atomics in its triangular solves (``ob_chol_set_deterministic``), so repeated solves return
identical arrays. Off (the default) the passes split the long inner dimensions of the upper tree
levels and accumulate them, and the forward updates of siblings into shared rows, atomically:
faster, equal to rounding. The rest of the path is deterministic either way (the numeric
factorisation sums every front entry in a fixed order, the divergence gathers each vertex's
corners in ascending order, the shifts and the CG dots fold their partials in a fixed order).

As in the reference, the setting is read when a factorization is built: state a ``Trimesh`` caches
keeps the mode it was built in, and a recorded pass keeps the mode it was recorded with.
``deterministic(...)`` overrides the process default for the current thread or task only.
"""

from __future__ import annotations

import contextlib
import contextvars
from collections.abc import Generator

_process_default = False
_override: contextvars.ContextVar[bool | None] = contextvars.ContextVar("ordito_b200_deterministic", default=None)


def set_deterministic(enabled: bool) -> None:
    """Set the process-wide default for reproducible results (ordito/config.py:125)."""
    global _process_default
    _process_default = bool(enabled)


def is_deterministic() -> bool:
    """The innermost active ``deterministic`` override of this thread or task, else the default."""
    override = _override.get()
    return _process_default if override is None else override


@contextlib.contextmanager
def deterministic(enabled: bool = True) -> Generator[None, None, None]:
    """Override the setting within a ``with`` block (this thread or task only; nests)."""
    token = _override.set(bool(enabled))
    try:
        yield
    finally:
        _override.reset(token)
