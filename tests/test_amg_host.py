"""The smoothed-aggregation hierarchy built on the host (no GPU): its shape on the path's
operators, determinism in the seed, and the no-hierarchy case (ordito/linalg.py:6412)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import _lib, creation


def _hierarchy(offsets, columns, values, seed=0):
    rows = (ctypes.c_longlong * 16)()
    nnz = (ctypes.c_longlong * 16)()
    levels = ctypes.c_int(0)
    offsets = np.ascontiguousarray(offsets, np.int32)
    columns = np.ascontiguousarray(columns, np.int32)
    values = np.ascontiguousarray(values, np.float64)
    _lib.call("ob_amg_host_setup", len(offsets) - 1, offsets.ctypes.data, columns.ctypes.data,
              values.ctypes.data, seed, rows, nnz, 16, ctypes.byref(levels))
    count = levels.value
    return [int(r) for r in rows[:max(count, 1)]], [int(z) for z in nnz[:max(count, 1)]], count


def _operators(v, f):
    ops = hp.heat_operators(v, f, hp.vertex_time(v, f, None)[0])
    return ops["pattern"], ops


@pytest.mark.parametrize("system", ["P", "H"])
def test_hierarchy_shape(system: str) -> None:
    v, f = creation.icosphere(5)
    pattern, ops = _operators(v, f)
    rows, nnz, count = _hierarchy(pattern["offsets"], pattern["columns"], ops[system])
    assert count >= 3
    assert rows[0] == v.shape[0] and nnz[0] == int(pattern["offsets"][-1])
    # Each level keeps under 90 % of the rows above it (ordito/linalg.py:6290); the first, over
    # the mesh's own graph, aggregates distance-2 neighbourhoods (several rows an aggregate).
    assert all(b < 0.9 * a for a, b in zip(rows, rows[1:]))
    assert rows[1] * 4 < rows[0]
    assert rows[-1] <= 384


def test_hierarchy_is_a_function_of_the_seed() -> None:
    v, f = creation.jittered_torus(64, 32, seed=0)
    pattern, ops = _operators(v, f)
    a = _hierarchy(pattern["offsets"], pattern["columns"], ops["P"], seed=7)
    b = _hierarchy(pattern["offsets"], pattern["columns"], ops["P"], seed=7)
    c = _hierarchy(pattern["offsets"], pattern["columns"], ops["P"], seed=8)
    assert a == b
    assert c[2] >= 2 and c[0][0] == a[0][0]


def test_uncoarsenable_operator() -> None:
    # A diagonal operator has no off-diagonal entries, so nothing aggregates: up to 512 rows the
    # one level is solved by its dense pseudo-inverse, past that there is no hierarchy (the
    # preconditioner is Jacobi), as ordito/linalg.py:7015-7058 decides.
    rows, nnz, count = _hierarchy(np.arange(501), np.arange(500), np.linspace(1, 2, 500))
    assert count == 1 and rows == [500]
    rows, nnz, count = _hierarchy(np.arange(1001), np.arange(1000), np.linspace(1, 2, 1000))
    assert count == 0


def test_small_operator_is_its_own_coarsest_level() -> None:
    v, f = creation.icosphere(2)  # 162 rows: below the 384-row dense limit
    pattern, ops = _operators(v, f)
    rows, nnz, count = _hierarchy(pattern["offsets"], pattern["columns"], ops["H"])
    assert count == 1 and rows == [162]  # the dense pseudo-inverse is the whole cycle
