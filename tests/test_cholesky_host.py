"""The sparse Cholesky's ordering, numeric factorisation and solve algorithm, run on the host
(``ob_chol_host_solve``) against scipy's direct solves. No device needed."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import _lib, creation
from tests import meshes


def host_solve(pattern, values, vertices, singular, rhs, coordinates=True, leaf_size=0):
    n = pattern["offsets"].size - 1
    off = np.ascontiguousarray(pattern["offsets"], dtype=np.int32)
    col = np.ascontiguousarray(pattern["columns"], dtype=np.int32)
    val = np.ascontiguousarray(values[: off[-1]], dtype=np.float64)
    xyz = np.ascontiguousarray(vertices, dtype=np.float32)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(n)
    info = (ctypes.c_longlong * 4)()
    _lib.call("ob_chol_host_solve", n, off.ctypes.data, col.ctypes.data, val.ctypes.data,
              xyz.ctypes.data if coordinates else None, int(leaf_size), int(singular),
              b.ctypes.data, x.ctypes.data, info)
    return x, [int(i) for i in info]


CASES = sorted(meshes.ALL) + ["ico5"]


def load(name):
    return creation.icosphere(5) if name == "ico5" else meshes.ALL[name]()


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("coordinates", [True, False])
def test_heat_system_solve_is_componentwise_exact(name: str, coordinates: bool) -> None:
    v, f = load(name)
    ops = hp.heat_operators(v, f)
    H = hp.csr_matrix(ops["pattern"], ops["H"])
    u0 = np.zeros(v.shape[0])
    u0[min(3, v.shape[0] - 1)] = 1.0
    x, info = host_solve(ops["pattern"], ops["H"], v, False, u0, coordinates)
    ref = hp.HeatFactor(H).solve(u0)
    mask = ref > 1e-250
    assert np.max(np.abs(x - ref)[mask] / ref[mask]) <= 1e-10
    assert info[0] == v.shape[0] and info[2] >= 1


@pytest.mark.parametrize("name", CASES)
def test_singular_poisson_system_is_solved_up_to_a_constant(name: str) -> None:
    v, f = load(name)
    ops = hp.heat_operators(v, f)
    pattern = ops["pattern"]
    P = hp.csr_matrix(pattern, ops["P"])
    active = np.diff(pattern["offsets"]) > 0
    rng = np.random.default_rng(1)
    b = rng.normal(size=v.shape[0])
    b[~active] = 0.0
    b[active] -= b[active].mean()
    x, _ = host_solve(pattern, ops["P"], v, True, b)
    ref = hp.PoissonFactor(P).solve(b)
    x = x[active] - x[active].mean()
    ref = ref[active] - ref[active].mean()
    assert hp.relative_linf(x, ref) <= 1e-9


def test_an_indefinite_operator_is_refused() -> None:
    v, f = creation.icosphere(2)
    ops = hp.heat_operators(v, f)
    with pytest.raises(_lib.CudaError):
        # -H is negative definite: the first pivot is negative.
        host_solve(ops["pattern"], -ops["H"], v, False, np.ones(v.shape[0]))


def _host_analysis_nodes(pattern, vertices):
    n = pattern["offsets"].size - 1
    off = np.ascontiguousarray(pattern["offsets"], dtype=np.int32)
    col = np.ascontiguousarray(pattern["columns"], dtype=np.int32)
    xyz = np.ascontiguousarray(vertices, dtype=np.float32)
    handle = ctypes.c_void_p(0)
    _lib.call("ob_chol_host_analyse", n, off.ctypes.data, col.ctypes.data, xyz.ctypes.data, 0,
              ctypes.byref(handle))
    try:
        info = (ctypes.c_longlong * 5)()
        _lib.call("ob_chol_analysis_info", handle, info)
        nodes = np.zeros((int(info[1]), 4), dtype=np.int32)
        _lib.call("ob_chol_analysis_nodes", handle, nodes.ctypes.data)
        return [int(i) for i in info], nodes
    finally:
        _lib.lib.ob_chol_analysis_destroy(handle)


def test_threaded_analysis_of_a_large_mesh_is_reproducible_and_solves() -> None:
    """A mesh past the sizes where the analysis spreads its adjacency and symbolic passes over
    host threads (65 536 vertices, 262 144 entries): two analyses give the same supernodes, the
    tree is consistent, and the host solve through it matches the oracle componentwise."""
    v, f = creation.jittered_torus(384, 192, seed=3)
    assert v.shape[0] > 1 << 16
    ops = hp.heat_operators(v, f)
    pattern = ops["pattern"]
    assert pattern["offsets"][-1] > 1 << 18
    info, nodes = _host_analysis_nodes(pattern, v)
    again_info, again = _host_analysis_nodes(pattern, v)
    assert info == again_info and np.array_equal(nodes, again)
    level, count, _, parent = nodes.T
    assert info[0] == v.shape[0] and int(count.sum()) == v.shape[0]
    has_parent = parent >= 0
    assert np.all(level[parent[has_parent]] > level[has_parent])
    assert int(level.max()) + 1 == info[2]
    u0 = np.zeros(v.shape[0])
    u0[17] = 1.0
    x, _ = host_solve(pattern, ops["H"], v, False, u0)
    ref = hp.HeatFactor(hp.csr_matrix(pattern, ops["H"])).solve(u0)
    mask = ref > 1e-250
    assert np.max(np.abs(x - ref)[mask] / ref[mask]) <= 1e-10
