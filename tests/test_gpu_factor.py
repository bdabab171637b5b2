"""The numeric Cholesky factorisation on the device (``ob_chol_factor``) against the host
multifrontal factorisation of the same analysis (``ob_chol_host_solve``) and the oracle, and the
``sparse_cholesky`` boundary: ``negated``, ``negated=None``, singular components, indefinite
operators (ordito/cholesky.py:538-660)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import _lib, creation
from ordito_b200 import heat as gheat
from ordito_b200 import laplacian as glap
from ordito_b200.array import CsrMatrix
from ordito_b200.cholesky import NotPositiveDefiniteError, sparse_cholesky
from ordito_b200.device import DeviceArray
from tests import meshes

pytestmark = pytest.mark.gpu


def host_factor_solve(matrix: CsrMatrix, vertices: np.ndarray, rhs: np.ndarray, singular: bool) -> np.ndarray:
    """The same ordering and supernodes, factored by the host multifrontal code, one column."""
    A = matrix.to_scipy()
    n = A.shape[0]
    offsets = np.ascontiguousarray(A.indptr, dtype=np.int32)
    columns = np.ascontiguousarray(A.indices, dtype=np.int32)
    values = np.ascontiguousarray(A.data, dtype=np.float64)
    xyz = np.ascontiguousarray(vertices, dtype=np.float32)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(n)
    _lib.call("ob_chol_host_solve", n, offsets.ctypes.data, columns.ctypes.data, values.ctypes.data,
              xyz.ctypes.data, 64, int(singular), b.ctypes.data, x.ctypes.data, None)
    return x


@pytest.mark.parametrize("name", ["ico3", "saddle_graded", "bumpy_sphere", "small_torus", "unreferenced"])
def test_device_factor_solves_as_the_host_factor(gpu, name: str) -> None:
    v, f = meshes.ALL[name]()
    n = v.shape[0]
    ops = gheat.heat_operators(v, f.reshape(-1), method="meshlab")
    rng = np.random.default_rng(2)
    b = rng.random(n)
    for matrix, singular in ((ops.heat_system, False), (ops.poisson_system, True)):
        rhs = b - b.mean() if singular else b
        chol = sparse_cholesky(matrix, v)
        x = DeviceArray.zeros(n, np.float64)
        chol.solve(rhs, x, refine=False)  # the factor alone, no refinement against the operator
        got = x.numpy()
        ref = host_factor_solve(matrix, v, rhs, singular)
        if singular:
            got, ref = got - got.mean(), ref - ref.mean()
        assert hp.relative_linf(got, ref) <= 1e-10


def stored_values(chol) -> np.ndarray:
    count = ctypes.c_longlong(0)
    _lib.call("ob_chol_values", chol.handle, None, 0, ctypes.byref(count), None)
    out = DeviceArray.empty(int(count.value), np.float64)
    _lib.call("ob_chol_values", chol.handle, out.ptr, out.size, ctypes.byref(count), None)
    return out.numpy()


def test_device_factor_is_bit_reproducible(gpu) -> None:
    # Every front entry is summed in a fixed order (no atomics anywhere in the factorisation):
    # two factorisations of one operator store the same values bit for bit.
    v, f = creation.jittered_torus(96, 48, seed=4)
    ops = gheat.heat_operators(v, f.reshape(-1), method="meshlab")
    for matrix in (ops.heat_system, ops.poisson_system):
        first = stored_values(sparse_cholesky(matrix, v))
        second = stored_values(sparse_cholesky(matrix, v))
        assert first.size > 0 and np.isfinite(first).all()
        assert np.array_equal(first, second)


def test_full_size_torus_factor_against_the_oracle(gpu) -> None:
    # The benchmark's mesh (131 072 vertices, 7 tree levels, fronts up to 1 333 rows): the device
    # factors of both systems against the oracle's exact solves, every entry to its own size for
    # the heat system (componentwise refinement), the Poisson solution to 1e-10 of its range.
    v, f = creation.jittered_torus(512, 256, seed=0)
    n = v.shape[0]
    ops = gheat.heat_operators(v, f.reshape(-1), method="meshlab")
    b = np.zeros(n)
    b[[5, 70_000]] = 1.0
    chol = sparse_cholesky(ops.heat_system, v)
    x = DeviceArray.zeros(n, np.float64)
    chol.solve(b, x, componentwise=True)
    got = x.numpy()
    ref = hp.solve_heat(ops.heat_system.to_scipy(), b[:, None])[:, 0]
    mask = ref > 1e-250
    assert np.max(np.abs(got - ref)[mask] / ref[mask]) <= 1e-8
    rng = np.random.default_rng(8)
    r = rng.normal(size=n)
    r -= r.mean()
    poisson = sparse_cholesky(ops.poisson_system, v)
    y = DeviceArray.zeros(n, np.float64)
    poisson.solve(r, y)
    got = y.numpy()
    ref = hp.PoissonFactor(ops.poisson_system.to_scipy()).solve(r)
    assert hp.relative_linf(got - got.mean(), ref - ref.mean()) <= 1e-10


def test_negated_factor_solves_the_operator_itself(gpu) -> None:
    # The cotangent Laplacian is negative semi-definite: negated=True factors -L, and the solve
    # still answers L x = b (consistent b; the constant component is pinned).
    v, f = meshes.bumpy_sphere()
    n = v.shape[0]
    L = glap.cotmatrix(v, f.reshape(-1), dtype=np.float64)
    rng = np.random.default_rng(4)
    b = rng.normal(size=n)
    b -= b.mean()
    for negated in (True, None):
        chol = sparse_cholesky(L, v, negated=negated)
        assert chol.negated
        x = DeviceArray.zeros(n, np.float64)
        chol.solve(b, x)
        got = x.numpy()
        ref = hp.PoissonFactor(-L.to_scipy()).solve(-b)
        assert hp.relative_linf(got - got.mean(), ref - ref.mean()) <= 1e-9
    with pytest.raises(NotPositiveDefiniteError):
        sparse_cholesky(L, v)  # as given, L is not positive definite


def test_negated_none_keeps_a_positive_operator(gpu) -> None:
    v, f = meshes.ALL["ico3"]()
    ops = gheat.heat_operators(v, f.reshape(-1), method="potpourri3d")
    chol = sparse_cholesky(ops.heat_system, v, negated=None)
    assert not chol.negated
    n = v.shape[0]
    x = DeviceArray.zeros(n, np.float64)
    mass = glap.mass_matrix_entries(v, f.reshape(-1), dtype=np.float64).numpy()
    chol.solve(mass, x)
    # M - t L maps the constant 1 to the lumped masses (ordito/cholesky.py:600-612).
    assert np.max(np.abs(x.numpy() - 1.0)) <= 1e-10


def test_indefinite_operator_is_refused(gpu) -> None:
    # [[1, 2], [2, 1]] has a negative eigenvalue: the second pivot is 1 - 4 < 0 either way round.
    matrix = CsrMatrix.from_host([0, 2, 4], [0, 1, 0, 1], [1.0, 2.0, 2.0, 1.0], (2, 2))
    for negated in (False, True):
        with pytest.raises(NotPositiveDefiniteError):
            sparse_cholesky(matrix, negated=negated)
    with pytest.raises(NotPositiveDefiniteError):
        sparse_cholesky(matrix, negated=None)


def test_factor_status_crosses_the_boundary(gpu) -> None:
    # The C ABI reports the bad pivot as OB_ERR_INDEFINITE with a message, not a fault.
    matrix = CsrMatrix.from_host([0, 2, 4], [0, 1, 0, 1], [1.0, 2.0, 2.0, 1.0], (2, 2))
    analysis = ctypes.c_void_p(0)
    _lib.call("ob_chol_analyse", 2, matrix.offsets.ptr, matrix.columns.ptr, None, 0, ctypes.byref(analysis), None)
    try:
        factor = ctypes.c_void_p(0)
        status = _lib.lib.ob_chol_factor(analysis, matrix.values.ptr, 0, 0, ctypes.byref(factor), None)
        assert status == _lib.OB_ERR_INDEFINITE
        assert b"positive definite" in _lib.lib.ob_last_error()
        assert not factor.value
    finally:
        _lib.lib.ob_chol_analysis_destroy(analysis)


def test_cotmatrix_signature_and_weights(gpu) -> None:
    # ordito/laplacian.py:371-378: float32 by default, float64 on request, and the clamped
    # weights with nonnegative_weights (rows still sum to zero, off-diagonals >= 0).
    v, f = meshes.saddle_graded()
    L32 = glap.cotmatrix(v, f.reshape(-1))
    L64 = glap.cotmatrix(v, f.reshape(-1), dtype=np.float64)
    assert L32.scalar_type == np.float32 and L64.scalar_type == np.float64
    a32, a64 = L32.to_scipy(), L64.to_scipy()
    assert np.array_equal(a32.indptr, a64.indptr) and np.array_equal(a32.indices, a64.indices)
    np.testing.assert_allclose(a32.data, a64.data, rtol=1e-6, atol=1e-6 * np.abs(a64.data).max())
    clamped = glap.cotmatrix(v, f.reshape(-1), dtype=np.float64, nonnegative_weights=True).to_scipy()
    off = clamped.copy()
    off.setdiag(0.0)
    assert off.data.min() >= 0.0
    assert np.abs(np.asarray(clamped.sum(axis=1))).max() <= 1e-12 * np.abs(clamped.data).max()
    cot = hp.cotmatrix_entries(v, f.reshape(-1, 3))
    ops = hp.heat_operators(v, f.reshape(-1, 3), 0.0, cot=np.maximum(cot, np.float32(0.0)))
    expected = hp.csr_matrix(ops["pattern"], ops["L"])
    np.testing.assert_allclose(clamped.data, expected.data, rtol=1e-6, atol=1e-6 * np.abs(expected.data).max())
    entries = glap.cotmatrix_entries(v, f.reshape(-1), nonnegative_weights=True).numpy()
    signed = glap.cotmatrix_entries(v, f.reshape(-1)).numpy()
    assert signed.min() < 0.0  # the graded saddle has obtuse angles
    assert np.array_equal(entries, np.maximum(signed, np.float32(0.0)))
    with pytest.raises(ValueError):
        glap.cotmatrix(v, f.reshape(-1), cot_entries=cot.astype(np.float32), nonnegative_weights=True)


def test_deterministic_passes_repeat_bit_for_bit(gpu) -> None:
    """ordito.config.set_deterministic for the factored solves: with the setting on when the
    factors are built, the passes take no atomics (no split tiles; forward updates gathered in
    supernode order), so repeated batches return identical arrays; they agree with the default
    passes to rounding."""
    from ordito_b200 import config
    from ordito_b200.mesh import Trimesh

    v, f = creation.jittered_torus(128, 64, seed=6)
    n = v.shape[0]
    rng = np.random.default_rng(2)
    sets = [[int(s)] for s in rng.choice(n, size=12, replace=False)]
    fast = gheat.heat_geodesic_batch(Trimesh(v, f.reshape(-1)), sets, refine=0).numpy()
    with config.deterministic(True):
        mesh = Trimesh(v, f.reshape(-1))
        first = gheat.heat_geodesic_batch(mesh, sets, refine=0).numpy()
        assert mesh.heat_solver(None, method="meshlab").heat_factor.deterministic
    runs = [gheat.heat_geodesic_batch(mesh, sets, refine=0).numpy() for _ in range(3)]
    for again in runs:
        assert np.array_equal(again, first)
    assert np.max(np.abs(first - fast)) <= 1e-12 * np.abs(fast).max()
    # A single column takes the narrow kernel, with the same tiles.
    one = [gheat.heat_geodesic_batch(mesh, [sets[0]], refine=0).numpy() for _ in range(2)]
    assert np.array_equal(one[0], one[1])


@pytest.mark.parametrize("k", [10, 12, 16, 40, 64])
def test_tile_widths_solve_alike(gpu, k: int) -> None:
    """The 32-column tiles (ob_chol_tile_columns) on every level against the 64-column ones; a
    batch of 9-16 columns takes the 16-column tiles whatever the width, checked against the
    float64 host solve as every width is."""
    v, f = creation.jittered_torus(96, 48, seed=1)
    n = v.shape[0]
    ops = gheat.heat_operators(v, f.reshape(-1), method="meshlab")
    chol = sparse_cholesky(ops.heat_system, v)
    rng = np.random.default_rng(k)
    B = rng.random((n, k))
    answers = []
    for narrow in (0, 64, 2):
        _lib.call("ob_chol_tile_columns", chol.handle, narrow, None)
        x = DeviceArray.zeros(n * k, np.float64)
        chol.solve(B.reshape(-1), x, refine=False)
        answers.append(x.numpy())
    ref = hp.solve_heat(ops.heat_system.to_scipy(), B).reshape(-1)
    for got in answers:
        assert np.max(np.abs(got - answers[0])) <= 1e-12 * np.abs(answers[0]).max()
        assert np.max(np.abs(got - ref)) <= 1e-9 * np.abs(ref).max()
