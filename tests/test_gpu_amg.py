"""The smoothed-aggregation multigrid and its mixed-precision solve (GPU): the hierarchy's shape,
the V-cycle's symmetry, and float32 CG inside float64 refinement against direct float64 solves
(ordito/linalg.py:5020 multigrid_preconditioner, :1356 solve_spd)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import creation
from ordito_b200 import heat as gheat
from ordito_b200 import laplacian as glap
from ordito_b200 import linalg as glinalg
from ordito_b200.array import CsrMatrix
from ordito_b200.device import DeviceArray
from ordito_b200.mesh import Trimesh
from tests import meshes

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-10  # relative residual of the refined solves
DISTANCE_TOL = 1e-5


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _operators(v, f):
    return gheat.heat_operators(v, f.reshape(-1))


def test_hierarchy_coarsens_the_torus(gpu) -> None:
    v, f = creation.jittered_torus(128, 64, seed=0)
    ops = _operators(v, f)
    for system in (ops.poisson_system, ops.heat_system):
        cycle = glinalg.multigrid_preconditioner(system)
        grid = cycle.grid
        assert not cycle.is_jacobi
        assert grid[0] == v.shape[0] and len(grid) >= 3
        assert all(a > b for a, b in zip(grid, grid[1:]))
        assert grid[-1] <= 384


def test_vcycle_is_symmetric(gpu) -> None:
    v, f = meshes.bumpy_sphere()
    ops = _operators(v, f)
    cycle = glinalg.multigrid_preconditioner(ops.heat_system)
    n = v.shape[0]
    rng = np.random.default_rng(3)
    x, y = rng.normal(size=n), rng.normal(size=n)
    mx, my = DeviceArray.zeros(n, np.float64), DeviceArray.zeros(n, np.float64)
    cycle.matvec(DeviceArray.from_host(x), None, mx, 1.0, 0.0)
    cycle.matvec(DeviceArray.from_host(y), None, my, 1.0, 0.0)
    a, b = float(y @ mx.numpy()), float(x @ my.numpy())
    assert abs(a - b) <= 1e-4 * max(abs(a), abs(b))
    assert float(x @ mx.numpy()) > 0.0  # positive definite on the heat system
    with pytest.raises(ValueError):
        cycle.matvec(DeviceArray.from_host(x), None, mx, 2.0, 0.0)


def test_heat_system_recovers_the_constant(gpu) -> None:
    # ordito/linalg.py:1444-1461: solve_spd(M - tL, M 1) = 1.
    v, f = creation.icosphere(4)
    ops = _operators(v, f)
    mass = glap.mass_matrix_entries(v, f.reshape(-1), dtype=np.float64)
    x = DeviceArray.zeros(v.shape[0], np.float64)
    cycle = glinalg.multigrid_preconditioner(ops.heat_system)
    iters, residual, tol = glinalg.solve_spd(ops.heat_system, mass, x, tol=SOLVE_TOL, preconditioner=cycle)
    assert residual <= SOLVE_TOL
    assert np.allclose(x.numpy(), 1.0, atol=1e-9)


@pytest.mark.parametrize("name", ["torus", "sphere"])
def test_poisson_solve_matches_a_direct_solve(gpu, name: str) -> None:
    if name == "torus":
        v, f = creation.jittered_torus(128, 64, seed=1)
    else:
        v, f = meshes.bumpy_sphere()
    ref = hp.heat_operators(v, f)
    P = hp.csr_matrix(ref["pattern"], ref["P"])
    rng = np.random.default_rng(0)
    b = rng.normal(size=v.shape[0])
    b -= b.mean()  # consistent: orthogonal to the constants
    direct = hp.PoissonFactor(P).solve(b)
    ops = _operators(v, f)
    cycle = glinalg.multigrid_preconditioner(ops.poisson_system)
    x = DeviceArray.zeros(v.shape[0], np.float64)
    iters, residual, _ = glinalg.solve_spd(ops.poisson_system, b, x, tol=SOLVE_TOL, preconditioner=cycle)
    assert residual <= SOLVE_TOL
    got = x.numpy() - x.numpy().mean()
    direct -= direct.mean()
    assert rel_err(got, direct) <= 1e-7
    assert iters < 200


def test_columns_solve_like_single_columns(gpu) -> None:
    v, f = creation.jittered_torus(96, 48, seed=2)
    ops = _operators(v, f)
    n = v.shape[0]
    H = ops.heat_system.to_scipy()
    rng = np.random.default_rng(5)
    k = 37  # pads to 64 device columns
    B = rng.normal(size=(n, k))
    cycle = glinalg.multigrid_preconditioner(ops.heat_system)
    X = DeviceArray.zeros(n * k, np.float64)
    glinalg.solve_spd(ops.heat_system, B.reshape(-1), X, tol=SOLVE_TOL, preconditioner=cycle)
    got = X.numpy().reshape(n, k)
    for c in (0, 17, 36):
        x1 = DeviceArray.zeros(n, np.float64)
        glinalg.solve_spd(ops.heat_system, np.ascontiguousarray(B[:, c]), x1, tol=SOLVE_TOL, preconditioner=cycle)
        assert rel_err(got[:, c], x1.numpy()) <= 1e-8
        assert np.linalg.norm(B[:, c] - H @ got[:, c]) <= SOLVE_TOL * np.linalg.norm(B[:, c])


def test_warm_start_and_zero_rhs(gpu) -> None:
    v, f = creation.icosphere(3)
    ops = _operators(v, f)
    n = v.shape[0]
    cycle = glinalg.multigrid_preconditioner(ops.heat_system)
    x = DeviceArray.zeros(n, np.float64)
    iters, residual, _ = glinalg.solve_spd(ops.heat_system, np.zeros(n), x, tol=SOLVE_TOL, preconditioner=cycle)
    assert iters == 0 and not x.numpy().any()
    mass = glap.mass_matrix_entries(v, f.reshape(-1), dtype=np.float64)
    x = DeviceArray.from_host(np.ones(n))
    iters, residual, _ = glinalg.solve_spd(ops.heat_system, mass, x, tol=1e-8, preconditioner=cycle)
    assert iters <= 2 and residual <= 1e-8


def test_uncoarsenable_operator_takes_jacobi(gpu) -> None:
    # A diagonal operator has no off-diagonal entries: every row is isolated, nothing aggregates,
    # and the preconditioner is Jacobi (ordito/linalg.py:5118).
    n = 1000
    d = np.linspace(1.0, 3.0, n)
    matrix = CsrMatrix.from_host(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), d, (n, n))
    cycle = glinalg.multigrid_preconditioner(matrix)
    assert cycle.is_jacobi and cycle.grid == [n]
    b = np.arange(n, dtype=np.float64)
    x = DeviceArray.zeros(n, np.float64)
    glinalg.solve_spd(matrix, b, x, tol=SOLVE_TOL, preconditioner=cycle)
    assert np.allclose(x.numpy(), b / d, rtol=1e-12)


def test_geodesic_with_multigrid_poisson(gpu) -> None:
    # Heat by the factored float64 solve, Poisson by the mixed-precision multigrid solve.
    v, f = creation.jittered_torus(128, 64, seed=4)
    mesh = Trimesh(v, f.reshape(-1))
    sources = np.array([5, 3000, 7000], dtype=np.int32)
    got = gheat.heat_geodesic_batch(mesh, [[int(s)] for s in sources], poisson="multigrid").numpy()
    ops = hp.heat_operators(v, f, hp.vertex_time(v, f, None)[0])
    for c, s in enumerate(sources):
        ref = hp.heat_geodesic(v, f, np.array([s]), operators=ops)
        assert rel_err(got[c], ref) <= DISTANCE_TOL


def test_time_kernels_reports_each_vcycle_kernel(gpu) -> None:
    """ob_amg_time_kernels: positive times for the finest level's four kernels and the whole
    V-cycle, algorithmic bytes at least the finest operator's stored entries and vectors."""
    import ctypes

    from ordito_b200 import _lib

    v, f = creation.jittered_torus(128, 64, seed=0)
    ops = _operators(v, f)
    cycle = glinalg.multigrid_preconditioner(ops.poisson_system)
    ms = (ctypes.c_float * 5)()
    nbytes = (ctypes.c_longlong * 5)()
    _lib.call("ob_amg_time_kernels", cycle.handle, 64, 2, ms, nbytes, None)
    n, nnz = ops.poisson_system.nrow, ops.poisson_system.nnz
    assert all(ms[i] > 0.0 for i in range(5))
    assert nbytes[0] >= 8 * nnz + 3 * 4 * n * 64
    assert nbytes[1] >= 8 * nnz + 3 * 4 * n * 64
    assert nbytes[2] > 4 * n * 64 and nbytes[3] > 2 * 4 * n * 64
    # The timed kernels leave the hierarchy usable: a solve still converges.
    rhs = np.random.default_rng(0).normal(size=n)
    rhs -= rhs.mean()
    x = DeviceArray.zeros(n, np.float64)
    glinalg.solve_spd(ops.poisson_system, DeviceArray.from_host(rhs), x, tol=1e-8,
                      preconditioner=cycle)
    A = ops.poisson_system.to_scipy()
    assert np.linalg.norm(A @ x.numpy() - rhs) <= 1e-6 * np.linalg.norm(rhs)


@pytest.mark.parametrize("name", ["torus", "sphere"])
def test_device_hierarchy_matches_the_host_build(gpu, name: str) -> None:
    """The levels of 32 768 rows or more built on the device (ob_amg_build_mode(1), the default)
    against the whole build on host threads, same seed: the same aggregates (level sizes and
    stored entries), and the same mixed-precision solve to its refinement's tolerance."""
    import ctypes

    from ordito_b200 import _lib

    if name == "torus":
        v, f = creation.jittered_torus(512, 256, seed=0)
    else:
        v, f = creation.icosphere(7)
    ops = _operators(v, f)
    n = v.shape[0]
    rng = np.random.default_rng(6)
    b = rng.normal(size=n)
    b -= b.mean()
    shapes, answers = [], []
    try:
        for mode in (0, 1):
            _lib.call("ob_amg_build_mode", mode)
            cycle = glinalg.multigrid_preconditioner(ops.poisson_system)
            shapes.append(list(cycle.grid) + [cycle.stored_entries])
            x = DeviceArray.zeros(n, np.float64)
            glinalg.solve_spd(ops.poisson_system, b, x, tol=SOLVE_TOL, preconditioner=cycle)
            answers.append(x.numpy())
            cycle.close()
    finally:
        _lib.call("ob_amg_build_mode", 1)
    assert shapes[0] == shapes[1]
    assert len(shapes[0]) >= 4  # at least two device levels on these meshes
    got, ref = answers[1] - answers[1].mean(), answers[0] - answers[0].mean()
    assert hp.relative_linf(got, ref) <= 1e-8
