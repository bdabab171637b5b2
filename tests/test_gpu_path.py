"""Parity of the CUDA path with the oracle (GPU): pattern bit-exact, values to 1e-6 relative,
distances to 1e-5 of their range (relative L-infinity), errors and edge cases."""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import _lib, creation
from ordito_b200 import heat as gheat
from ordito_b200 import laplacian as glap
from ordito_b200 import linalg as glinalg
from ordito_b200.mesh import Trimesh
from tests import meshes

pytestmark = pytest.mark.gpu

VALUE_RTOL = 1e-6  # Laplacian / mass values against the float64 oracle (relative)
DISTANCE_TOL = 1e-5  # distance: max |d - d_oracle| / max |d_oracle|
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


@pytest.mark.parametrize("name", sorted(meshes.ALL))
def test_pattern_is_bit_exact(gpu, name: str) -> None:
    v, f = meshes.ALL[name]()
    n = v.shape[0]
    ref = hp.mesh_operator_pattern(f, n)
    got = glap.mesh_operator_pattern(f.reshape(-1), n)
    nnz = int(ref["offsets"][-1])
    assert np.array_equal(got.offsets.numpy(), ref["offsets"])
    assert np.array_equal(got.columns.numpy()[:nnz], ref["columns"])
    assert np.array_equal(got.run_start.numpy()[:nnz], ref["run_start"])
    assert np.array_equal(got.keys.numpy(), ref["keys"])
    order = got.order.numpy()
    in_face = ref["order"] >= 0
    assert np.array_equal(order[in_face], ref["order"][in_face])


def test_pattern_of_a_high_degree_vertex_is_bit_exact(gpu) -> None:
    # A fan of 600 triangles around one vertex: its row holds 1201 keys (each rim edge both ways
    # and the diagonal), far past the short rows of a mesh.
    rim = 600
    angle = np.linspace(0.0, 2.0 * np.pi, rim, endpoint=False)
    v = np.vstack([[0.0, 0.0, 0.0], np.column_stack([np.cos(angle), np.sin(angle), np.zeros(rim)])])
    f = np.array([[0, 1 + i, 1 + (i + 1) % rim] for i in range(rim)], dtype=np.int32)
    n = v.shape[0]
    ref = hp.mesh_operator_pattern(f, n)
    got = glap.mesh_operator_pattern(f.reshape(-1), n)
    nnz = int(ref["offsets"][-1])
    assert np.array_equal(got.offsets.numpy(), ref["offsets"])
    assert np.array_equal(got.columns.numpy()[:nnz], ref["columns"])
    assert np.array_equal(got.run_start.numpy()[:nnz], ref["run_start"])
    assert np.array_equal(got.keys.numpy(), ref["keys"])
    assert np.array_equal(got.order.numpy(), ref["order"])


@pytest.mark.parametrize("name", sorted(meshes.ALL))
def test_face_terms_and_operators(gpu, name: str) -> None:
    v, f = meshes.ALL[name]()
    ref = hp.heat_operators(v, f)
    mesh = Trimesh(v, f.reshape(-1))
    terms = mesh.face_terms
    assert np.allclose(terms.cot.numpy(), ref["cot"], rtol=VALUE_RTOL, atol=1e-6 * np.abs(ref["cot"]).max())
    assert np.allclose(terms.normals.numpy(), ref["normals"], atol=1e-6)
    assert np.allclose(terms.areas.numpy(), ref["areas"], rtol=VALUE_RTOL)
    # The corner sums are exact float64 sums of the device's own float32 areas (order-free), and
    # inherit those areas' rounding against the oracle's.
    own = hp.area_sums(f, terms.areas.numpy(), v.shape[0])
    assert np.array_equal(terms.area_sums.numpy(), own)
    assert np.allclose(terms.area_sums.numpy(), ref["area_sums"], rtol=VALUE_RTOL)
    built = glap.assemble_rows(
        mesh.mesh_operator_pattern, mesh.vertices, terms.cot, terms.area_sums, t=None, face_edges=True
    )
    nnz = int(ref["pattern"]["offsets"][-1])
    scale = np.abs(ref["L"]).max()
    for key, matrix in (("L", built.laplacian), ("H", built.heat), ("P", built.poisson)):
        got = matrix.values.numpy()[:nnz]
        assert np.allclose(got, ref[key], rtol=VALUE_RTOL, atol=VALUE_RTOL * scale), key
    # The mass is a third of those exact sums; against the oracle it carries the areas' rounding
    # (a needle's float32 area can differ by an ulp from the oracle's).
    assert np.allclose(built.mass.numpy(), own / 3.0, rtol=1e-15, atol=0.0)
    assert np.allclose(built.mass.numpy(), ref["mass"], rtol=VALUE_RTOL)
    total, count = built.edge_sums.numpy()
    # Each length is a float32 sqrt of a float32 dot (fused on the device): h agrees to a few
    # float32 ulps averaged over the edges.
    assert total / count == pytest.approx(np.sqrt(ref["t"]), rel=VALUE_RTOL)


def test_golden_ico3_fixture(gpu) -> None:
    g = np.load(os.path.join(GOLDEN, "oracle_ico3.npz"))
    d = gheat.heat_geodesic(g["vertices"], g["faces"].reshape(-1), np.array([0], dtype=np.int32))
    assert rel_err(d.numpy(), g["distance"]) <= DISTANCE_TOL


@pytest.mark.parametrize(
    ("name", "sources"),
    [("ico3", [0]), ("saddle_graded", [17]), ("bumpy_sphere", [5]), ("small_torus", [0, 400, 900]),
     ("grid", [3]), ("unreferenced", [1]), ("sphere_irregular", [0, 250]), ("torus_irregular", [7])],
)
def test_heat_geodesic_matches_the_oracle(gpu, name: str, sources: list[int]) -> None:
    v, f = meshes.ALL[name]()
    ref = hp.heat_geodesic(v, f, np.array(sources))
    got = gheat.heat_geodesic(v, f.reshape(-1), np.array(sources, dtype=np.int32)).numpy()
    # A vertex no face references has no equation: its value is the Poisson solution's arbitrary
    # constant (each solver picks its own) less the shift, not a distance. Compare the rest.
    referenced = np.zeros(v.shape[0], dtype=bool)
    referenced[f.reshape(-1)] = True
    assert rel_err(got[referenced], ref[referenced]) <= DISTANCE_TOL


def test_icosphere5_single_source(gpu) -> None:
    v, f = creation.icosphere(5)
    ref = hp.heat_geodesic(v, f, np.array([0]))
    got = gheat.heat_geodesic(v, f.reshape(-1), np.array([0], dtype=np.int32)).numpy()
    assert got[0] == 0.0
    assert rel_err(got, ref) <= DISTANCE_TOL


def test_trimesh_reuses_its_solver(gpu) -> None:
    v, f = meshes.small_torus()
    mesh = Trimesh(v, f.reshape(-1))
    for src in ([0], [123], [5, 600]):
        ref = hp.heat_geodesic(v, f, np.array(src))
        got = gheat.heat_geodesic(mesh, np.array(src, dtype=np.int32)).numpy()
        assert rel_err(got, ref) <= DISTANCE_TOL
    assert len(mesh._solvers) == 1


def test_out_of_range_sources_raise(gpu) -> None:
    v, f = creation.icosphere(1)
    with pytest.raises(ValueError):
        gheat.heat_geodesic(v, f.reshape(-1), np.array([0, v.shape[0]], dtype=np.int32))
    with pytest.raises(ValueError):
        gheat.heat_geodesic(v, f.reshape(-1), np.array([-1], dtype=np.int32))


def test_empty_inputs_return_zero_fields(gpu) -> None:
    v, f = creation.icosphere(1)
    out = gheat.heat_geodesic(v, f.reshape(-1), np.zeros(0, dtype=np.int32))
    assert out.shape == (v.shape[0],) and not out.numpy().any()
    empty = gheat.heat_geodesic(v, np.zeros(0, dtype=np.int32), np.array([0], dtype=np.int32))
    assert not empty.numpy().any()


def test_solve_spd_recovers_the_constant(gpu) -> None:
    v, f = creation.icosphere(2)
    ops = gheat.heat_operators(v, f.reshape(-1))
    mass = glap.mass_matrix_entries(v, f.reshape(-1), dtype=np.float64)
    x = glap.DeviceArray.zeros(v.shape[0], np.float64)
    iters, residual, tol = glinalg.solve_spd(ops.heat_system, mass, x)
    assert residual <= tol
    assert np.allclose(x.numpy(), 1.0, atol=1e-6)


def test_poisson_solve_matches_a_direct_solve(gpu) -> None:
    v, f = meshes.bumpy_sphere()
    ref = hp.heat_operators(v, f)
    P = hp.csr_matrix(ref["pattern"], ref["P"])
    rng = np.random.default_rng(0)
    b = rng.normal(size=v.shape[0])
    b -= b.mean()
    direct = hp.PoissonFactor(P).solve(b)
    ops = gheat.heat_operators(v, f.reshape(-1))
    x = glap.DeviceArray.zeros(v.shape[0], np.float64)
    glinalg.solve_spd(ops.poisson_system, b, x, tol=1e-10, preconditioner=ops.poisson_preconditioner)
    got = x.numpy()
    got -= got.mean()
    direct -= direct.mean()
    assert rel_err(got, direct) <= 1e-6


def test_launches_are_counted(gpu) -> None:
    before = _lib.launch_count()
    v, f = creation.icosphere(2)
    gheat.heat_geodesic(v, f.reshape(-1), np.array([0], dtype=np.int32))
    assert _lib.launch_count() - before >= 10


def test_freed_memory_stays_in_the_pool_and_counts_as_free(gpu) -> None:
    # The library's pool keeps freed memory across synchronisations (reused by the next call
    # without mapping pages again) instead of handing it back to the driver; ob_mem_info adds the
    # pool's unused reservation to the driver's free count; ob_mem_trim hands it back. Read
    # against the pool's and the driver's own counts, so other live allocations do not matter.
    import ctypes

    from cuda.bindings import driver

    from ordito_b200.device import synchronize, trim_pool

    assert driver.cuInit(0)[0] == driver.CUresult.CUDA_SUCCESS

    def counts() -> dict:
        free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
        _lib.call("ob_mem_info", ctypes.byref(free), ctypes.byref(total))
        err, driver_free, _ = driver.cuMemGetInfo()
        assert err == driver.CUresult.CUDA_SUCCESS
        err, device = driver.cuCtxGetDevice()
        err, pool = driver.cuDeviceGetDefaultMemPool(device)
        attr = driver.CUmemPool_attribute
        reserved = int(driver.cuMemPoolGetAttribute(pool, attr.CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT)[1])
        used = int(driver.cuMemPoolGetAttribute(pool, attr.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)[1])
        threshold = int(driver.cuMemPoolGetAttribute(pool, attr.CU_MEMPOOL_ATTR_RELEASE_THRESHOLD)[1])
        return {"free": int(free.value), "driver_free": int(driver_free), "reserved": reserved,
                "used": used, "threshold": threshold}

    size = 256 << 20
    ptr = ctypes.c_void_p(0)
    _lib.call("ob_malloc", size, ctypes.byref(ptr), None)
    held = counts()
    assert held["threshold"] == 2**64 - 1, held
    _lib.call("ob_free", ptr, None)
    synchronize()
    freed = counts()
    assert freed["used"] <= held["used"] - size, (held, freed)  # freed into the pool
    assert freed["driver_free"] < held["driver_free"] + size, (held, freed)  # and kept there
    assert freed["free"] == freed["driver_free"] + max(0, freed["reserved"] - freed["used"]), freed
    trim_pool(0)
    trimmed = counts()
    # What trimming can hand back depends on how the pool laid out other live allocations.
    assert trimmed["reserved"] <= freed["reserved"], (freed, trimmed)
    assert trimmed["driver_free"] >= freed["driver_free"], (freed, trimmed)


def test_solver_state_rebinds_to_an_operator_of_the_same_shape(gpu) -> None:
    # A released operator's solver state serves the next operator of its shape (its own copy of
    # the operator, rebound, its recorded loop replayed): the answers are the new operator's.
    import scipy.sparse.linalg as spla

    v, f = creation.icosphere(3)
    n = v.shape[0]
    rng = np.random.default_rng(2)
    b = rng.normal(size=n)
    for t in (1e-3, 4e-3):
        ops = gheat.heat_operators(v, f.reshape(-1), t)
        x = glap.DeviceArray.zeros(n, np.float64)
        glinalg.solve_spd(ops.heat_system, b, x, tol=1e-12)
        exact = spla.spsolve(ops.heat_system.to_scipy().tocsc(), b)
        assert rel_err(x.numpy(), exact) <= 1e-9
        ops.heat_system.release()  # the state goes back to the pool for the next t


def test_single_query_with_held_factors(gpu) -> None:
    v, f = meshes.small_torus()
    n = v.shape[0]
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    assert solver.factor()
    for sources in ([3], [0, 17, 40], list(range(0, n, 7))):
        got = gheat.heat_geodesic(mesh, np.array(sources, dtype=np.int32), method="meshlab").numpy()
        batch = gheat.heat_geodesic_batch(mesh, [sources], refine=0).numpy()[0]
        assert rel_err(got, batch) <= 1e-12
        assert rel_err(got, hp.heat_geodesic(v, f, np.array(sources))) <= DISTANCE_TOL
    device_sources = glap.DeviceArray.from_host(np.array([5, 9], dtype=np.int32))
    got = gheat.heat_geodesic(mesh, device_sources, method="meshlab").numpy()
    assert rel_err(got, hp.heat_geodesic(v, f, np.array([5, 9]))) <= DISTANCE_TOL
    with pytest.raises(ValueError):
        gheat.heat_geodesic(mesh, np.array([n], dtype=np.int32), method="meshlab")


@pytest.mark.parametrize(("name", "t"), [("sphere_irregular", None), ("saddle_graded", None),
                                         ("sphere_irregular", 0.05), ("torus_irregular", None)])
def test_device_heat_operators_are_the_matrices_they_name(gpu, name: str, t) -> None:
    """ordito tests/test_heat.py:126-188 on the device's operators (the reference's default
    method, potpourri3d): P is -L bit for bit, L is the float64 cotmatrix bit for bit, H is M - t L
    for one t (read off an off-diagonal entry) to 1e-12, that t is the squared mean unique edge
    length to 1e-6 (or the explicit t as given), normals and areas match a float64 computation
    from the same float32 positions to 1e-5."""
    from ordito_b200 import laplacian as glap

    v, f = meshes.ALL[name]()
    ops = gheat.heat_operators(v, f.reshape(-1), t)
    L = ops.laplacian.to_scipy().toarray()
    H = ops.heat_system.to_scipy().toarray()
    P = ops.poisson_system.to_scipy().toarray()
    assert np.array_equal(L, glap.cotmatrix(v, f.reshape(-1), dtype=np.float64).to_scipy().toarray())
    assert np.array_equal(P, -L)
    row, col = np.argwhere(np.triu(L, k=1) != 0.0)[0]
    diffusion_time = float(-H[row, col] / L[row, col])
    v64, f64 = v.astype(np.float64), f.astype(np.int64)
    edges = np.unique(np.sort(np.concatenate([f64[:, [0, 1]], f64[:, [1, 2]], f64[:, [2, 0]]]), axis=1), axis=0)
    unique_mean = float(np.linalg.norm(v64[edges[:, 0]] - v64[edges[:, 1]], axis=1).mean())
    assert np.isclose(diffusion_time, unique_mean**2 if t is None else t, rtol=1e-6, atol=0.0)
    if t is not None:
        diffusion_time = t
    mass = glap.mass_matrix_entries(v, f.reshape(-1), dtype=np.float64).numpy()
    assert np.allclose(H, np.diag(mass) - diffusion_time * L, rtol=1e-12, atol=1e-15)
    corners = v64[f64]
    cross = np.cross(corners[:, 1] - corners[:, 0], corners[:, 2] - corners[:, 0])
    norm = np.linalg.norm(cross, axis=1)
    assert ops.cot_entries.shape == (f.shape[0], 3)
    assert np.allclose(ops.face_normals.numpy().reshape(-1, 3), cross / norm[:, None], rtol=1e-5, atol=1e-5)
    assert np.allclose(ops.face_areas.numpy(), 0.5 * norm, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("name", ["saddle_graded", "sphere_irregular", "torus_irregular"])
def test_device_distance_is_zero_at_the_source_and_nonnegative(gpu, name: str) -> None:
    """ordito tests/test_heat.py:653-663, and against the oracle, on the reference's fixtures."""
    v, f = meshes.ALL[name]()
    d = gheat.heat_geodesic(v, f.reshape(-1), np.array([0], dtype=np.int32)).numpy()
    assert np.all(d >= -1e-6)
    assert abs(d[0]) <= 1e-4
    assert hp.relative_linf(d, hp.heat_geodesic(v, f, np.array([0]))) <= 1e-5


def test_torch_cuda_tensors_cross_zero_copy(gpu) -> None:
    """Arrays from another framework (PyTorch CUDA tensors, through __cuda_array_interface__) are
    read in place, and ``solution`` is written in place: its pointer is the tensor's own."""
    import torch

    from ordito_b200.device import device_pointer

    v, f = creation.icosphere(3)
    n = v.shape[0]
    tv = torch.from_numpy(v).cuda()
    tf = torch.from_numpy(f.reshape(-1).copy()).cuda()
    ts = torch.tensor([0], dtype=torch.int32, device="cuda")
    for tensor, dtype in ((tv, np.float32), (tf, np.int32), (ts, np.int32)):
        pointer, keep = device_pointer(tensor, dtype)
        assert pointer == tensor.data_ptr() and keep is tensor
    distance = gheat.heat_geodesic(tv, tf, ts).numpy()
    assert hp.relative_linf(distance, gheat.heat_geodesic(v, f.reshape(-1), np.array([0], dtype=np.int32)).numpy()) == 0.0
    assert hp.relative_linf(distance, hp.heat_geodesic(v, f, np.array([0]))) <= 1e-5
    # solve_spd warm-starts from `solution` and writes it in place.
    ops = gheat.heat_operators(tv, tf)
    mass = torch.from_numpy(glap.mass_matrix_entries(v, f.reshape(-1), dtype=np.float64).numpy()).cuda()
    solution = torch.zeros(n, dtype=torch.float64, device="cuda")
    before = solution.data_ptr()
    glinalg.solve_spd(ops.heat_system, mass, solution, tol=1e-12, preconditioner=ops.heat_preconditioner)
    torch.cuda.synchronize()
    assert solution.data_ptr() == before
    assert torch.max(torch.abs(solution - 1.0)).item() <= 1e-9
    # A tensor of the wrong dtype is refused, not converted behind the caller's back.
    with pytest.raises(ValueError):
        gheat.heat_geodesic(tv.double(), tf, ts)
