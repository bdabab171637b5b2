"""``method="igl"`` and ``method="potpourri3d"`` on the CUDA path against the oracle (GPU).

igl: the Voronoi lumped mass (the heat system at t = 0 is its mass), the rim-pinned heat, and the
distance with its Neumann/pinned average (ordito/heat.py:594-597, 4153-4233; the reference's
tests/test_heat.py:266-290, 436-490). potpourri3d: geometry-central's regularized Poisson system
-L + 1e-6 I (ordito/heat.py:3124-3129, 4086-4116)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import creation
from ordito_b200 import heat as gheat
from ordito_b200.device import DeviceArray
from ordito_b200.mesh import Trimesh
from tests import meshes

pytestmark = pytest.mark.gpu

VALUE_RTOL = 1e-6  # mass values against the float64 oracle (relative)
DISTANCE_TOL = 1e-5  # distance: max |d - d_oracle| / range of d_oracle


def _range_err(got: np.ndarray, ref: np.ndarray) -> float:
    return float(np.max(np.abs(got - ref)) / np.ptp(ref))


@pytest.mark.parametrize("name", ["bumpy_sphere", "saddle_graded"])
def test_igl_heat_system_at_zero_time_is_the_voronoi_mass(gpu, name: str) -> None:
    v, f = getattr(meshes, name)()
    n = v.shape[0]
    ops = gheat.heat_operators(v, f.reshape(-1), t=0.0, method="igl")
    H = ops.heat_system.to_scipy().toarray()
    mass = hp.voronoi_area_sums(v, f, n)
    assert np.allclose(np.diag(H), mass, rtol=VALUE_RTOL, atol=1e-12)
    assert not (H - np.diag(np.diag(H))).any()
    barycentric = gheat.heat_operators(v, f.reshape(-1), t=0.0, method="meshlab").heat_system
    gap = np.abs(np.diag(barycentric.to_scipy().toarray()) - mass).max()
    assert gap > 1e-3 * mass.max()


@pytest.mark.parametrize("method", ["igl", "potpourri3d"])
@pytest.mark.parametrize("name,source", [("bumpy_sphere", "first"), ("saddle_graded", "first"),
                                         ("saddle_graded", "middle")])
def test_heat_geodesic_method_matches_the_oracle(gpu, method: str, name: str, source: str) -> None:
    v, f = getattr(meshes, name)()
    n = v.shape[0]
    src = np.array([0 if source == "first" else n // 2 + 17], dtype=np.int32)
    ref = hp.heat_geodesic(v, f, src, method=method)
    assert np.ptp(ref) > 0.5  # the distance propagated
    got = gheat.heat_geodesic(v, f.reshape(-1), src, method=method).numpy()
    assert _range_err(got, ref) <= DISTANCE_TOL
    # The Trimesh form keeps the solver and its extra systems, and answers the same on a second
    # call, which runs on the factorizations the first earned.
    mesh = Trimesh(v, f.reshape(-1))
    for _ in range(2):
        again = gheat.heat_geodesic(mesh, src, method=method).numpy()
        assert _range_err(again, ref) <= DISTANCE_TOL
    mesh.dispose()


def test_the_method_choices_matter(gpu) -> None:
    # From the saddle's middle the rim average and the Voronoi mass move the answer well past
    # the tolerance, and geometry-central's regularization moves it measurably.
    v, f = meshes.saddle_graded()
    src = np.array([v.shape[0] // 2 + 17], dtype=np.int32)
    meshlab = gheat.heat_geodesic(v, f.reshape(-1), src).numpy()
    igl = gheat.heat_geodesic(v, f.reshape(-1), src, method="igl").numpy()
    assert _range_err(igl, meshlab) > 1e-3
    gc = gheat.heat_geodesic(v, f.reshape(-1), src, method="potpourri3d").numpy()
    assert _range_err(gc, meshlab) > 1e-6


def test_diffuse_pinned_holds_the_rim_at_zero(gpu) -> None:
    # The pinned solve is zero on the rim and solves the heat system restricted to the interior
    # (the reference's test_heat_solver_diffuse_pinned_holds_the_rim_at_zero: a point source, the
    # solver's default discretization, against a direct solve).
    v, f = meshes.saddle_graded()
    n = v.shape[0]
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver()
    rhs = np.zeros(n)
    rhs[n // 2 + 17] = 1.0
    out = DeviceArray.zeros(n, np.float64)
    assert solver.diffuse_pinned(DeviceArray.from_host(rhs), out)
    got = out.numpy()
    ops = hp.heat_operators(v, f, hp.vertex_time(v, f, None, "potpourri3d")[0], method="potpourri3d")
    rim = hp.rim_vertices(ops["pattern"])
    assert not got[rim != 0].any()
    H = solver.operators.heat_system.to_scipy()
    interior = np.flatnonzero(rim == 0)
    expected = np.zeros(n)
    expected[interior] = np.linalg.solve(H[interior][:, interior].toarray(), rhs[interior])
    assert np.allclose(got, expected, rtol=1e-6, atol=1e-12 * expected.max())
    # A closed mesh has no rim: nothing is solved and the solution is left as it was.
    sv, sf = creation.icosphere(2)
    closed = Trimesh(sv, sf.reshape(-1)).heat_solver(None, method="igl")
    keep = DeviceArray.from_host(np.full(sv.shape[0], 7.0))
    assert not closed.diffuse_pinned(DeviceArray.zeros(sv.shape[0], np.float64), keep)
    assert np.all(keep.numpy() == 7.0)
    mesh.dispose()


def test_batched_paths_serve_meshlab_only(gpu) -> None:
    v, f = creation.icosphere(2)
    mesh = Trimesh(v, f.reshape(-1))
    with pytest.raises(NotImplementedError):
        gheat.heat_geodesic_batch(mesh, [[0], [1]], method="igl")
    with pytest.raises(NotImplementedError):
        gheat.BatchPipeline(mesh, 2, method="potpourri3d")
    mesh.dispose()


@pytest.mark.parametrize("name", ["saddle_graded", "degenerate"])
def test_mollified_cotangents_match_the_oracle(gpu, name: str) -> None:
    import ctypes

    from ordito_b200 import _lib

    v, f = meshes.ALL[name]()
    nf = f.shape[0]
    lengths = DeviceArray.empty((nf, 3), np.float32)
    cot = DeviceArray.empty((nf, 3), np.float32)
    delta = ctypes.c_double(0.0)
    mesh = Trimesh(v, f.reshape(-1))
    _lib.call("ob_mollified_cot", mesh.vertices.ptr, mesh.faces.ptr, nf, 1e-5, lengths.ptr, cot.ptr,
              ctypes.byref(delta), None)
    ref_lengths, ref_delta = hp.mollified_lengths(v, f)
    assert np.isclose(delta.value, ref_delta, rtol=1e-6, atol=0.0)
    assert (delta.value > 0.0) == (name == "degenerate")
    ref = hp.cot_from_lengths(ref_lengths)
    assert np.allclose(cot.numpy(), ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())


@pytest.mark.parametrize("method", ["meshlab", "igl"])
@pytest.mark.parametrize("name", ["saddle_graded", "degenerate"])
def test_robust_heat_geodesic_matches_the_oracle(gpu, method: str, name: str) -> None:
    v, f = meshes.ALL[name]()
    src = np.array([5], dtype=np.int32)
    ref = hp.heat_geodesic(v, f, src, method=method, use_robust=True)
    got = gheat.heat_geodesic(v, f.reshape(-1), src, method=method, use_robust=True).numpy()
    assert np.all(np.isfinite(got))
    assert _range_err(got, ref) <= DISTANCE_TOL
