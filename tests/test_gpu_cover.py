"""The intrinsic tufted cover on the CUDA path against the oracle (GPU).

``heat_geodesic(method="potpourri3d", use_robust=True)`` (ordito/heat.py:5084, :3749,
kernels/heat.py:710-1204): the cover's faces, twins and flipped lengths bit for bit (every float64
step of both rounds once, in the same order; the meshes here need no mollification, which alone
adds a sum whose order differs), the half-cotangents, area sums and divergence bit for bit, the
operators within 1e-12 (the time step's mean edge is a sum in a different order), and the distance
within 1e-5 of the oracle's range.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import heat_path as hp
from oracle import tufted_cover as tc
from ordito_b200 import cover as gcover
from ordito_b200 import creation
from ordito_b200 import heat as gheat
from ordito_b200.device import DeviceArray
from ordito_b200.mesh import Trimesh
from tests import meshes

pytestmark = pytest.mark.gpu

DISTANCE_TOL = 1e-5  # max |d - d_oracle| / range of d_oracle
VALUE_RTOL = 1e-12   # operator values against the oracle's (relative to the largest)


def _mesh(name: str) -> tuple[np.ndarray, np.ndarray]:
    if name == "jittered_torus":
        v, f = creation.jittered_torus(48, 24, 1.0, 0.3, 0.6, seed=3)
        return v, np.asarray(f).reshape(-1, 3)
    if name == "book":
        # An edge of three faces and a pair wound the same way, beside ordinary faces.
        v = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, -1, 0], [0.5, 0, 1], [1.5, 0.8, 0.1]],
                     dtype=np.float32)
        f = np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4], [1, 5, 2]], dtype=np.int32)
        return v, f
    v, f = getattr(meshes, name)()
    return v, np.asarray(f).reshape(-1, 3)


NAMES = ["saddle_graded", "sphere_irregular", "torus_irregular", "jittered_torus", "book"]


@pytest.mark.parametrize("name", NAMES)
def test_cover_matches_the_oracle_flip_for_flip(gpu, name: str) -> None:
    v, f = _mesh(name)
    # These meshes need no mollification (every triangle inequality holds by more than the
    # margin), so the lengths are the positions' own on both sides.
    _, raw, _ = tc.tufted_cover(v, f, tc.halfedge_mates(f))
    total, count, worst = tc.length_sums(raw[: f.shape[0]])
    assert worst + tc.TOLERANCE_MOLLIFY * total / count < 0.0
    mesh = Trimesh(v, f.reshape(-1))
    cover, area_sums, _ = gcover.build_cover(mesh)
    ref_cover, ref_lengths, ref_twin, ref_rounds = tc.intrinsic_delaunay(v, f)
    assert cover.rounds == ref_rounds
    assert np.array_equal(cover.faces.numpy(), ref_cover)
    assert np.array_equal(cover.twin.numpy(), ref_twin)
    assert np.array_equal(cover.lengths.numpy().reshape(-1), ref_lengths.reshape(-1))
    ref_cot, ref_sums = tc.cover_face_terms(ref_cover, ref_lengths, v.shape[0])
    assert np.array_equal(cover.cot.numpy(), ref_cot)
    assert np.array_equal(area_sums.numpy(), ref_sums)
    mesh.dispose()


@pytest.mark.parametrize("name", ["saddle_graded", "torus_irregular"])
def test_cover_operators_and_divergence_match_the_oracle(gpu, name: str) -> None:
    v, f = _mesh(name)
    n = v.shape[0]
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver(None, use_robust=True, method="potpourri3d")
    ops = solver.operators
    ref = tc.cover_operators(v, f, solver._vertex_time()[0])
    for got, key in ((ops.laplacian, "L"), (ops.heat_system, "H"), (ops.poisson_system, "P")):
        A = got.to_scipy().toarray()
        B = hp.csr_matrix(ref["pattern"], ref[key]).toarray()
        assert np.abs(A - B).max() <= VALUE_RTOL * np.abs(B).max()
    # The divergence of one field, bit for bit against the oracle's.
    u = np.random.default_rng(7).random(n)
    cover = solver.cover
    out = DeviceArray.empty(n, np.float64)
    gcover.cover_divergence(cover, DeviceArray.from_host(u), out)
    expected = tc.cover_divergence(ref["cover_faces"], ref["lengths"], ref["cot"], u, n)
    assert np.array_equal(out.numpy(), expected)
    mesh.dispose()


@pytest.mark.parametrize("name,source", [("saddle_graded", 0), ("sphere_irregular", 0),
                                         ("torus_irregular", 11), ("jittered_torus", 5)])
def test_robust_heat_geodesic_matches_the_oracle(gpu, name: str, source: int) -> None:
    v, f = _mesh(name)
    src = np.array([source], dtype=np.int32)
    ref = tc.heat_geodesic_robust(v, f, src)
    assert np.ptp(ref) > 0.5
    got = gheat.heat_geodesic(v, f.reshape(-1), src, method="potpourri3d", use_robust=True).numpy()
    assert float(np.max(np.abs(got - ref)) / np.ptp(ref)) <= DISTANCE_TOL
    # The Trimesh form keeps the cover and answers the same again (through the factors the
    # second solve earns).
    mesh = Trimesh(v, f.reshape(-1))
    for _ in range(2):
        again = gheat.heat_geodesic(mesh, src, method="potpourri3d", use_robust=True).numpy()
        assert float(np.max(np.abs(again - ref)) / np.ptp(ref)) <= DISTANCE_TOL
    mesh.dispose()


def test_mollified_cover_matches_the_oracle(gpu) -> None:
    # A collinear triangle: every length grows by the worst violation plus the margin (the mean
    # front length's sum runs in another order here and in the oracle, so the lengths agree to
    # rounding rather than bit for bit), then the flips and the distance as on any mesh.
    v, f = meshes.ALL["degenerate"]()
    f = np.asarray(f).reshape(-1, 3)
    mesh = Trimesh(v, f.reshape(-1))
    cover, _, _ = gcover.build_cover(mesh)
    ref_cover, ref_lengths, ref_twin, _ = tc.intrinsic_delaunay(v, f)
    _, raw, _ = tc.tufted_cover(v, f, tc.halfedge_mates(f))
    assert np.all(ref_lengths.reshape(-1) > raw.reshape(-1).min())  # the shift was applied
    assert np.array_equal(cover.faces.numpy(), ref_cover)
    assert np.array_equal(cover.twin.numpy(), ref_twin)
    assert np.allclose(cover.lengths.numpy(), ref_lengths, rtol=1e-14, atol=0.0)
    src = np.array([5], dtype=np.int32)
    ref = tc.heat_geodesic_robust(v, f, src)
    got = gheat.heat_geodesic(mesh, src, method="potpourri3d", use_robust=True).numpy()
    assert np.all(np.isfinite(got))
    assert float(np.max(np.abs(got - ref)) / np.ptp(ref)) <= DISTANCE_TOL
    mesh.dispose()


def test_robust_solver_has_no_pinned_diffusion(gpu) -> None:
    v, f = creation.icosphere(1)
    mesh = Trimesh(v, f.reshape(-1))
    field = DeviceArray.zeros(v.shape[0], np.float64)
    with pytest.raises(ValueError, match="no use_robust variant at method='potpourri3d'"):
        mesh.heat_solver(use_robust=True).diffuse_pinned(field, DeviceArray.zeros(v.shape[0], np.float64))
    mesh.dispose()
