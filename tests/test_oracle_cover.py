"""The tufted-cover oracle against the properties the reference states for it (CPU only).

ordito/kernels/heat.py:710-735 and :749-1130 describe the cover: each face doubled into a front
and a reversed back copy; two faces winding an edge opposite ways glued front to front, the same
way front to back, a rim edge to its own face's back copy, an edge of three or more faces along a
chain; lengths mollified; flipped until every edge passes the Euclidean Delaunay test; and on a
closed orientable mesh, whose cover is two copies of it, every operator entry is twice the
copy's (ordito/heat.py:3756-3760).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import heat_path as hp
from oracle import tufted_cover as tc
from ordito_b200 import creation
from tests import meshes


def _slots_ok(cover: np.ndarray, lengths: np.ndarray, twin: np.ndarray) -> None:
    h = np.arange(twin.size)
    assert np.all(twin >= 0) and np.all(twin[twin] == h), "twin is an involution over every slot"
    nxt = h - h % 3 + (h + 1) % 3
    prv = h - h % 3 + (h + 2) % 3
    ends = np.sort(np.stack([cover[nxt], cover[prv]], 1), 1)
    assert np.array_equal(ends, ends[twin]), "twins span the same vertex pair"
    flat = lengths.reshape(-1)
    assert np.array_equal(flat, flat[twin]), "twins carry one length"


def _delaunay_weights(lengths: np.ndarray, twin: np.ndarray) -> np.ndarray:
    h = np.arange(twin.size)
    live = (twin > h) & (h // 3 != twin // 3)
    return tc.slot_half_cotangent(lengths, h[live]) + tc.slot_half_cotangent(lengths, twin[live])


@pytest.mark.parametrize("name", ["saddle_graded", "sphere_irregular", "torus_irregular", "jittered"])
def test_cover_is_closed_and_flipped_to_delaunay(name: str) -> None:
    if name == "jittered":
        v, f = creation.jittered_torus(40, 20, 1.0, 0.3, 0.6, seed=3)
    else:
        v, f = getattr(meshes, name)()
    cover, lengths, twin, rounds = tc.intrinsic_delaunay(v, f)
    assert cover.size == 6 * (f.size // 3 if f.ndim == 1 else f.shape[0])
    _slots_ok(cover, lengths, twin)
    assert _delaunay_weights(lengths, twin).min() >= -tc.DELAUNAY_EPSILON
    assert 1 <= rounds < tc.FLIP_ROUNDS
    # Every cover face is a valid triangle of positive area after the flips.
    assert np.all(tc.heron(lengths[:, 0], lengths[:, 1], lengths[:, 2]) > 0)


def test_graded_saddle_needs_flips() -> None:
    v, f = meshes.saddle_graded()
    cover, lengths, twin, rounds = tc.intrinsic_delaunay(v, f)
    before = tc.tufted_cover(v, f, tc.halfedge_mates(f))
    assert rounds > 1 and not np.array_equal(cover, before[0])
    assert _delaunay_weights(before[1], before[2]).min() < -tc.DELAUNAY_EPSILON


def test_rim_edge_glues_to_its_own_back_copy() -> None:
    v, f = creation.flat_grid((3, 3))
    f = np.asarray(f).reshape(-1)
    mates = tc.halfedge_mates(f)
    cover, lengths, twin = tc.tufted_cover(v, f, mates)
    n_faces = f.size // 3
    rim = np.flatnonzero(mates == -1)
    assert rim.size > 0
    for h in rim:
        slot = h - h % 3 + (h + 2) % 3  # the front slot of halfedge h: opposite corner k + 2
        face, e = slot // 3, slot % 3
        assert twin[slot] == 3 * (n_faces + face) + (0 if e == 0 else 3 - e)
    _slots_ok(cover, lengths, twin)


def test_edge_of_three_faces_is_chained() -> None:
    # Three triangles on the edge (0, 1): a book of three pages, two wound one way, one the other.
    v = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, -1, 0], [0.5, 0, 1]], dtype=np.float32)
    f = np.array([0, 1, 2, 1, 0, 3, 0, 1, 4], dtype=np.int32)
    mates = tc.halfedge_mates(f)
    assert np.all(mates[[0, 3, 6]] == -2)  # halfedge 0 is the edge's lowest
    cover, lengths, twin = tc.tufted_cover(v, f, mates)
    _slots_ok(cover, lengths, twin)


def test_same_way_pair_glues_front_to_back() -> None:
    v = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, -1, 0]], dtype=np.float32)
    f = np.array([0, 1, 2, 0, 1, 3], dtype=np.int32)  # both run 0 -> 1
    mates = tc.halfedge_mates(f)
    assert mates[0] == 3 and mates[3] == 0
    cover, lengths, twin = tc.tufted_cover(v, f, mates)
    _slots_ok(cover, lengths, twin)
    front0 = 2  # halfedge 0's front slot (opposite corner 2 of face 0)
    assert twin[front0] // 3 == 2 + 1  # the other face's back copy (cover face F + 1)


def test_closed_orientable_cover_entries_are_twice_the_copys() -> None:
    # The icosphere is Delaunay already: no flips, and the cover is two copies of the mesh with
    # its float64 intrinsic geometry.
    v, f = creation.icosphere(2)
    ops = tc.cover_operators(v, f, t=0.01)
    assert ops["rounds"] == 1
    f64 = np.asarray(f, dtype=np.int64).reshape(-1, 3)
    lengths = ops["lengths"][: f64.shape[0]]
    cot, sums = tc.cover_face_terms(f64.reshape(-1), lengths, v.shape[0])
    single = hp.heat_operators(v, f64, 0.01, method="potpourri3d", cot=cot, area_sums=sums)
    pattern = ops["pattern"]
    L_cover = hp.csr_matrix(pattern, ops["L"]).toarray()
    L_single = hp.csr_matrix(single["pattern"], single["L"]).toarray()
    np.testing.assert_allclose(L_cover, 2.0 * L_single, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(ops["mass"], 2.0 * single["mass"], rtol=1e-13)


def test_robust_distance_on_a_delaunay_mesh_matches_the_plain_method(monkeypatch) -> None:
    # With nothing to flip or mollify the cover changes the discretisation by its float64
    # geometry and by its doubled operators, against which the fixed 1e-6 Poisson shift weighs
    # half: the plain method with the shift halved is the same system up to the geometry's
    # float32 rounding (measured 4e-9; 1.0e-5 against the unhalved shift).
    v, f = creation.icosphere(3)
    robust = tc.heat_geodesic_robust(v, f, np.array([0]))
    monkeypatch.setattr(hp, "GEOMETRY_CENTRAL_POISSON_SHIFT", 0.5 * hp.GEOMETRY_CENTRAL_POISSON_SHIFT)
    plain = hp.heat_geodesic(v, f, np.array([0]), method="potpourri3d")
    assert hp.relative_linf(robust, plain) < 1e-7


def test_mollification_shifts_every_length() -> None:
    # A collinear triangle violates the strict triangle inequality: every length grows by the
    # worst violation plus the margin.
    v = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [1, 1, 0]], dtype=np.float32)
    f = np.array([0, 1, 3, 1, 2, 3, 0, 2, 1], dtype=np.int32)
    cover, lengths, twin = tc.tufted_cover(v, f, tc.halfedge_mates(f))
    total, count, worst = tc.length_sums(lengths[:3])
    shifted = tc.mollify(lengths, 3)
    delta = worst + tc.TOLERANCE_MOLLIFY * total / count
    assert worst == 0.0 and delta > 0.0
    np.testing.assert_array_equal(shifted, lengths + delta)
