"""The vector heat oracle against the reference's known answers and its invariants (CPU only).

The known answers are the reference's own docstring examples (``tests/golden/known_answers.json``,
each cited); the invariants are those its tests assert (ordito's tests/test_tangent_space.py and
tests/test_heat.py): every ring's angles span the rescaled disk, transport across an edge and back
is the identity, frames are orthonormal and right-handed, transport on a flat patch is constant,
a single source's magnitude is carried everywhere, nothing crosses between components, and the
log map's radius is the geodesic distance.
"""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from oracle import heat_path as hp
from oracle import vector_heat as vh
from ordito_b200 import creation
from tests import meshes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def known() -> dict:
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def grid_state():
    v, f = creation.flat_grid((11, 11), (1.0, 1.0))
    return vh.VectorHeat(v, f)


def test_octahedron_rings(known: dict) -> None:
    item = known["octahedron_one_rings"]
    v, f = creation.octahedron()
    ring, offsets, boundary = vh.vertex_one_rings(f, v.shape[0])
    assert np.diff(offsets).tolist() == item["degrees"]
    assert bool(boundary.any()) == item["boundary"]
    first = ring[offsets[0]:offsets[1]]
    far = f.reshape(-1)[3 * (first // 3) + (first + 1) % 3]
    assert far.tolist() == item["far_ends_of_vertex_0"]


def test_icosphere2_tangent_and_transport_angles(known: dict) -> None:
    item = known["icosphere2_tangent_angles"]
    v, f = creation.icosphere(2)
    rings = vh.vertex_one_rings(f, v.shape[0])
    angles = vh.halfedge_tangent_angles(v, f, rings)
    assert angles.shape == (item["count"],)
    assert int((angles == 0.0).sum()) == item["zeros"] == v.shape[0]
    assert f"{angles.max():.4f}" == item["max"]
    twins = vh.halfedge_twins(f)
    rho = vh.halfedge_transport_angles(twins, angles)
    trip = known["icosphere2_transport_round_trip"]
    assert np.allclose(np.cos(rho[twins] + rho), trip["round_trip_cos"], atol=trip["atol"])


def test_grid_transport_and_log_map(known: dict, grid_state) -> None:
    item = known["grid_transport"]
    transported, resolved = vh.transport_tangent_vectors(grid_state, np.array([item["source"]]),
                                                         np.array([item["vector"]]))
    bx, by, _ = grid_state.frames
    world = vh.tangent_to_world(transported, bx, by)
    assert bool(resolved.all()) == item["resolved_all"]
    a, b = item["same_world_direction"]
    assert np.allclose(world[a], world[b], atol=item["atol"])
    lm = known["grid_log_map"]
    for method in ("heat_geodesic", "potpourri3d"):
        x, y = vh.log_map(grid_state, lm["source"], method)[lm["vertex"]]
        w = x * bx[lm["source"]] + y * by[lm["source"]]
        assert np.round(w[:2].astype(np.float64), 2).tolist() == lm[method]


@pytest.mark.parametrize("name", ["sphere_irregular", "torus_irregular", "grid", "saddle_graded"])
def test_tangent_angles_span_the_rescaled_disk(name: str) -> None:
    v, f = meshes.ALL[name]()
    ring, offsets, boundary = rings = vh.vertex_one_rings(f, v.shape[0])
    angles = vh.halfedge_tangent_angles(v, f, rings)
    corners = vh.corner_angles(v, f).reshape(-1)
    for vertex in range(v.shape[0]):
        r = ring[offsets[vertex]:offsets[vertex + 1]]
        if r.size == 0:
            continue
        start = 0 if boundary[vertex] else int(np.argmax(r))
        r = np.roll(r, -start)
        turn = np.pi if boundary[vertex] else 2 * np.pi
        scale = turn / corners[r].sum()
        assert angles[r[0]] == 0.0
        assert np.allclose(angles[r], scale * np.concatenate([[0.0], np.cumsum(corners[r])[:-1]]), atol=1e-9)
        assert np.isclose(angles[r[-1]] + scale * corners[r[-1]], turn, atol=1e-9)


@pytest.mark.parametrize("name", ["sphere_irregular", "torus_irregular", "saddle_graded"])
def test_frames_and_transport_invariants(name: str) -> None:
    v, f = meshes.ALL[name]()
    rings = vh.vertex_one_rings(f, v.shape[0])
    bx, by, normal = vh.vertex_tangent_frames(v, f, rings)
    assert np.allclose(np.linalg.norm(bx, axis=1), 1.0, atol=1e-5)
    assert np.allclose((bx * normal).sum(axis=1), 0.0, atol=1e-5)
    assert np.allclose((np.cross(bx, by) * normal).sum(axis=1), 1.0, atol=1e-5)
    twins = vh.halfedge_twins(f)
    rho = vh.halfedge_transport_angles(twins, vh.halfedge_tangent_angles(v, f, rings))
    interior = np.flatnonzero(twins >= 0)
    assert np.allclose(np.angle(np.exp(1j * (rho[interior] + rho[twins[interior]]))), 0.0, atol=1e-9)
    assert np.all(np.abs(rho) <= np.pi + 1e-12)


def test_vector_system_is_symmetric_positive_definite() -> None:
    v, f = meshes.ALL["sphere_irregular"]()
    state = vh.VectorHeat(v, f)
    a = state.system
    assert abs(a - a.T).max() <= 1e-12 * abs(a).max()
    # A constant world direction on a flat patch is in the connection Laplacian's kernel, so
    # (M + t L) x = M x on every row whose vertex and neighbours are interior (a rim vertex's fan is
    # rescaled to half a turn, which bends the transport there).
    vg, fg = creation.flat_grid((7, 7), (1.0, 1.0))
    flat = vh.VectorHeat(vg, fg)
    bx, by, _ = flat.frames
    world = np.array([0.6, 0.8, 0.0])
    x = np.stack((bx @ world, by @ world), axis=1).reshape(-1)
    mass = np.repeat(flat.ops["mass"], 2)
    rim = flat.rings[2]
    adjacency = hp.csr_matrix(flat.ops["pattern"], np.ones(flat.ops["H"].size))
    inner = np.flatnonzero(~rim & (adjacency @ rim.astype(float) == 0))
    rows = np.stack((2 * inner, 2 * inner + 1), axis=1).reshape(-1)
    assert inner.size > 0
    assert np.allclose((flat.system @ x)[rows], (mass * x)[rows], atol=1e-6 * np.abs(mass * x).max())


def test_flat_patch_transport_is_constant() -> None:
    v, f = creation.flat_grid((9, 9), (1.0, 1.0), center=False)
    state = vh.VectorHeat(v, f)
    transported, _ = vh.transport_tangent_vectors(state, np.array([40]), np.array([[1.0, 0.0]]))
    bx, by, _ = state.frames
    world = vh.tangent_to_world(transported, bx, by)
    unit = world / np.linalg.norm(world, axis=1, keepdims=True)
    interior = ~state.rings[2]
    assert np.allclose(unit[interior] @ unit[interior][0], 1.0, atol=1e-4)
    assert np.allclose(np.linalg.norm(world, axis=1), 1.0, atol=1e-4)


def test_transport_magnitude_and_components() -> None:
    v, f = meshes.ALL["sphere_irregular"]()
    state = vh.VectorHeat(v, f)
    transported, resolved = vh.transport_tangent_vectors(state, np.array([0]), np.array([[0.0, 2.5]]))
    assert np.allclose(np.linalg.norm(transported, axis=1), 2.5, atol=1e-4)
    assert resolved.all()
    # Two disjoint copies: nothing reaches the second.
    v2 = np.concatenate((v, v + np.float32(3.0)))
    f2 = np.concatenate((f, f + v.shape[0]))
    both = vh.VectorHeat(v2, f2)
    transported, resolved = vh.transport_tangent_vectors(both, np.array([0]), np.array([[1.0, 0.0]]))
    n = v.shape[0]
    assert np.allclose(np.linalg.norm(transported[:n], axis=1), 1.0, atol=1e-4)
    assert np.all(transported[n:] == 0.0)
    assert resolved[:n].all() and not resolved[n:].any()


def test_log_map_radius_is_the_geodesic_distance() -> None:
    v, f = meshes.ALL["sphere_irregular"]()
    state = vh.VectorHeat(v, f)
    lm = vh.log_map(state, 0)
    distance = hp.heat_geodesic(v, f, np.array([0]), state.t, method="potpourri3d")
    assert np.allclose(np.linalg.norm(lm, axis=1), distance, rtol=1e-4, atol=1e-4)
    assert np.allclose(lm[0], 0.0, atol=1e-6)


def test_halfedge_tables_reject_what_the_reference_rejects() -> None:
    # Three faces on one edge.
    with pytest.raises(ValueError, match="three or more"):
        vh.halfedge_twins(np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4]]))
    # Two faces wound against each other.
    with pytest.raises(ValueError, match="same way"):
        vh.halfedge_twins(np.array([[0, 1, 2], [0, 1, 3]]))
    # Two fans meeting at vertex 0 only.
    with pytest.raises(ValueError, match="pinched"):
        vh.vertex_one_rings(np.array([[0, 1, 2], [0, 3, 4]]), 5)
