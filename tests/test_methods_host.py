"""The oracle's ``method="igl"`` and ``method="potpourri3d"`` pieces on the host: the Voronoi lumped
mass against hand-computed shares, the rim, the rim-pinned heat rows, and the time steps each
method names (ordito/heat.py:2002-2012, kernels/triangles.py:276, kernels/heat.py:469-518)."""

from __future__ import annotations

import numpy as np

from oracle import heat_path as hp
from ordito_b200 import creation
from tests import meshes


def test_voronoi_shares_of_an_obtuse_and_an_equilateral_face() -> None:
    # Obtuse at corner 2 (vectors to the others dot to -2.75), area 1: half to the obtuse
    # corner, a quarter to each other.
    v = np.array([[0, 0, 0], [4, 0, 0], [1, 0.5, 0]], dtype=np.float32)
    f = np.array([[0, 1, 2]], dtype=np.int64)
    assert np.array_equal(hp.voronoi_area_sums(v, f, 3), [0.25, 0.25, 0.5])
    # Equilateral: the circumcentric split gives every corner a third.
    s = np.sqrt(3.0) / 2.0
    v = np.array([[0, 0, 0], [1, 0, 0], [0.5, s, 0]], dtype=np.float32)
    sums = hp.voronoi_area_sums(v, f, 3)
    area = float(hp.face_normals_and_areas(v, f)[1][0])
    assert np.allclose(sums, area / 3.0, rtol=1e-6)


def test_voronoi_mass_sums_to_the_area_and_differs_from_barycentric() -> None:
    v, f = meshes.bumpy_sphere()
    n = v.shape[0]
    voronoi = hp.voronoi_area_sums(v, f, n)
    _, areas = hp.face_normals_and_areas(v, f)
    assert np.isclose(voronoi.sum(), areas.astype(np.float64).sum(), rtol=1e-6)
    barycentric = hp.area_sums(f, areas, n) / 3.0
    assert np.abs(voronoi - barycentric).max() > 1e-3 * barycentric.max()
    ops = hp.heat_operators(v, f, 0.0, method="igl")
    assert np.allclose(ops["mass"], voronoi)


def test_rim_of_a_grid_and_of_a_closed_mesh() -> None:
    v, f = creation.grid((6, 5))
    n = v.shape[0]
    rim = hp.rim_vertices(hp.mesh_operator_pattern(f.reshape(-1, 3), n))
    # The boundary of a 6 x 5 vertex grid.
    assert int(rim.sum()) == 2 * (6 + 5) - 4
    sv, sf = creation.icosphere(2)
    assert not hp.rim_vertices(hp.mesh_operator_pattern(sf.reshape(-1, 3), sv.shape[0])).any()


def test_pinned_rows_are_identity_on_the_rim() -> None:
    v, f = meshes.saddle_graded()
    ops = hp.heat_operators(v, f, None, method="igl")
    pattern = ops["pattern"]
    rim = hp.rim_vertices(pattern)
    pinned = hp.csr_matrix(pattern, hp.pinned_heat_values(pattern, ops["H"], rim)).toarray()
    on = np.flatnonzero(rim)
    off = np.flatnonzero(rim == 0)
    assert np.array_equal(pinned[on][:, on], np.eye(on.size))
    assert not pinned[off][:, on].any() and not pinned[on][:, off].any()
    H = hp.csr_matrix(pattern, ops["H"]).toarray()
    assert np.array_equal(pinned[off][:, off], H[off][:, off])


def test_methods_take_their_own_time_step() -> None:
    # An open mesh: its rim edges lie on one face, so the face-edge and unique-edge means differ.
    v, f = meshes.saddle_graded()
    t_meshlab = hp.heat_operators(v, f, None)["t"]
    t_igl = hp.heat_operators(v, f, None, method="igl")["t"]
    t_gc = hp.heat_operators(v, f, None, method="potpourri3d")["t"]
    pattern = hp.mesh_operator_pattern(f, v.shape[0])
    total, count = hp.edge_length_sums(v, pattern, face_edges=False)
    assert np.isclose(t_igl, (total / count) ** 2) and t_igl == t_gc
    assert t_meshlab != t_igl


def test_igl_averages_only_where_there_is_a_rim() -> None:
    # A closed mesh has no rim: igl is meshlab's path on the Voronoi mass and unique-edge step.
    v, f = creation.icosphere(2)
    src = np.array([3])
    t, _ = hp.vertex_time(v, f, None, "igl")
    ops = hp.heat_operators(v, f, t, method="igl")
    H = hp.csr_matrix(ops["pattern"], ops["H"])
    P = hp.csr_matrix(ops["pattern"], ops["P"])
    plain = hp.heat_geodesic(v, f, src, operators=ops, factors=(hp.HeatFactor(H), hp.PoissonFactor(P)))
    assert np.allclose(hp.heat_geodesic(v, f, src, method="igl"), plain, rtol=0, atol=1e-12)


def test_intrinsic_cotangents_and_mollification_known_answers() -> None:
    # The reference's docstring examples (ordito/laplacian.py:318-324, 822-838): an equilateral
    # triangle weighs every edge cot(60)/2, the 3-4-5 triangle gives its hypotenuse nothing; a
    # box needs no repair, a collinear triangle gets every length lengthened by 1e-5 x 4/3.
    cot = hp.cot_from_lengths(np.array([[1.0, 1.0, 1.0], [5.0, 4.0, 3.0]], dtype=np.float32))
    assert np.allclose(cot[0], 1.0 / (2.0 * np.sqrt(3.0)), rtol=1e-6)
    assert np.allclose(cot[1], [0.0, 0.375, 2.0 / 3.0], rtol=1e-6, atol=1e-7)
    bv, bf = creation.box()
    assert hp.mollified_lengths(bv, bf)[1] == 0.0
    line = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0]], dtype=np.float32)
    lengths, delta = hp.mollified_lengths(line, np.array([[0, 1, 2]]))
    assert f"{delta:.2e}" == "1.33e-05"
    assert np.allclose(lengths, np.array([[1.0, 2.0, 1.0]]) + delta, rtol=0, atol=1e-7)
    # A repeated-vertex face has a zero margin, so every face of its mesh is lengthened; a clean
    # mesh's intrinsic weights are its positional ones to float32 rounding.
    dv, df = meshes.with_degenerate_face()
    assert hp.mollified_lengths(dv, df)[1] > 0.0
    sv, sf = meshes.saddle_graded()
    lengths, delta = hp.mollified_lengths(sv, sf)
    assert delta == 0.0
    positional = hp.cotmatrix_entries(sv, sf)
    intrinsic = hp.cot_from_lengths(lengths)
    assert np.allclose(intrinsic, positional, rtol=1e-3, atol=1e-4 * np.abs(positional).max())
