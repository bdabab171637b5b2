"""The oracle against the reference's known answers and the path's invariants (CPU only)."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import heat_path as hp
from ordito_b200 import creation
from tests import meshes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def known() -> dict:
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


def test_cot_entries_of_the_unit_square(known: dict) -> None:
    v, f = creation.grid((2, 2))
    item = known["cot_grid_2x2"]
    assert hp.cotmatrix_entries(v, f).round(item["round"]).tolist() == item["value"]


def test_lumped_mass_sums(known: dict) -> None:
    v, f = creation.box()
    assert hp.heat_operators(v, f)["mass"].sum() == pytest.approx(known["mass_sum_unit_box"]["value"], abs=1e-6)
    v, f = creation.icosphere(3)
    total = hp.heat_operators(v, f)["mass"].sum()
    assert round(total, 4) == known["mass_sum_icosphere3"]["value"]


def test_icosphere2_area(known: dict) -> None:
    v, f = creation.icosphere(2)
    _, areas = hp.face_normals_and_areas(v, f)
    assert round(float(areas.astype(np.float64).sum()), 3) == known["area_sum_icosphere2"]["value"]


def test_pole_to_pole_on_icosphere3(known: dict) -> None:
    item = known["pole_to_pole_icosphere3"]
    v, f = creation.icosphere(3)
    north, south = int(np.argmax(v[:, 2])), int(np.argmin(v[:, 2]))
    d = hp.heat_geodesic(v, f, np.array([north]))
    assert d[north] == item["source"]
    assert round(float(d[south]), item["digits"]) == item["antipode"]


def test_heat_solve_of_the_mass_is_one(known: dict) -> None:
    v, f = creation.icosphere(2)
    ops = hp.heat_operators(v, f)
    H = hp.csr_matrix(ops["pattern"], ops["H"])
    x = hp.solve_heat(H, ops["mass"])
    assert np.allclose(x, known["heat_solve_of_mass_is_one"]["value"], atol=1e-10)


def test_csr_from_keys_toy(known: dict) -> None:
    item = known["csr_from_keys_toy"]
    out = hp.csr_from_keys(
        np.array(item["keys"], dtype=np.uint64), np.array(item["order"], dtype=np.int32),
        item["n_rows"], item["n_cols"],
    )
    assert out["offsets"].tolist() == item["offsets"]
    assert out["columns"].tolist() == item["columns"]
    starts = np.append(out["run_start"], hp.run_ends(out["keys"], out["run_start"][-1:]))
    assert starts.tolist() == item["starts"]
    assert out["order"][:3].tolist() == item["sorted_order"]


def test_golden_fixture_is_current() -> None:
    g = np.load(os.path.join(GOLDEN, "oracle_ico3.npz"))
    v, f = creation.icosphere(3)
    assert np.array_equal(g["vertices"], v) and np.array_equal(g["faces"], f)
    ops = hp.heat_operators(v, f)
    assert np.array_equal(g["offsets"], ops["pattern"]["offsets"])
    assert np.array_equal(g["L"], ops["L"])
    d = hp.heat_geodesic(v, f, np.array([0]))
    assert np.allclose(g["distance"], d, rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", sorted(meshes.ALL))
def test_operator_invariants(name: str) -> None:
    v, f = meshes.ALL[name]()
    ops = hp.heat_operators(v, f)
    pattern = ops["pattern"]
    L = hp.csr_matrix(pattern, ops["L"])
    H = hp.csr_matrix(pattern, ops["H"])
    ones = np.ones(L.shape[0])
    # Rows of L sum to zero; (M - tL) 1 = M 1; L is symmetric.
    assert np.max(np.abs(L @ ones)) <= 1e-12 * max(1.0, np.abs(ops["L"]).max())
    assert np.allclose(H @ ones, ops["mass"] * (np.diff(pattern["offsets"]) > 0), atol=1e-12)
    assert abs(L - L.T).max() <= 1e-15 * np.abs(ops["L"]).max()


@pytest.mark.parametrize("name", sorted(meshes.ALL))
def test_pattern_matches_a_brute_force_build(name: str) -> None:
    v, f = meshes.ALL[name]()
    n = v.shape[0]
    pattern = hp.mesh_operator_pattern(f, n)
    rows, cols = [], []
    for tri in f:
        for e in range(3):
            i, j = int(tri[(e + 1) % 3]), int(tri[(e + 2) % 3])
            rows += [i, j]
            cols += [j, i]
        rows += list(map(int, tri))
        cols += list(map(int, tri))
    m = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    m.sum_duplicates()
    m.sort_indices()
    assert np.array_equal(pattern["offsets"], m.indptr)
    assert np.array_equal(pattern["columns"], m.indices)


def test_source_is_zero_and_nonnegative() -> None:
    v, f = meshes.bumpy_sphere()
    d = hp.heat_geodesic(v, f, np.array([3]))
    assert d[3] == 0.0
    assert d.min() >= -1e-6


def test_out_of_range_sources_raise() -> None:
    v, f = creation.icosphere(1)
    with pytest.raises(ValueError):
        hp.heat_geodesic(v, f, np.array([0, v.shape[0]]))


def test_empty_inputs_return_zero_fields() -> None:
    v, f = creation.icosphere(1)
    assert not hp.heat_geodesic(v, f, np.array([], dtype=np.int64)).any()


# ---- known answers of the reference's docstrings, and the invariants its own tests assert ----


def test_intrinsic_cotangents_of_two_triangles(known: dict) -> None:
    item = known["cot_intrinsic_equilateral_and_345"]
    cot = hp.cot_from_lengths(np.array(item["lengths"], dtype=np.float32)).astype(np.float64)
    assert cot.round(item["round"]).tolist() == item["value"]


def test_mollify_delta_on_the_box_and_a_collinear_triangle(known: dict) -> None:
    item = known["mollify_delta"]
    v, f = creation.box()
    lengths, delta = hp.mollified_lengths(v, f)
    assert lengths.shape == (12, 3) and delta == item["box"]
    v = np.array(item["collinear_vertices"], dtype=np.float32)
    _, delta = hp.mollified_lengths(v, np.array([[0, 1, 2]]))
    assert f"{delta:.2e}" == item["collinear"]


def test_box_pattern_entries(known: dict) -> None:
    item = known["box_pattern_entries"]
    v, f = creation.box()
    pattern = hp.mesh_operator_pattern(f, v.shape[0])
    assert [pattern["offsets"].size - 1] * 2 == item["shape"]
    assert int(pattern["offsets"][-1]) == item["nnz"]


def test_cotmatrix_row_sums_and_linear_precision(known: dict) -> None:
    item = known["cotmatrix_row_sums_and_linear_precision"]
    v, f = creation.icosphere(2)
    ops = hp.heat_operators(v, f)
    L = hp.csr_matrix(ops["pattern"], ops["L"])
    assert L.shape == (item["icosphere2_rows"],) * 2
    assert np.abs(L @ np.ones(L.shape[0])).max() < item["row_sum_bound"]
    v, f = creation.grid(tuple(item["grid"]))
    ops = hp.heat_operators(v, f)
    L = hp.csr_matrix(ops["pattern"], ops["L"])
    interior = (L @ v[:, 0].astype(np.float64)).reshape(item["grid"])[1:-1, 1:-1]
    assert np.abs(interior).max() < item["interior_bound"]


@pytest.mark.parametrize(("name", "t"), [("sphere_irregular", None), ("saddle_graded", None),
                                         ("sphere_irregular", 0.05), ("torus_irregular", None)])
def test_heat_operators_are_the_matrices_they_name(name: str, t: float | None) -> None:
    """ordito tests/test_heat.py:126-188 on the oracle: P is -L exactly, H is M - t L for one t
    (read off an off-diagonal entry) to 1e-12, that t is the squared mean unique edge length (the
    potpourri3d default) to 1e-6 or the explicit t as given, and the face normals and areas match a
    float64 computation from the same float32 positions to 1e-5."""
    v, f = meshes.ALL[name]()
    t_eff, _ = hp.vertex_time(v, f, t, "potpourri3d")
    ops = hp.heat_operators(v, f, t_eff, method="potpourri3d")
    pattern = ops["pattern"]
    L = hp.csr_matrix(pattern, ops["L"]).toarray()
    H = hp.csr_matrix(pattern, ops["H"]).toarray()
    P = hp.csr_matrix(pattern, ops["P"]).toarray()
    assert np.array_equal(P, -L)
    row, col = np.argwhere(np.triu(L, k=1) != 0.0)[0]
    diffusion_time = float(-H[row, col] / L[row, col])
    v64 = v.astype(np.float64)
    f64 = f.astype(np.int64)
    edges = np.unique(np.sort(np.concatenate([f64[:, [0, 1]], f64[:, [1, 2]], f64[:, [2, 0]]]), axis=1), axis=0)
    unique_mean = float(np.linalg.norm(v64[edges[:, 0]] - v64[edges[:, 1]], axis=1).mean())
    expected_t = unique_mean**2 if t is None else t
    assert np.isclose(diffusion_time, expected_t, rtol=1e-6, atol=0.0)
    if t is not None:
        diffusion_time = t
    assert np.allclose(H, np.diag(ops["mass"]) - diffusion_time * L, rtol=1e-12, atol=1e-15)
    corners = v64[f64]
    cross = np.cross(corners[:, 1] - corners[:, 0], corners[:, 2] - corners[:, 0])
    norm = np.linalg.norm(cross, axis=1)
    assert np.allclose(ops["normals"], cross / norm[:, None], rtol=1e-5, atol=1e-5)
    assert np.allclose(ops["areas"], 0.5 * norm, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("name", ["saddle_graded", "sphere_irregular", "torus_irregular"])
def test_source_is_zero_and_distance_nonnegative_on_the_reference_fixtures(name: str) -> None:
    """ordito tests/test_heat.py:653-663 (saddle_graded, source 0), also on the irregular closed
    fixtures: the distance is >= -1e-6 and 0 at the source to 1e-4."""
    v, f = meshes.ALL[name]()
    d = hp.heat_geodesic(v, f, np.array([0]))
    assert np.all(d >= -1e-6)
    assert abs(d[0]) <= 1e-4
    assert d.max() > 0.5  # the distance propagated


def test_dissection_ordering_solves_as_the_default_ordering() -> None:
    """The oracle's ordering for meshes too large for SuperLU's own: a permutation, and the same
    exact solves (every heat entry to its own size) as the default column ordering."""
    v, f = creation.jittered_torus(64, 32, seed=2)
    t_eff, _ = hp.vertex_time(v, f, None)
    ops = hp.heat_operators(v, f, t_eff)
    H = hp.csr_matrix(ops["pattern"], ops["H"])
    order = hp.dissection_order(v, H, leaf=16)
    assert np.array_equal(np.sort(order), np.arange(v.shape[0]))
    b = np.zeros(v.shape[0])
    b[5] = 1.0
    default, dissected = hp.HeatFactor(H).solve(b), hp.HeatFactor(H, v).solve(b)
    mask = default > 1e-250
    assert np.max(np.abs(dissected - default)[mask] / default[mask]) <= 1e-12
    P = hp.csr_matrix(ops["pattern"], ops["P"])
    r = np.random.default_rng(1).normal(size=v.shape[0])
    r -= r.mean()
    x, y = hp.PoissonFactor(P).solve(r), hp.PoissonFactor(P, v).solve(r)
    assert hp.relative_linf(y - y.mean(), x - x.mean()) <= 1e-12


def test_extend_scalar_between_the_poles(known: dict) -> None:
    """ordito/heat.py:2394-2411: +1 at the north pole, -1 at the south; each hemisphere away from
    the equator takes its pole's value."""
    item = known["extend_scalar_poles_icosphere3"]
    v, f = creation.icosphere(3)
    heights = v[:, 2]
    poles = np.array([np.argmax(heights), np.argmin(heights)])
    extended, excess = hp.extend_scalar(v, f, poles, np.array(item["values"]))
    assert f"{extended[heights > 0.5].min():.2f}" == item["north_min"]
    assert f"{extended[heights < -0.5].max():.2f}" == item["south_max"]
    assert excess <= 1e-4
