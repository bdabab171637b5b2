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
