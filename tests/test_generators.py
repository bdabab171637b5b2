"""Host-side mesh generators (the synthetic workloads' inputs)."""

from __future__ import annotations

import numpy as np
import pytest

from ordito_b200 import creation


@pytest.mark.parametrize("s", [0, 1, 2, 3, 5])
def test_icosphere_sizes_and_radius(s: int) -> None:
    v, f = creation.icosphere(s)
    assert v.shape == (10 * 4**s + 2, 3) and f.shape == (20 * 4**s, 3)
    assert v.dtype == np.float32 and f.dtype == np.int32
    assert np.allclose(np.linalg.norm(v.astype(np.float64), axis=1), 1.0, atol=1e-6)
    assert np.unique(f).size == v.shape[0]


def test_icosphere_numbering_starts_with_the_base_corners() -> None:
    base, _ = creation.icosphere(0)
    v, _ = creation.icosphere(3)
    assert np.array_equal(v[:12], base)


def test_icosphere_is_closed_and_oriented() -> None:
    v, f = creation.icosphere(3)
    edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    directed = {tuple(e) for e in edges.tolist()}
    assert len(directed) == edges.shape[0]
    assert all((b, a) in directed for a, b in directed)
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    assert (np.einsum("ij,ij->i", n, v[f].mean(axis=1)) > 0).all()


def test_torus_sizes_and_jitter_is_seeded() -> None:
    v, f = creation.jittered_torus(512, 256, seed=11)
    assert v.shape == (131072, 3) and f.shape == (262144, 3)
    v2, _ = creation.jittered_torus(512, 256, seed=11)
    assert np.array_equal(v, v2)
    clean, _ = creation.torus(512, 256)
    h = creation.mean_face_edge_length(clean, f)
    assert 0.05 * h < np.std(v.astype(np.float64) - clean) < 0.2 * h
