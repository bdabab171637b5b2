"""Packed meshes (GPU): many meshes of uneven sizes as one block-diagonal system, every mesh's
single-source queries answered by one batched pass, each equal to the mesh solved alone and to the
float64 oracle."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import _lib, creation
from ordito_b200 import heat as gheat
from ordito_b200.mesh import Trimesh
from ordito_b200.packed import PackedMeshes

pytestmark = pytest.mark.gpu

DISTANCE_TOL = 1e-5
ALONE_TOL = 1e-9  # the same mesh solved alone: the same blocks, another ordering and h summation


def _meshes():
    return [
        creation.icosphere(2),
        creation.jittered_torus(24, 12, seed=1),
        creation.icosphere(3),
        creation.jittered_torus(40, 20, seed=2),
        creation.jittered_torus(16, 8, seed=3),
        creation.icosphere(4),
    ]


def test_packed_batch_matches_each_mesh(gpu) -> None:
    meshes = _meshes()
    rng = np.random.default_rng(0)
    queries = [rng.choice(v.shape[0], size=int(rng.integers(1, 6)), replace=False).tolist()
               for v, _ in meshes]
    packed = PackedMeshes(meshes, max_columns=8)
    results = packed.solve(queries)
    for (v, f), q, got in zip(meshes, queries, results):
        assert got.shape == (len(q), v.shape[0])
        alone = gheat.heat_geodesic_batch(Trimesh(v, f.reshape(-1)), [[s] for s in q], refine=0).numpy()
        assert hp.relative_linf(got, alone) <= ALONE_TOL
        assert hp.relative_linf(got[0], hp.heat_geodesic(v, f, np.array([q[0]]))) <= DISTANCE_TOL
    packed.close()


def test_packed_recorded_pass(gpu) -> None:
    meshes = _meshes()
    queries = [[0], [5, 6], [1], [2, 3, 4], [7], [9, 10]]
    packed = PackedMeshes(meshes, max_columns=4)
    k = packed.load(queries)
    eager = packed.run(k).numpy()[:k].copy()
    stream = ctypes.c_void_p(0)
    _lib.call("ob_stream_create", ctypes.byref(stream))
    packed.record(k, stream)
    before = _lib.launch_count()
    packed.replay(k, stream)
    _lib.call("ob_stream_synchronize", stream)
    assert _lib.launch_count() > before
    assert hp.relative_linf(packed.out.numpy()[:k], eager) <= 1e-12
    with pytest.raises(ValueError):
        packed.load([[0]] * 5)  # one list per mesh
    with pytest.raises(ValueError):
        packed.load([[10**6]] + [[0]] * 5)
    packed.close()
    _lib.call("ob_stream_destroy", stream)
