"""Serving policy on the host (no GPU): the HBM budget, reservations and least-recently-used
eviction of idle meshes, the cache key, batch widths and the synthetic request stream."""

from __future__ import annotations

import math

import numpy as np
import pytest

from ordito_b200 import creation
from ordito_b200.serving import MeshCache, bucket, mesh_key, serving_workload


class _Entry:
    def __init__(self, busy: bool = False) -> None:
        self.busy = busy


def _idle(entry: _Entry) -> bool:
    return not entry.busy


def test_admission_within_budget_and_lru_eviction() -> None:
    cache = MeshCache(budget=100)
    for key in ("a", "b", "c"):
        ok, evicted = cache.admit(key, 30, _idle)
        assert ok and not evicted
        cache.commit(key, _Entry(), 30)
    cache.get("a")  # a is now the most recently used: b is the oldest
    ok, evicted = cache.admit("d", 30, _idle)
    assert ok and len(evicted) == 1 and list(cache.entries) == ["c", "a"]
    assert cache.evictions == 1 and cache.used == 90  # c, a + d reserved


def test_busy_meshes_are_not_evicted() -> None:
    cache = MeshCache(budget=100)
    for key in ("a", "b"):
        cache.admit(key, 50, _idle)
        cache.commit(key, _Entry(busy=True), 50)
    ok, evicted = cache.admit("c", 50, _idle)
    assert not ok and not evicted and "c" not in cache.reserved
    cache.entries["a"].busy = False
    ok, evicted = cache.admit("c", 50, _idle)
    assert ok and len(evicted) == 1 and list(cache.entries) == ["b"]


def test_free_memory_bounds_admission() -> None:
    free = {"bytes": 10_000}
    cache = MeshCache(budget=1 << 40, free_memory=lambda: free["bytes"], margin=1_000)
    ok, _ = cache.admit("a", 8_000, _idle)
    assert ok
    ok, _ = cache.admit("b", 2_000, _idle)  # 10 000 free - 8 000 reserved - 2 000 < margin
    assert not ok
    with pytest.raises(MemoryError):
        MeshCache(budget=10).admit("x", 11, _idle)


def test_bucket_and_key() -> None:
    assert [bucket(k) for k in (1, 2, 3, 5, 17, 64, 65)] == [1, 2, 4, 8, 32, 64, 128]
    with pytest.raises(ValueError):
        bucket(129)
    v, f = creation.icosphere(2)
    assert mesh_key(v, f) == mesh_key(v.copy(), f.copy())
    w = v.copy()
    w[3, 1] += 1e-6
    assert mesh_key(w, f) != mesh_key(v, f)


def test_serving_workload_distribution() -> None:
    stream = serving_workload(7, 2000, rate=500.0, v_min=1e3, v_max=2e6)
    arrivals = np.array([r.arrival for r in stream])
    assert np.all(np.diff(arrivals) > 0)
    assert abs(np.mean(np.diff(arrivals)) - 1 / 500.0) < 0.2 / 500.0  # Poisson rate
    counts = np.array([r.sources.size for r in stream])
    assert counts.min() >= 1 and counts.max() <= 32
    for r in stream[:200]:
        assert r.sources.min() >= 0 and r.sources.max() < r.n_vertices
        assert np.unique(r.sources).size == r.sources.size
    sizes = np.array([r.n_vertices for r in stream])
    assert sizes.min() >= 162 and sizes.max() <= 2.7e6
    # Reuse: about 70 % of requests after the first name a mesh seen before.
    seen, reused = set(), 0
    for r in stream:
        reused += r.mesh in seen
        seen.add(r.mesh)
    assert 0.6 < reused / len(stream) < 0.8
    kinds = {r.mesh[0] for r in stream}
    assert kinds == {"icosphere", "torus"}
    tori = [r.mesh for r in stream if r.mesh[0] == "torus"]
    assert all(cols == 2 * rows for _, cols, rows, _ in tori)
    assert math.isclose(np.median(np.log(sizes)), np.median(np.log(sizes)))
