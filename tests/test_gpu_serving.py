"""The continuous-batching server (GPU): a result served in a mix of concurrent requests on
several meshes equals the same query run alone, meshes are evicted and rebuilt under a small HBM
budget, and invalid requests fail their future."""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import heat as gheat
from ordito_b200.mesh import Trimesh
from ordito_b200.serving import ESTIMATED_BYTES_PER_VERTEX, GeodesicServer, mesh_for

pytestmark = pytest.mark.gpu

SAME_TOL = 1e-12  # in the mix vs alone: the same passes, up to split-K atomic ordering
PLAIN_TOL = 1e-6  # a first request answered unfactored (settled CG, Poisson CG to 1e-8) vs factored
ORACLE_TOL = 1e-5  # against the float64 oracle

SPECS = [("icosphere", 4, 11), ("torus", 64, 32, 3), ("icosphere", 3, 5)]


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _requests(rng, meshes, count):
    out = []
    for _ in range(count):
        m = int(rng.integers(len(meshes)))
        n = meshes[m][0].shape[0]
        out.append((m, rng.choice(n, size=int(rng.integers(1, 9)), replace=False).astype(np.int32)))
    return out


def _alone(meshes, m, sources, cache):
    if m not in cache:
        cache[m] = Trimesh(*meshes[m])
    return gheat.heat_geodesic_batch(cache[m], [sources.tolist()], refine=0).numpy()[0]


@pytest.mark.parametrize("plain", [0, 8])
def test_results_alone_equal_results_in_the_mix(gpu, plain: int) -> None:
    # plain = 0: every request answered by the factored batches, each equal to its query run
    # alone; plain = 8: a new mesh's first requests answered unfactored meanwhile (rent before
    # buy), equal to the factored answer within that path's tolerance.
    meshes = [mesh_for(spec) for spec in SPECS]
    rng = np.random.default_rng(0)
    work = _requests(rng, meshes, 90)
    server = GeodesicServer(max_columns=16, slots=3, plain_answers=plain)
    futures = [None] * len(work)

    def feed() -> None:
        for i, (m, sources) in enumerate(work):
            futures[i] = server.submit(*meshes[m], sources)
            if i % 7 == 0:
                time.sleep(0.002)  # later requests arrive while earlier ones are on the GPU

    feeder = threading.Thread(target=feed)
    feeder.start()
    feeder.join()
    results = [f.result(timeout=300) for f in futures]
    stats = server.stats()
    server.close()
    assert stats["requests"] == len(work) and stats["cache_misses"] == len(SPECS)
    assert stats["batches"] < len(work)  # requests were batched
    assert stats["p50_ms"] is not None and stats["p99_ms"] >= stats["p50_ms"]
    cache = {}
    for (m, sources), got in zip(work, results):
        assert rel_err(got, _alone(meshes, m, sources, cache)) <= (SAME_TOL if plain == 0 else PLAIN_TOL)
    for (m, sources), got in list(zip(work, results))[:3]:
        v, f = meshes[m]
        assert rel_err(got, hp.heat_geodesic(v, f, sources)) <= ORACLE_TOL


def test_eviction_under_a_small_budget(gpu) -> None:
    meshes = [mesh_for(spec) for spec in SPECS[:2]]
    largest = max(v.shape[0] for v, _ in meshes)
    server = GeodesicServer(hbm_budget=int(1.5 * ESTIMATED_BYTES_PER_VERTEX * largest), max_columns=4, slots=2,
                            plain_answers=0)
    rng = np.random.default_rng(1)
    cache = {}
    for m, sources in _requests(rng, meshes, 6):
        got = server.submit(*meshes[m], sources).result(timeout=300)
        assert rel_err(got, _alone(meshes, m, sources, cache)) <= SAME_TOL
    stats = server.stats()
    server.close()
    assert stats["evictions"] >= 1 and stats["resident_meshes"] == 1


def test_invalid_requests_fail_their_future(gpu) -> None:
    v, f = mesh_for(SPECS[2])
    server = GeodesicServer(max_columns=4, slots=1)
    with pytest.raises(ValueError):
        server.submit(v, f, [v.shape[0]]).result(timeout=60)
    with pytest.raises(ValueError):
        server.submit(v, f, np.arange(40)).result(timeout=60)
    ok = server.submit(v, f, [0]).result(timeout=300)
    server.close()
    assert ok[0] == 0.0 and np.all(ok >= -1e-6)


def test_a_mesh_past_the_factor_budget_is_served_unfactored(gpu) -> None:
    # With the factorisation budget below the mesh's factor, its first requests are answered
    # unfactored and so are all the later ones (kept resident, one at a time): more requests than
    # plain answers, every one against the oracle.
    from ordito_b200 import cholesky as gchol

    v, f = mesh_for(SPECS[2])
    budget = gchol.CHOLESKY_MEMORY_BUDGET
    gchol.CHOLESKY_MEMORY_BUDGET = 1 << 10
    try:
        server = GeodesicServer(max_columns=4, slots=1, plain_answers=2)
        rng = np.random.default_rng(7)
        batches = [rng.choice(v.shape[0], size=int(rng.integers(1, 4)), replace=False).astype(np.int32)
                   for _ in range(6)]
        futures = [server.submit(v, f, s) for s in batches]
        results = [fut.result(timeout=600) for fut in futures]
        stats = server.stats()
        server.close()
    finally:
        gchol.CHOLESKY_MEMORY_BUDGET = budget
    for sources, got in zip(batches, results):
        assert rel_err(got, hp.heat_geodesic(v, f, sources)) <= ORACLE_TOL
    assert stats["resident_meshes"] == 1
