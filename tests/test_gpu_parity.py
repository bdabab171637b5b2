"""Parity of the benchmarked configurations against the float64 oracle, at their full sizes.

- The served + batched pass the benchmark times: the jittered torus 512 x 256 (seed 0), 64
  single-source queries (``default_rng(1)``), one recorded pass a batch on each of the factors'
  three work sets: every column of every work set against the oracle.
- The same workload's other reading: one query whose source set is all 64 vertices.
- The packed batch of 256 uneven meshes (seed 0): 16 sampled meshes, every query of each.
- The large sphere (icosphere(9) + 1 % radial noise, 8 queries), past the factorisation budget:
  the mixed-precision path (settled CG + band march for the heat, float32 multigrid CG inside
  float64 refinement for the Poisson system) and a plain float64 path (Poisson by float64 CG under
  the Jacobi-Chebyshev polynomial), both against the oracle's distances committed in
  ``tests/golden/oracle_ico9_sample.npz`` (the oracle needs minutes and tens of GB there).

Distances are compared as the relative L-inf error over the oracle's range, at 1e-5.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import _lib, creation
from ordito_b200 import heat as gheat
from ordito_b200 import linalg as twl
from ordito_b200.device import DeviceArray, synchronize
from ordito_b200.mesh import Trimesh

pytestmark = pytest.mark.gpu

DISTANCE_TOL = 1e-5
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def torus_workload() -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    vertices, faces = creation.jittered_torus(512, 256, 1.0, 0.3, 0.1, seed=0)
    sources = np.random.default_rng(1).choice(vertices.shape[0], size=64, replace=False).astype(np.int32)
    return vertices, faces, sources


@pytest.fixture(scope="module")
def torus():
    vertices, faces, sources = torus_workload()
    t_eff, _ = hp.vertex_time(vertices, faces, None)
    ops = hp.heat_operators(vertices, faces, t_eff)
    factors = (hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"])),
               hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"])))
    mesh = Trimesh(vertices, faces.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    assert solver.factor()
    yield vertices, faces, sources, ops, factors, mesh, solver
    mesh.dispose()


def test_benchmark_pass_every_column_every_work_set(gpu, torus) -> None:
    vertices, faces, sources, ops, factors, mesh, solver = torus
    n, k = vertices.shape[0], len(sources)
    src, offsets, _ = gheat._source_columns([[int(s)] for s in sources], n)
    streams, steps = [], []
    for w in range(3):
        stream = ctypes.c_void_p(0)
        _lib.call("ob_stream_create", ctypes.byref(stream))
        streams.append(stream)
        steps.append(gheat.BatchStep(mesh, solver, src, offsets, k, DeviceArray.empty((k, n), np.float64),
                                     stream, work_set=w))
    # Three batches in flight, as the benchmark runs them, then every result read back.
    for _ in range(2):
        for w in range(3):
            steps[w].launch(streams[w])
    synchronize()
    results = [steps[w].out.numpy() for w in range(3)]
    reference = np.stack([hp.heat_geodesic(vertices, faces, np.array([s]), operators=ops, factors=factors)
                          for s in sources])
    for w in range(3):
        errors = [hp.relative_linf(results[w][c], reference[c]) for c in range(k)]
        assert max(errors) <= DISTANCE_TOL, (w, int(np.argmax(errors)), max(errors))
        assert np.all(results[w][np.arange(k), sources] == 0.0)
    # The work sets share only the read-only factors: the same batch answers alike on each.
    assert np.max(np.abs(results[1] - results[0])) <= 1e-12 * np.abs(results[0]).max()
    assert np.max(np.abs(results[2] - results[0])) <= 1e-12 * np.abs(results[0]).max()
    for step in steps:
        step.close()
    for stream in streams:
        _lib.call("ob_stream_destroy", stream)


def test_benchmark_multi_source_query(gpu, torus) -> None:
    vertices, faces, sources, ops, factors, mesh, _ = torus
    got = gheat.heat_geodesic(mesh, sources).numpy()
    ref = hp.heat_geodesic(vertices, faces, sources, operators=ops, factors=factors)
    assert hp.relative_linf(got, ref) <= DISTANCE_TOL
    # The shift takes the mean over the sources (heat.py:3134): it is their mean that is 0.
    assert abs(float(got[sources].mean())) <= 1e-12


def test_packed_batch_sampled_meshes(gpu) -> None:
    from ordito_b200.packed import PackedMeshes, packed_workload

    work = packed_workload(0, 256)
    packed = PackedMeshes(work.meshes, max_columns=16)
    try:
        k = packed.load(work.queries)
        stream = ctypes.c_void_p(0)
        _lib.call("ob_stream_create", ctypes.byref(stream))
        packed.record(k, stream)
        packed.replay(k, stream)
        _lib.call("ob_stream_synchronize", stream)
        out = packed.out.numpy()
        picked = np.random.default_rng(11).choice(len(work.meshes), size=16, replace=False)
        worst = 0.0
        for m in sorted(int(x) for x in picked):
            v, f = work.meshes[m]
            t_eff, _ = hp.vertex_time(v, f, None)
            ops = hp.heat_operators(v, f, t_eff)
            factors = (hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"])),
                       hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"])))
            rows = slice(packed.vertex_offsets[m], packed.vertex_offsets[m + 1])
            for c, s in enumerate(work.queries[m]):
                ref = hp.heat_geodesic(v, f, np.array([s]), operators=ops, factors=factors)
                error = hp.relative_linf(out[c, rows], ref)
                worst = max(worst, error)
                assert error <= DISTANCE_TOL, (m, c, error)
        assert worst > 0.0
        _lib.call("ob_stream_destroy", stream)
    finally:
        packed.close()


@pytest.fixture(scope="module")
def large_sphere():
    golden = np.load(os.path.join(GOLDEN, "oracle_ico9_sample.npz"))
    vertices, faces = creation.icosphere(9)
    vertices = creation.radial_noise(vertices, 0.01, 0)
    sources = np.random.default_rng(5).choice(vertices.shape[0], 8, replace=False).astype(np.int32)
    assert np.array_equal(sources, golden["sources"])
    mesh = Trimesh(vertices, faces.reshape(-1))
    yield mesh, sources, golden
    mesh.dispose()


def _sampled_error(distance: np.ndarray, golden, c: int) -> float:
    sample = golden["sample"]
    return float(np.max(np.abs(distance[sample] - golden["distance"][c])) / golden["scale"][c])


def test_large_sphere_mixed_precision_path(gpu, large_sphere) -> None:
    mesh, sources, golden = large_sphere
    solver = mesh.heat_solver(None, method="meshlab")
    assert not solver.factor()  # 2.6 M vertices: over the factorisation budget
    for c, s in enumerate(sources):
        got = gheat.heat_geodesic(mesh, np.array([s], dtype=np.int32), method="meshlab").numpy()
        assert _sampled_error(got, golden, c) <= DISTANCE_TOL, (c, _sampled_error(got, golden, c))
        assert abs(float(got.sum()) - golden["total"][c]) <= 1e-5 * golden["scale"][c] * got.size


def test_large_sphere_plain_float64_path(gpu, large_sphere) -> None:
    # The same heat solve, the Poisson system by float64 CG under the Jacobi-Chebyshev polynomial
    # (no float32 anywhere in that solve), two of the queries.
    mesh, sources, golden = large_sphere
    solver = mesh.heat_solver(None, method="meshlab")
    n = mesh.n_vertices
    poisson = solver.operators.poisson_system
    chebyshev = twl.chebyshev_preconditioner(poisson)
    for c in (0, 5):
        host = np.zeros(n)
        host[int(sources[c])] = 1.0
        seed = DeviceArray.from_host(host)
        heat = DeviceArray.zeros(n, np.float64)
        solver.diffuse(seed, heat)
        neg_div = DeviceArray.empty(n, np.float64)
        gheat._divergence(mesh, solver, 1, heat.ptr, 1, None, neg_div.ptr, 1, None, None, None)
        phi = DeviceArray.zeros(n, np.float64)
        twl.solve_spd(poisson, neg_div, phi, tol=1e-8, preconditioner=chebyshev, name="plain")
        src = DeviceArray.from_host(np.array([sources[c]], dtype=np.int32))
        _lib.call("ob_shift", phi.ptr, n, src.ptr, 1, None, 1, 1, None)
        got = phi.numpy()
        assert _sampled_error(got, golden, c) <= DISTANCE_TOL, (c, _sampled_error(got, golden, c))
