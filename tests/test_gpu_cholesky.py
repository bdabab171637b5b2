"""Device Cholesky solves and the batched served path against the oracle (GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import creation
from ordito_b200 import heat as gheat
from ordito_b200.cholesky import OperatorFactorization, sparse_cholesky
from ordito_b200.device import DeviceArray
from ordito_b200.mesh import Trimesh
from tests import meshes

pytestmark = pytest.mark.gpu

DISTANCE_TOL = 1e-5


@pytest.mark.parametrize("name", ["ico3", "saddle_graded", "bumpy_sphere", "small_torus", "unreferenced"])
@pytest.mark.parametrize("k", [1, 5, 64])
def test_heat_system_factor_solves_many_columns(gpu, name: str, k: int) -> None:
    v, f = meshes.ALL[name]()
    n = v.shape[0]
    ops = gheat.heat_operators(v, f.reshape(-1), method="meshlab")
    chol = sparse_cholesky(ops.heat_system, v)
    rng = np.random.default_rng(k)
    B = np.zeros((n, k))
    for c in range(k):
        B[rng.integers(0, n), c] = 1.0
    X = DeviceArray.zeros(n * k, np.float64)
    chol.solve(B.reshape(-1), X, componentwise=True)
    got = X.numpy().reshape(n, k)
    # The device's own operator, solved directly on the host (its float32 geometry rounds like
    # the device's, not like the oracle's).
    ref = hp.solve_heat(ops.heat_system.to_scipy(), B)
    mask = ref > 1e-250
    assert np.max(np.abs(got - ref)[mask] / ref[mask]) <= 1e-8


def test_poisson_factor_is_the_consistent_solution(gpu) -> None:
    v, f = meshes.bumpy_sphere()
    ops = gheat.heat_operators(v, f.reshape(-1), method="meshlab")
    slot = OperatorFactorization(ops.poisson_system, v, singular=True)
    assert slot.factor()
    rng = np.random.default_rng(3)
    b = rng.normal(size=v.shape[0])
    b -= b.mean()
    x = DeviceArray.zeros(v.shape[0], np.float64)
    slot.solve(b, x)
    got = x.numpy()
    ref = hp.PoissonFactor(ops.poisson_system.to_scipy()).solve(b)
    assert hp.relative_linf(got - got.mean(), ref - ref.mean()) <= 1e-9


@pytest.mark.parametrize("name", ["ico3", "small_torus", "bumpy_sphere", "saddle_graded"])
def test_batched_queries_match_the_oracle_and_single_queries(gpu, name: str) -> None:
    v, f = meshes.ALL[name]()
    n = v.shape[0]
    rng = np.random.default_rng(7)
    sets = [rng.choice(n, size=int(s), replace=False) for s in rng.integers(1, 6, size=9)]
    mesh = Trimesh(v, f.reshape(-1))
    batch = gheat.heat_geodesic_batch(mesh, sets).numpy()
    assert batch.shape == (len(sets), n)
    t_eff, _ = hp.vertex_time(v, f, None)
    ops = hp.heat_operators(v, f, t_eff)
    factors = (hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"])),
               hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"])))
    for c, s in enumerate(sets):
        ref = hp.heat_geodesic(v, f, s, operators=ops, factors=factors)
        assert hp.relative_linf(batch[c], ref) <= DISTANCE_TOL
        alone = gheat.heat_geodesic_batch(mesh, [s]).numpy()[0]
        assert hp.relative_linf(alone, batch[c]) <= 1e-9


def test_batched_sources_are_validated(gpu) -> None:
    v, f = creation.icosphere(2)
    mesh = Trimesh(v, f.reshape(-1))
    with pytest.raises(ValueError):
        gheat.heat_geodesic_batch(mesh, [[0], [v.shape[0]]])
    with pytest.raises(ValueError):
        gheat.heat_geodesic_batch(mesh, [[0], []])


def test_full_size_torus_single_query(gpu) -> None:
    """The 131 072-vertex jittered torus: the settled iterate fails its backward-error check
    (the idle bound stops it before the far field settles), and the factored fallback answers."""
    v, f = creation.jittered_torus(512, 256, seed=0)
    src = np.array([5], dtype=np.int32)
    got = gheat.heat_geodesic(v, f.reshape(-1), src).numpy()
    ref = hp.heat_geodesic(v, f, src)
    assert hp.relative_linf(got, ref) <= DISTANCE_TOL


@pytest.mark.parametrize("name", ["ico3", "bumpy_sphere", "unreferenced", "degenerate"])
def test_corner_index_is_the_stable_sort_of_the_faces(gpu, name: str) -> None:
    v, f = meshes.ALL[name]()
    mesh = Trimesh(v, f.reshape(-1))
    offsets, slots = mesh.corner_index
    flat = f.reshape(-1)
    order = np.argsort(flat, kind="stable")
    expected_offsets = np.searchsorted(flat[order], np.arange(v.shape[0] + 1))
    assert np.array_equal(offsets.numpy(), expected_offsets)
    assert np.array_equal(slots.numpy()[: flat.size], order)


@pytest.mark.parametrize("k", [1, 3, 64])
def test_gathered_divergence_matches_the_scattered_one_and_repeats_bit_for_bit(gpu, k: int) -> None:
    from ordito_b200 import _lib

    v, f = meshes.bumpy_sphere()
    n = v.shape[0]
    mesh = Trimesh(v, f.reshape(-1))
    terms = mesh.face_terms
    rng = np.random.default_rng(k)
    u = DeviceArray.from_host(np.exp(-5.0 * rng.random((n, k))).reshape(-1))
    scattered = DeviceArray.empty(n * k, np.float64)
    _lib.call("ob_grad_div", mesh.vertices.ptr, mesh.faces.ptr, mesh.n_faces, n, terms.normals.ptr,
              terms.areas.ptr, u.ptr, terms.cot.ptr, k, scattered.ptr, None)
    offsets, slots = mesh.corner_index
    gathered = [DeviceArray.empty(n * k, np.float64) for _ in range(2)]
    for out in gathered:
        _lib.call("ob_grad_div_gather", mesh.vertices.ptr, mesh.faces.ptr, terms.normals.ptr,
                  terms.areas.ptr, terms.cot.ptr, offsets.ptr, slots.ptr, n, k, u.ptr, k, None,
                  out.ptr, k, None, None, None)
    a, b, c = scattered.numpy(), gathered[0].numpy(), gathered[1].numpy()
    assert np.array_equal(b, c)
    assert np.allclose(b, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


@pytest.mark.parametrize("k", [1, 3, 64])
def test_divergence_from_face_terms(gpu, k: int) -> None:
    # The per-face-terms divergence agrees with the gathered one, repeats bit for bit, and -- its
    # gradient rescaled by an exact power of two -- is unchanged bit for bit when u is scaled by
    # 2^-900, the far field's magnitude (the unit gradient is scale-free).
    from ordito_b200 import _lib

    v, f = meshes.bumpy_sphere()
    n = v.shape[0]
    mesh = Trimesh(v, f.reshape(-1))
    terms = mesh.face_terms
    rng = np.random.default_rng(k)
    host_u = np.exp(-5.0 * rng.random((n, k))).reshape(-1)
    u = DeviceArray.from_host(host_u)
    tiny = DeviceArray.from_host(np.ldexp(host_u, -900))
    offsets, slots = mesh.corner_index
    gathered = DeviceArray.empty(n * k, np.float64)
    _lib.call("ob_grad_div_gather", mesh.vertices.ptr, mesh.faces.ptr, terms.normals.ptr,
              terms.areas.ptr, terms.cot.ptr, offsets.ptr, slots.ptr, n, k, u.ptr, k, None,
              gathered.ptr, k, None, None, None)
    table = DeviceArray.empty((mesh.n_faces, 18), np.float64)
    _lib.call("ob_face_gradient_terms", mesh.vertices.ptr, mesh.faces.ptr, mesh.n_faces,
              terms.normals.ptr, terms.areas.ptr, terms.cot.ptr, table.ptr, None)
    outs = []
    for field in (u, u, tiny):
        out = DeviceArray.empty(n * k, np.float64)
        _lib.call("ob_grad_div_terms", table.ptr, mesh.faces.ptr, offsets.ptr, slots.ptr, n, k,
                  field.ptr, k, None, out.ptr, k, None, None, None)
        outs.append(out.numpy())
    reference = gathered.numpy()
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], outs[2])
    assert np.allclose(outs[0], reference, rtol=1e-12, atol=1e-12 * np.abs(reference).max())
    # Face by face over tiles: the same sums to rounding, the same bits on every run.
    tiles = mesh.corner_tiles
    tiled = []
    for field in (u, u, tiny):
        out = DeviceArray.empty(n * k, np.float64)
        _lib.call("ob_grad_div_tiled", table.ptr, mesh.faces.ptr, *(a.ptr for a in tiles), n, k,
                  field.ptr, k, None, out.ptr, k, None, None, None)
        tiled.append(out.numpy())
    assert np.array_equal(tiled[0], tiled[1])
    assert np.array_equal(tiled[0], tiled[2])
    assert np.allclose(tiled[0], outs[0], rtol=1e-13, atol=1e-13 * np.abs(outs[0]).max())
    # Over corner records: the per-corner form's arithmetic in its corner order, so its bits.
    from ordito_b200.heat import corner_records

    records, ids = corner_records(table, mesh.faces, slots, mesh.n_faces)
    for field, expected in ((u, outs[0]), (tiny, outs[2])):
        out = DeviceArray.empty(n * k, np.float64)
        _lib.call("ob_grad_div_records", records.ptr, ids.ptr, offsets.ptr, n, k, field.ptr, k, None, out.ptr, k,
                  None, None, None)
        assert np.array_equal(out.numpy(), expected)


def test_tiled_divergence_on_a_crowded_fan(gpu) -> None:
    # A vertex on 1 500 faces: its tile has too many corners for shared memory and takes the
    # per-corner form; every other tile the face-major one. Both against the per-corner kernel.
    from ordito_b200 import _lib

    ring = 1500
    angle = 2.0 * np.pi * np.arange(ring) / ring
    rim = np.column_stack((np.cos(angle), np.sin(angle), 0.1 * np.sin(7 * angle)))
    v = np.vstack(([[0.0, 0.0, 0.3]], rim)).astype(np.float32)
    f = np.array([[0, 1 + i, 1 + (i + 1) % ring] for i in range(ring)], dtype=np.int32)
    n, k = v.shape[0], 6
    mesh = Trimesh(v, f.reshape(-1))
    terms = mesh.face_terms
    table = DeviceArray.empty((mesh.n_faces, 18), np.float64)
    _lib.call("ob_face_gradient_terms", mesh.vertices.ptr, mesh.faces.ptr, mesh.n_faces,
              terms.normals.ptr, terms.areas.ptr, terms.cot.ptr, table.ptr, None)
    u = DeviceArray.from_host(np.random.default_rng(3).random(n * k))
    offsets, slots, tile_faces, tile_counts, codes = mesh.corner_tiles
    assert tile_counts.numpy()[0] == -1 and (tile_counts.numpy()[1:] > 0).all()
    expected, got = DeviceArray.empty(n * k, np.float64), DeviceArray.empty(n * k, np.float64)
    _lib.call("ob_grad_div_terms", table.ptr, mesh.faces.ptr, offsets.ptr, slots.ptr, n, k, u.ptr, k,
              None, expected.ptr, k, None, None, None)
    _lib.call("ob_grad_div_tiled", table.ptr, mesh.faces.ptr, offsets.ptr, slots.ptr, tile_faces.ptr,
              tile_counts.ptr, codes.ptr, n, k, u.ptr, k, None, got.ptr, k, None, None, None)
    e = expected.numpy()
    assert np.allclose(got.numpy(), e, rtol=1e-13, atol=1e-13 * np.abs(e).max())


def test_recorded_batch_step_matches_the_eager_pass(gpu) -> None:
    import ctypes

    from ordito_b200 import _lib

    v, f = meshes.small_torus()
    n = v.shape[0]
    rng = np.random.default_rng(9)
    sets = [rng.choice(n, size=int(s), replace=False).tolist() for s in rng.integers(1, 4, size=8)]
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    assert solver.factor()
    src, offsets, k = gheat._source_columns(sets, n)
    eager = gheat._batch_columns(mesh, solver, src, offsets, k, 0, True).numpy()
    stream = ctypes.c_void_p(0)
    _lib.call("ob_stream_create", ctypes.byref(stream))
    step = gheat.BatchStep(mesh, solver, src, offsets, k, DeviceArray.empty((k, n), np.float64), stream)
    assert step.kernels > 0
    before = _lib.launch_count()
    out = step.launch()
    _lib.call("ob_stream_synchronize", stream)
    assert _lib.launch_count() - before == step.kernels
    assert hp.relative_linf(out.numpy(), eager) <= 1e-12
    # New sources written into the same buffers are read by the next replay.
    other = [[int(s[0]) + 1] for s in sets]
    src2, offsets2, _ = gheat._source_columns(other, n)
    _lib.call("ob_memcpy", src.ptr, src2.ptr, src2.nbytes, 2, None, 1)
    _lib.call("ob_memcpy", offsets.ptr, offsets2.ptr, offsets2.nbytes, 2, None, 1)
    step.launch()
    _lib.call("ob_stream_synchronize", stream)
    replay = step.out.numpy()
    expected = gheat._batch_columns(mesh, solver, src2, offsets2, k, 0, True).numpy()
    assert hp.relative_linf(replay, expected) <= 1e-12
    step.close()
    _lib.call("ob_stream_destroy", stream)


@pytest.mark.parametrize("refine", [0, 1])
def test_batched_modes_agree_and_repeat(gpu, refine: int) -> None:
    v, f = meshes.small_torus()
    n = v.shape[0]
    rng = np.random.default_rng(3)
    sets = [rng.choice(n, size=int(s), replace=False) for s in rng.integers(1, 4, size=7)]
    mesh = Trimesh(v, f.reshape(-1))
    first = gheat.heat_geodesic_batch(mesh, sets, refine=refine).numpy()
    again = gheat.heat_geodesic_batch(mesh, sets, refine=refine).numpy()
    assert np.array_equal(first, again) or hp.relative_linf(again, first) <= 1e-12
    t_eff, _ = hp.vertex_time(v, f, None)
    ops = hp.heat_operators(v, f, t_eff)
    factors = (hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"])),
               hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"])))
    for c, s in enumerate(sets):
        ref = hp.heat_geodesic(v, f, s, operators=ops, factors=factors)
        assert hp.relative_linf(first[c], ref) <= DISTANCE_TOL
    untransposed = gheat.heat_geodesic_batch(mesh, sets, refine=refine, transpose=False).numpy()
    assert np.allclose(untransposed.T, first, rtol=0, atol=1e-12 * np.abs(first).max())


def test_batch_pipeline_matches_the_batched_pass(gpu) -> None:
    v, f = meshes.small_torus()
    n = v.shape[0]
    mesh = Trimesh(v, f.reshape(-1))
    rng = np.random.default_rng(4)
    batches = [[rng.choice(n, size=int(s), replace=False).tolist() for s in rng.integers(1, 4, size=5)]
               for _ in range(5)]
    pipe = gheat.BatchPipeline(mesh, 5)
    results = [r.copy() for r in pipe.map(batches)]
    pipe.close()
    assert len(results) == len(batches)
    for sets, got in zip(batches, results):
        expected = gheat.heat_geodesic_batch(mesh, sets, refine=0).numpy()
        assert hp.relative_linf(got, expected) <= 1e-12
    with pytest.raises(ValueError):
        list(gheat.BatchPipeline(mesh, 2).map([[[0], [n]]]))


def test_two_work_sets_give_the_same_answers(gpu) -> None:
    import ctypes

    from ordito_b200 import _lib

    v, f = meshes.small_torus()
    n = v.shape[0]
    rng = np.random.default_rng(11)
    sets = [rng.choice(n, size=2, replace=False).tolist() for _ in range(9)]
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    assert solver.factor()
    src, offsets, k = gheat._source_columns(sets, n)
    streams = [ctypes.c_void_p(0), ctypes.c_void_p(0)]
    for s in streams:
        _lib.call("ob_stream_create", ctypes.byref(s))
    steps = [gheat.BatchStep(mesh, solver, src, offsets, k, DeviceArray.empty((k, n), np.float64),
                             streams[w], work_set=w) for w in range(2)]
    for _ in range(3):  # both sets in flight at once
        for w in range(2):
            steps[w].launch(streams[w])
    for s in streams:
        _lib.call("ob_stream_synchronize", s)
    a, b = steps[0].out.numpy(), steps[1].out.numpy()
    assert hp.relative_linf(a, b) <= 1e-12
    expected = gheat._batch_columns(mesh, solver, src, offsets, k, 0, True).numpy()
    assert hp.relative_linf(a, expected) <= 1e-12
    for step in steps:
        step.close()
    for s in streams:
        _lib.call("ob_stream_destroy", s)


def test_pass_schedules_agree_and_the_tuner_keeps_one(gpu) -> None:
    # Every tile schedule computes the same solve (split tiles only change the order of the
    # atomic sums); the tuner keeps one of its candidates, and a recorded batch pass made before
    # the retiling records again and still answers the same.
    from ordito_b200 import _lib
    from ordito_b200.tuning import CANDIDATES, tune_pass

    v, f = meshes.small_torus()
    n = v.shape[0]
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    assert solver.factor()
    rng = np.random.default_rng(2)
    sets = [[int(s)] for s in rng.choice(n, size=8, replace=False)]
    src, offsets, k = gheat._source_columns(sets, n)
    import ctypes

    stream = ctypes.c_void_p(0)
    _lib.call("ob_stream_create", ctypes.byref(stream))
    out = DeviceArray.empty((k, n), np.float64)
    step = gheat.BatchStep(mesh, solver, src, offsets, k, out, stream)
    step.launch()
    _lib.call("ob_stream_synchronize", stream)
    before = step.out.numpy()
    answers = []
    for chunk, waves in ((0, 0), (32, 4), (64, 2)):
        _lib.call("ob_chol_tile", solver.heat_factor.handle, chunk, waves, None)
        _lib.call("ob_chol_tile", solver.poisson_factor.handle, chunk, waves, None)
        answers.append(gheat._batch_columns(mesh, solver, src, offsets, k, 0, True).numpy())
    for a in answers:
        assert np.allclose(a, before, rtol=0, atol=1e-12 * np.abs(before).max())
    report = tune_pass(solver.heat_factor, k, reps=2)
    assert report["best"] in CANDIDATES and set(report["ms"]) == set(CANDIDATES)
    step.launch()
    _lib.call("ob_stream_synchronize", stream)
    after = step.out.numpy()
    assert np.allclose(after, before, rtol=0, atol=1e-12 * np.abs(before).max())
    step.close()
    _lib.call("ob_stream_destroy", stream)
    mesh.dispose()


def test_forward_pass_over_marked_sources_equals_the_full_pass(gpu) -> None:
    # Source indicators leave every supernode off their paths to the root with a zero input
    # block: the pass that runs only the marked ones (narrow and tensor-core kernels) answers as
    # the full pass does.
    from ordito_b200 import _lib

    v, f = meshes.small_torus()
    n = v.shape[0]
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    assert solver.factor()
    factor = solver.heat_factor
    rng = np.random.default_rng(4)
    for k in (1, 5, 64):
        sets = [rng.choice(n, size=int(rng.integers(1, 4)), replace=False).tolist() for _ in range(k)]
        src, offsets, _ = gheat._source_columns(sets, n)
        results = []
        for sparse in (False, True):
            rhs, sol, stride, iperm, pinned = factor.work(k)
            _lib.call("ob_seed_permuted", src.ptr, offsets.ptr, k, n, iperm, pinned, stride, rhs, None)
            if sparse:
                factor.solve_in_place_sources(k, src, offsets, None)
            else:
                factor.solve_in_place(k, None)
            results.append(DeviceArray(sol, (n, stride), np.float64, owned=False).numpy()[:, :k].copy())
        full, marked = results
        assert np.allclose(marked, full, rtol=0, atol=1e-14 * np.abs(full).max())
    mesh.dispose()
