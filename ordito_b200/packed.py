"""Many meshes of uneven sizes solved together: one block-diagonal system, one batched pass.

The batched form of ``heat_geodesic`` over many meshes (ordito/heat.py:391 for each): the meshes'
vertices and faces are concatenated -- each face offset by its mesh's first vertex -- so the
pattern (a1), the face terms (a2, a3), the operator rows (a5, each mesh with its own time step
t = h^2 from its own face edges and its own diffusion floor, a4), the two factorisations (a11) and
the divergence (a8) are built and run once over the union, whose operators are block diagonal. For
the nested-dissection analysis only, each mesh is translated apart, so the dissection separates
meshes first at no fill. Queries are single-source: column c of the batch carries every mesh's
c-th source, so one pass over ``max queries per mesh`` columns answers every query of every mesh;
the shift (a13) runs per (mesh, column). The whole pass can be recorded as one CUDA graph
(``PackedMeshes.record``) and replayed with a single launch.

Each mesh's distances equal its own ``heat_geodesic`` up to rounding: the blocks do not couple, and
a mesh's rows of L are the same sums in the same order as its own.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

import numpy as np

from ordito_b200 import _lib
from ordito_b200.array import CsrMatrix
from ordito_b200.cholesky import CholeskyAnalysis, SparseCholesky
from ordito_b200.device import DEFAULT_STREAM, DeviceArray
from ordito_b200.heat import _bounds_floor_length, capture_guard
from ordito_b200.laplacian import face_terms, mesh_operator_pattern


def mesh_bounds(xyz: np.ndarray, vertex_offsets: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Each packed mesh's bounding box in one pass over the union's float32 vertices (``xyz``,
    mesh m's rows ``vertex_offsets[m] .. vertex_offsets[m + 1]``): its low and high corners (the
    float32 extremes a per-mesh ``min`` / ``max`` gives; zeros for an empty mesh) and the indices
    of the meshes that have vertices."""
    counts = np.diff(vertex_offsets)
    nonempty = np.flatnonzero(counts > 0)
    low = np.zeros((counts.size, 3), dtype=np.float32)
    high = np.zeros((counts.size, 3), dtype=np.float32)
    if nonempty.size:
        starts = np.asarray(vertex_offsets)[nonempty]
        low[nonempty] = np.minimum.reduceat(xyz, starts, axis=0)
        high[nonempty] = np.maximum.reduceat(xyz, starts, axis=0)
    return low, high, nonempty


class PackedMeshes:
    """Meshes ``[(vertices, faces), ...]`` held on the device as one block-diagonal system with
    both factors, for batches of single-source queries (``solve``)."""

    def __init__(self, meshes: list[tuple[Any, Any]], *, max_columns: int = 16) -> None:
        verts = [np.ascontiguousarray(v, dtype=np.float32).reshape(-1, 3) for v, _ in meshes]
        tris = [np.ascontiguousarray(f, dtype=np.int32).reshape(-1, 3) for _, f in meshes]
        self.n_meshes = len(meshes)
        if self.n_meshes == 0:
            raise ValueError("PackedMeshes: no meshes")
        counts = np.array([v.shape[0] for v in verts], dtype=np.int64)
        self.vertex_offsets = np.zeros(self.n_meshes + 1, dtype=np.int32)
        np.cumsum(counts, out=self.vertex_offsets[1:])
        n = int(self.vertex_offsets[-1])
        xyz = np.concatenate(verts)
        tri = np.concatenate([f + self.vertex_offsets[m] for m, f in enumerate(tris)])
        self.n = n
        self.n_faces = int(tri.shape[0])
        self.max_columns = int(max_columns)
        self.xyz = DeviceArray.from_host(xyz)
        self.faces = DeviceArray.from_host(tri.reshape(-1))
        self.d_vertex_offsets = DeviceArray.from_host(self.vertex_offsets)
        # a1-a3: pattern and face terms over the union.
        pattern = mesh_operator_pattern(self.faces, n)
        terms = face_terms(self.xyz, self.faces, n, self.n_faces)
        self.terms = terms
        # a4: each mesh's MeshLab time step h^2 (the mean of its faces' edges), floored by its
        # bounding box's diagonal / 400 (ordito/heat.py:3714-3748, 5228-5243).
        sums = DeviceArray.empty(2 * self.n_meshes, np.float64)
        _lib.call(
            "ob_edge_sums_segments", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
            pattern.keys.ptr, pattern.n_keys, self.xyz.ptr, 1, self.d_vertex_offsets.ptr,
            self.n_meshes, sums.ptr, DEFAULT_STREAM,
        )  # fmt: skip
        s = sums.numpy().reshape(self.n_meshes, 2)
        h = np.where(s[:, 1] > 0, s[:, 0] / np.where(s[:, 1] > 0, s[:, 1], 1.0), 0.0)
        t = h * h
        low, high, nonempty = mesh_bounds(xyz, self.vertex_offsets)
        for m in nonempty:
            floor = _bounds_floor_length(low[m], high[m]) ** 2
            if floor > t[m]:
                t[m] = floor
        self.time_steps = t
        row_factor = np.repeat(-t, counts)
        d_factor = DeviceArray.from_host(row_factor)
        capacity = max(pattern.n_keys, 1)
        values = DeviceArray.empty(3 * capacity, np.float64)
        L, H, P = (values.view(i * capacity, (i + 1) * capacity) for i in range(3))
        mass = DeviceArray.empty(n, np.float64)
        _lib.call(
            "ob_heat_rows_packed", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
            pattern.keys.ptr, pattern.n_keys, pattern.order.ptr, n, terms.cot.ptr, d_factor.ptr,
            terms.area_sums.ptr, 3.0, L.ptr, H.ptr, P.ptr, mass.ptr, DEFAULT_STREAM,
        )  # fmt: skip
        self._keep = (pattern, values, mass)
        laplacian = CsrMatrix(n, n, pattern.offsets, pattern.columns, L)
        self.heat_system = laplacian.with_values(H)
        self.poisson_system = laplacian.with_values(P)
        # a11: one analysis (the meshes translated apart for it) for both factors.
        extent = float((high - low).max()) if nonempty.size else 0.0
        spacing = 4.0 * max(extent, 1.0)
        shifted = xyz.copy()
        shifted[:, 0] += np.repeat((np.arange(self.n_meshes) * spacing).astype(np.float32), counts)
        self.analysis = CholeskyAnalysis(self.heat_system, DeviceArray.from_host(shifted))
        self.heat_factor = SparseCholesky(self.heat_system, self.analysis, singular=False)
        self.poisson_factor = SparseCholesky(self.poisson_system, self.analysis, singular=True)
        # The passes' tile schedule tuned to the union's tree at the batch width.
        from ordito_b200.tuning import tune_shared  # noqa: PLC0415

        # Both factors share the union's analysis: one search (three timed passes a candidate: a
        # packed pass takes milliseconds) serves both.
        self.tuning = tune_shared({"heat": self.heat_factor, "poisson": self.poisson_factor}, max_columns,
                                  reps=3)
        # a8: the divergence's corner index and per-face terms over the union.
        self.corner_offsets = DeviceArray.empty(n + 1, np.int32)
        self.corner_slots = DeviceArray.empty(max(3 * self.n_faces, 1), np.int32)
        size = ctypes.c_size_t(0)
        _lib.call("ob_corner_index_workspace", n, self.n_faces, ctypes.byref(size))
        workspace = DeviceArray.empty(int(size.value), np.uint8)
        _lib.call("ob_corner_index", self.faces.ptr, self.n_faces, n, self.corner_offsets.ptr,
                  self.corner_slots.ptr, workspace.ptr, int(size.value), DEFAULT_STREAM)
        from ordito_b200.heat import divergence_tiles  # noqa: PLC0415

        self.tile_faces, self.tile_counts, self.corner_codes = divergence_tiles(
            self.corner_offsets, self.corner_slots, n, self.n_faces)
        self.gradient_terms = DeviceArray.empty((max(self.n_faces, 1), 18), np.float64)
        _lib.call("ob_face_gradient_terms", self.xyz.ptr, self.faces.ptr, self.n_faces,
                  terms.normals.ptr, terms.areas.ptr, terms.cot.ptr, self.gradient_terms.ptr,
                  DEFAULT_STREAM)
        # Batch buffers at the widest batch: column sources, their offsets, the shift's table.
        K = self.max_columns
        self.d_sources = DeviceArray.empty(K * self.n_meshes, np.int32)
        self.d_offsets = DeviceArray.empty(K + 1, np.int32)
        self.d_shift = DeviceArray.empty(K * self.n_meshes, np.int32)
        self.d_sums = DeviceArray.empty(2 * K * self.n_meshes, np.float64)
        self.out = DeviceArray.empty((K, n), np.float64)
        self.heat_factor.work(K)
        self.poisson_factor.work(K)
        self._graphs: dict[int, tuple] = {}

    @property
    def nbytes(self) -> int:
        return self.heat_factor.nbytes + self.poisson_factor.nbytes

    def load(self, queries: list[list[int]]) -> int:
        """Write a batch: ``queries[m]`` are mesh m's single-source queries (local vertex indices,
        at most ``max_columns``); returns the batch width k (the most queries of any mesh)."""
        if len(queries) != self.n_meshes:
            raise ValueError(f"queries for {len(queries)} meshes, {self.n_meshes} held")
        k = max((len(q) for q in queries), default=0)
        if k == 0 or k > self.max_columns:
            raise ValueError(f"each mesh takes 1 to {self.max_columns} queries (got {k} at most)")
        columns: list[list[int]] = [[] for _ in range(k)]
        shift = np.full((self.n_meshes, k), -1, dtype=np.int32)
        for m, q in enumerate(queries):
            count = int(self.vertex_offsets[m + 1] - self.vertex_offsets[m])
            for c, s in enumerate(q):
                if not 0 <= int(s) < count:
                    raise ValueError(f"mesh {m}: source {s} out of range [0, {count})")
                columns[c].append(int(self.vertex_offsets[m]) + int(s))
                shift[m, c] = int(s)
        sizes = np.array([len(c) for c in columns], dtype=np.int32)
        offsets = np.zeros(k + 1, dtype=np.int32)
        np.cumsum(sizes, out=offsets[1:])
        sources = np.concatenate([np.array(c, dtype=np.int32) for c in columns])
        _lib.call("ob_memcpy", self.d_sources.ptr, sources.ctypes.data, sources.nbytes, 0, DEFAULT_STREAM, 0)
        _lib.call("ob_memcpy", self.d_offsets.ptr, offsets.ctypes.data, offsets.nbytes, 0, DEFAULT_STREAM, 0)
        _lib.call("ob_memcpy", self.d_shift.ptr, shift.ctypes.data, shift.nbytes, 0, DEFAULT_STREAM, 0)
        return k

    def run(self, k: int, stream: Any = DEFAULT_STREAM) -> DeviceArray:
        """The batched pass over the loaded batch (``load``) at width k: the ``(k, V)`` distances of
        the union (rows of mesh m: ``vertex_offsets[m]:vertex_offsets[m + 1]``; 0 where a mesh has
        no query in a column)."""
        n = self.n
        hf, pf = self.heat_factor, self.poisson_factor
        h_rhs, h_sol, h_stride, h_iperm, h_pinned = hf.work(k, stream)
        p_rhs, p_sol, p_stride, p_iperm, p_pinned = pf.work(k, stream)
        _lib.call("ob_seed_permuted", self.d_sources.ptr, self.d_offsets.ptr, k, n, h_iperm, h_pinned,
                  h_stride, h_rhs, stream)
        hf.solve_in_place_sources(k, self.d_sources, self.d_offsets, stream)
        from ordito_b200.heat import _grad_div_index  # noqa: PLC0415

        _grad_div_index(self.gradient_terms, self.faces,
                        (self.corner_offsets, self.corner_slots, self.tile_faces, self.tile_counts,
                         self.corner_codes), n, k, h_sol, h_stride, h_iperm, p_rhs, p_stride, p_iperm,
                        p_pinned, stream)
        pf.solve_in_place(k, stream)
        _lib.call("ob_shift_packed", p_sol, n, p_stride, p_iperm, self.d_vertex_offsets.ptr,
                  self.n_meshes, self.d_shift.ptr, k, self.d_sums.ptr, self.out.ptr, stream)
        return self.out

    def record(self, k: int, stream: ctypes.c_void_p) -> None:
        """Record the pass at width k on ``stream`` (a created stream) as one CUDA graph."""
        self.close_graph(k)
        _lib.call("ob_device_synchronize")
        self.run(k, stream)
        _lib.call("ob_stream_synchronize", stream)
        generations = (self.heat_factor.generation, self.poisson_factor.generation)
        with capture_guard():
            _lib.call("ob_capture_begin", stream)
            error: BaseException | None = None
            try:
                self.run(k, stream)
            except BaseException as exc:  # noqa: BLE001 -- the capture must be closed first
                error = exc
            handle, kernels = ctypes.c_void_p(0), ctypes.c_int(0)
            status = _lib.lib.ob_capture_end(stream, ctypes.byref(handle), ctypes.byref(kernels))
        if error is not None:
            raise error
        _lib.check(status, "ob_capture_end")
        self._graphs[k] = (handle, generations, int(kernels.value), stream)

    def replay(self, k: int, stream: Any = DEFAULT_STREAM) -> DeviceArray:
        """The recorded pass at width k (recorded again if a factor's buffers moved)."""
        graph = self._graphs.get(k)
        if graph is None or graph[1] != (self.heat_factor.generation, self.poisson_factor.generation):
            record_stream = graph[3] if graph is not None else None
            if record_stream is None:
                raise RuntimeError(f"PackedMeshes.replay: width {k} was not recorded")
            self.record(k, record_stream)
            graph = self._graphs[k]
        _lib.call("ob_graph_launch", graph[0], stream)
        return self.out

    def solve(self, queries: list[list[int]]) -> list[np.ndarray]:
        """Distances for every query: ``result[m]`` is mesh m's ``(len(queries[m]), V_m)``."""
        k = self.load(queries)
        out = self.run(k).numpy()[:k]
        return [out[: len(q), self.vertex_offsets[m]:self.vertex_offsets[m + 1]]
                for m, q in enumerate(queries)]

    def close_graph(self, k: int) -> None:
        graph = self._graphs.pop(k, None)
        if graph is not None:
            _lib.lib.ob_graph_destroy(graph[0])

    def close(self) -> None:
        for k in list(self._graphs):
            self.close_graph(k)
        self.heat_factor.close()
        self.poisson_factor.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


# -- the synthetic packed workload ------------------------------------------------------------

@dataclass
class PackedWorkload:
    specs: list[tuple]
    meshes: list[tuple[np.ndarray, np.ndarray]]
    queries: list[list[int]]


def packed_workload(seed: int, count: int = 256, *, max_queries: int = 16) -> PackedWorkload:
    """``count`` meshes drawn from ``seed``: each an icosphere at subdivision level 2-6
    (162-40 962 vertices) or a jittered torus with 16-256 columns x 8-128 rows, each with 1 to
    ``max_queries`` distinct uniform-random single-source queries."""
    from ordito_b200 import creation  # noqa: PLC0415

    rng = np.random.default_rng(seed)
    specs, meshes, queries = [], [], []
    cache: dict[tuple, tuple[np.ndarray, np.ndarray]] = {}
    for _ in range(count):
        if rng.random() < 0.5:
            spec = ("icosphere", int(rng.integers(2, 7)))
        else:
            spec = ("torus", int(rng.integers(16, 257)), int(rng.integers(8, 129)), int(rng.integers(1 << 30)))
        if spec not in cache:
            if spec[0] == "icosphere":
                v, f = creation.icosphere(spec[1])
            else:
                v, f = creation.jittered_torus(spec[1], spec[2], seed=spec[3])
            cache[spec] = (np.ascontiguousarray(v, np.float32), np.ascontiguousarray(f, np.int32))
        v, f = cache[spec]
        k = int(rng.integers(1, max_queries + 1))
        specs.append(spec)
        meshes.append((v, f))
        queries.append([int(s) for s in rng.choice(v.shape[0], size=min(k, v.shape[0]), replace=False)])
    return PackedWorkload(specs, meshes, queries)


def total_queries(queries: list[list[int]]) -> int:
    return int(sum(len(q) for q in queries))
