"""``Trimesh``: the per-mesh state the heat path keeps resident (ordito/mesh.py:345).

A mesh holds its device vertices and faces and caches what depends on them alone: the operator
pattern, the per-face terms, the mean edge length and bounds, and one ``HeatSolver`` per
``(t, use_robust, method)`` with its operators, solver states and factorizations -- so distance
from many source sets on one mesh pays for them once (ordito/mesh.py:1878-2266).
"""

from __future__ import annotations

from typing import Any

import numpy as np

from ordito_b200 import _lib
from ordito_b200.device import DEFAULT_STREAM, DeviceArray
from ordito_b200.laplacian import FaceTerms, MeshOperatorPattern, face_terms, mesh_arrays, mesh_operator_pattern


class Trimesh:
    """A triangle mesh on the device: ``vertices`` float32 ``(V, 3)``, ``faces`` int32 ``(3F,)``."""

    def __init__(self, vertices: Any, faces: Any) -> None:
        xyz, tri, n_vertices, n_faces = mesh_arrays(vertices, faces)
        self.vertices = xyz.reshape(n_vertices, 3) if n_vertices else xyz
        self.faces = tri.reshape(3 * n_faces) if n_faces else tri
        self.n_vertices = n_vertices
        self.n_faces = n_faces
        self._pattern: MeshOperatorPattern | None = None
        self._face_terms: FaceTerms | None = None
        self._mean_edge_length: float | None = None
        self._bounds: tuple[np.ndarray, np.ndarray] | None = None
        self._solvers: dict[tuple, Any] = {}

    @property
    def mesh_operator_pattern(self) -> MeshOperatorPattern:
        if self._pattern is None:
            self._pattern = mesh_operator_pattern(self.faces, self.n_vertices)
        return self._pattern

    @property
    def face_terms(self) -> FaceTerms:
        if self._face_terms is None:
            self._face_terms = face_terms(self.vertices, self.faces, self.n_vertices, self.n_faces)
        return self._face_terms

    @property
    def cotmatrix_entries(self) -> DeviceArray:
        return self.face_terms.cot

    @property
    def corner_index(self) -> tuple[DeviceArray, DeviceArray]:
        """``(corner_offsets[V + 1], corner_slots[3 F])``: each vertex's corners in ascending slot
        order (a stable sort of the face buffer; ordito/heat.py:3198 ``_corner_order``)."""
        if getattr(self, "_corner_index", None) is None:
            import ctypes

            offsets = DeviceArray.empty(self.n_vertices + 1, np.int32)
            slots = DeviceArray.empty(max(3 * self.n_faces, 1), np.int32)
            size = ctypes.c_size_t(0)
            _lib.call("ob_corner_index_workspace", self.n_vertices, self.n_faces, ctypes.byref(size))
            workspace = DeviceArray.empty(int(size.value), np.uint8)
            _lib.call("ob_corner_index", self.faces.ptr, self.n_faces, self.n_vertices, offsets.ptr,
                      slots.ptr, workspace.ptr, int(size.value), DEFAULT_STREAM)
            self._corner_index = (offsets, slots)
        return self._corner_index

    @property
    def corner_tiles(self) -> tuple[DeviceArray, ...]:
        """The corner index and its divergence tiles, ``(corner_offsets, corner_slots, tile_faces,
        tile_counts, corner_codes)`` (``ob_divergence_tiles``), made once."""
        if getattr(self, "_corner_tiles", None) is None:
            from ordito_b200.heat import divergence_tiles  # noqa: PLC0415

            offsets, slots = self.corner_index
            self._corner_tiles = (offsets, slots) + divergence_tiles(offsets, slots, self.n_vertices,
                                                                     self.n_faces)
        return self._corner_tiles

    # -- the vector heat method's tables (ordito/mesh.py:2187 caches them the same way) ----------
    @property
    def halfedge_twins(self) -> DeviceArray:
        """Each halfedge's opposite, -1 on the boundary (``halfedge.halfedge_twins``), made once."""
        if getattr(self, "_twins", None) is None:
            from ordito_b200.halfedge import twins_from_pattern  # noqa: PLC0415

            self._twins = twins_from_pattern(self.mesh_operator_pattern, self.faces, self.n_faces)
        return self._twins

    @property
    def vertex_one_rings(self) -> tuple[DeviceArray, DeviceArray, DeviceArray]:
        """``(ring_halfedges, offsets, is_boundary)`` (``halfedge.vertex_one_rings``), made once."""
        if getattr(self, "_rings", None) is None:
            from ordito_b200.halfedge import rings_from_twins  # noqa: PLC0415

            self._rings = rings_from_twins(self.faces, self.n_faces, self.n_vertices, self.halfedge_twins,
                                           self.corner_index)
        return self._rings

    @property
    def halfedge_tangent_angles(self) -> DeviceArray:
        """Every halfedge's float64 polar angle in its origin's frame, made once."""
        if getattr(self, "_tangent_angles", None) is None:
            from ordito_b200.tangent_space import tangent_angles_of  # noqa: PLC0415

            self._tangent_angles = tangent_angles_of(self.vertices.reshape(3 * self.n_vertices), self.faces,
                                                     self.n_faces, self.n_vertices, self.vertex_one_rings)
        return self._tangent_angles

    @property
    def halfedge_transport(self) -> tuple[DeviceArray, DeviceArray]:
        """``(transport_angles (3F,), rotations (3F, 2))``: the connection, made once."""
        if getattr(self, "_transport", None) is None:
            from ordito_b200.tangent_space import transport_of  # noqa: PLC0415

            self._transport = transport_of(self.halfedge_twins, self.halfedge_tangent_angles, 3 * self.n_faces,
                                           angles=True, rotations=True)
        return self._transport

    @property
    def halfedge_transport_angles(self) -> DeviceArray:
        return self.halfedge_transport[0]

    @property
    def vertex_tangent_frames(self) -> tuple[DeviceArray, DeviceArray, DeviceArray]:
        """``(basis_x, basis_y, normal)`` float32 ``(V, 3)`` each, made once."""
        if getattr(self, "_frames", None) is None:
            from ordito_b200.tangent_space import frames_of  # noqa: PLC0415

            self._frames = frames_of(self.vertices.reshape(3 * self.n_vertices), self.faces, self.n_vertices,
                                     self.vertex_one_rings)
        return self._frames

    @property
    def vector_heat_operators(self) -> Any:
        """The default solver's ``vector_heat_operators`` (ordito/mesh.py's cached bundle)."""
        return self.heat_solver().vector_operators

    @property
    def mean_edge_length(self) -> float:
        """Mean over all ``3 n_faces`` per-face edges (ordito/mesh.py:1179), read back once."""
        if self._mean_edge_length is None:
            if self.n_faces == 0:
                self._mean_edge_length = 0.0
            else:
                pattern = self.mesh_operator_pattern
                sums = DeviceArray.empty(2, np.float64)
                _lib.call(
                    "ob_edge_sums", pattern.offsets.ptr, pattern.columns.ptr,
                    pattern.run_start.ptr, pattern.keys.ptr, pattern.n_keys, self.n_vertices,
                    self.vertices.ptr, 1, sums.ptr, DEFAULT_STREAM,
                )  # fmt: skip
                total, count = sums.numpy()
                self._mean_edge_length = float(total / count) if count > 0 else 0.0
        return self._mean_edge_length

    @property
    def bounds(self) -> tuple[np.ndarray, np.ndarray]:
        """Axis-aligned bounding box ``(min, max)`` (ordito/mesh.py:1045), read back once."""
        if self._bounds is None:
            out = DeviceArray.empty(6, np.float64)
            _lib.call("ob_bounds", self.vertices.ptr, self.n_vertices, out.ptr, DEFAULT_STREAM)
            host = out.numpy()
            self._bounds = (host[:3], host[3:])
        return self._bounds

    def heat_solver(self, t: float | None = None, *, use_robust: bool = False,
                    method: str = "potpourri3d"):
        """The mesh's ``HeatSolver`` for ``(t, use_robust, method)``, made on first use."""
        from ordito_b200.heat import HeatSolver  # noqa: PLC0415

        key = (None if t is None else float(t), bool(use_robust), method)
        solver = self._solvers.get(key)
        if solver is None:
            solver = self._solvers[key] = HeatSolver(self, t, use_robust=use_robust, method=method)
        return solver

    def dispose(self) -> None:
        """Release every device resource this mesh holds now (solvers, factors, operators); the
        mesh is unusable afterwards. ``heat_geodesic(vertices, faces, ...)`` disposes of the mesh
        it builds for the call."""
        for solver in self._solvers.values():
            solver.dispose()
        self._solvers.clear()
        self._pattern = None
        self._face_terms = None
        self._corner_index = None
        self._twins = self._rings = self._tangent_angles = self._transport = self._frames = None

    def release_factorizations(self) -> None:
        """Drop every solver's factorizations (ordito/mesh.py:3457)."""
        for solver in self._solvers.values():
            solver.release_factorizations()

    @property
    def nbytes(self) -> int:
        """Device bytes this mesh holds resident (buffers, pattern, operators, factors)."""
        total = self.vertices.nbytes + self.faces.nbytes
        if self._pattern is not None:
            p = self._pattern
            total += sum(a.nbytes for a in (p.offsets, p.columns, p.run_start, p.keys, p.order))
        if self._face_terms is not None:
            total += sum(a.nbytes for a in self._face_terms)
        total += sum(s.nbytes for s in self._solvers.values())
        return total


def mesh_arguments(caller: str, mesh: Any, vertices: Any, faces: Any, sources: Any
                   ) -> tuple[Trimesh, bool, Any]:
    """Resolve ``f(mesh, sources)`` and ``f(vertices, faces, sources)`` (ordito/mesh.py:3612).

    Returns the mesh, whether the caller holds it (passed a ``Trimesh``) and the sources. In the
    ``Trimesh`` form the second positional argument (bound to ``faces``) is the sources.
    """
    if isinstance(mesh, Trimesh):
        if vertices is not None:
            raise TypeError(f"{caller}: pass a Trimesh, or vertices and faces, not both")
        return mesh, True, faces if sources is None else sources
    verts = mesh if vertices is None else vertices
    if verts is None or faces is None:
        raise TypeError(f"{caller}: needs a Trimesh, or vertices and faces")
    return Trimesh(verts, faces), False, sources
