"""The intrinsic tufted cover: ``heat_geodesic(method="potpourri3d", use_robust=True)``.

geometry-central's robust heat method (ordito/heat.py:5084 ``_tufted_intrinsic_delaunay``, :3749
``HeatSolver._cover_operators``): every face doubled into a front and a reversed back copy over the
same vertices and glued into a closed surface, the float64 lengths mollified and flipped to
intrinsic Delaunay, and the lumped mass, the cotangent Laplacian, the default time step and the
divergence all formed from the flipped lengths. The cover keeps every vertex, so its systems are
``n_vertices`` square as the extrinsic ones are (``ob_cover_build``, ``ob_cover_face_terms``,
``ob_heat_rows_f64``, ``ob_cover_divergence``).
"""

from __future__ import annotations

import ctypes
from typing import NamedTuple

import numpy as np

from ordito_b200 import _lib
from ordito_b200.device import DEFAULT_STREAM, DeviceArray
from ordito_b200.halfedge import corner_index
from ordito_b200.laplacian import Assembled, CsrMatrix, mesh_operator_pattern

TOLERANCE_MOLLIFY = 1e-5          # ordito/constants.py:31
DELAUNAY_EPSILON = 1e-6           # ordito/heat.py:194 (_GEOMETRY_CENTRAL_DELAUNAY_EPSILON)
FLIP_ROUNDS = 4096                # ordito/heat.py:197 (_COVER_FLIP_ROUNDS)


class TuftedCover(NamedTuple):
    """A mesh's intrinsic Delaunay tufted cover: ``faces`` ``(6 F,)`` (cover face ``f < F`` the
    front copy of face ``f``, ``F + f`` its back copy), ``lengths`` ``(2 F, 3)`` float64 (column
    ``e`` opposite corner ``e``), ``twin`` ``(6 F,)``, the float64 half-cotangents ``cot``
    ``(2 F, 3)``, each vertex's ascending cover corners and the flip rounds run."""

    faces: DeviceArray
    lengths: DeviceArray
    twin: DeviceArray
    cot: DeviceArray
    corner_offsets: DeviceArray
    corner_slots: DeviceArray
    n_vertices: int
    rounds: int

    @property
    def n_cover(self) -> int:
        return self.faces.size // 3


def build_cover(mesh) -> tuple[TuftedCover, DeviceArray, DeviceArray]:
    """The mesh's mollified tufted cover flipped to intrinsic Delaunay, its half-cotangents and
    corner index, with the per-vertex corner area sums and the cover's edge-length sums."""
    n, n_faces = mesh.n_vertices, mesh.n_faces
    pattern = mesh.mesh_operator_pattern
    n_cover = 2 * n_faces
    faces = DeviceArray.empty(max(3 * n_cover, 1), np.int32)
    lengths = DeviceArray.empty((max(n_cover, 1), 3), np.float64)
    twin = DeviceArray.empty(max(3 * n_cover, 1), np.int32)
    rounds = ctypes.c_int(0)
    _lib.call("ob_cover_build", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
              pattern.keys.ptr, pattern.n_keys, pattern.order.ptr, n, mesh.vertices.ptr, mesh.faces.ptr,
              n_faces, TOLERANCE_MOLLIFY, DELAUNAY_EPSILON, FLIP_ROUNDS, faces.ptr, lengths.ptr, twin.ptr,
              ctypes.byref(rounds), DEFAULT_STREAM)
    faces = faces.view(0, 3 * n_cover)
    offsets, slots = corner_index(faces, n_cover, n)
    cot = DeviceArray.empty((max(n_cover, 1), 3), np.float64)
    area_sums = DeviceArray.empty(max(n, 1), np.float64)
    edge_sums = DeviceArray.empty(2, np.float64)
    _lib.call("ob_cover_face_terms", faces.ptr, lengths.ptr, n_cover, n, offsets.ptr, slots.ptr, cot.ptr,
              area_sums.ptr, edge_sums.ptr, DEFAULT_STREAM)
    cover = TuftedCover(faces, lengths, twin, cot, offsets, slots, n, int(rounds.value))
    return cover, area_sums, edge_sums


def cover_rows(mesh, cover: TuftedCover, area_sums: DeviceArray, edge_sums: DeviceArray,
               t: float | None) -> Assembled:
    """``L``, ``M - t L`` and ``-L`` over the cover's own cotmatrix pattern from its float64
    half-cotangents, the lumped mass a third of each vertex's corner areas; with ``t`` None the
    time is the squared mean cover edge (ordito/heat.py:3786-3813)."""
    n = mesh.n_vertices
    pattern = mesh_operator_pattern(cover.faces, n)
    capacity = max(pattern.n_keys, 1)
    values = DeviceArray.empty(3 * capacity, np.float64)
    L = values.view(0, capacity)
    H = values.view(capacity, 2 * capacity)
    P = values.view(2 * capacity, 3 * capacity)
    mass = DeviceArray.empty(n, np.float64)
    _lib.call(
        "ob_heat_rows_f64", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
        pattern.keys.ptr, pattern.n_keys, pattern.order.ptr, n, cover.cot.ptr,
        -1.0 if t is None else -float(t), edge_sums.ptr, 1 if t is None else 0, area_sums.ptr, 3.0,
        L.ptr, H.ptr, P.ptr, mass.ptr, DEFAULT_STREAM,
    )  # fmt: skip
    laplacian = CsrMatrix(n, n, pattern.offsets, pattern.columns, L)
    return Assembled(laplacian, laplacian.with_values(H), laplacian.with_values(P), mass,
                     edge_sums if t is None else None)


def cover_divergence(cover: TuftedCover, u: DeviceArray, out: DeviceArray, n_columns: int = 1) -> None:
    """``div`` of the unit gradient of ``u`` on the cover, per vertex (``[V][n_columns]``)."""
    _lib.call("ob_cover_divergence", cover.faces.ptr, cover.lengths.ptr, cover.cot.ptr, cover.n_vertices,
              cover.corner_offsets.ptr, cover.corner_slots.ptr, u.ptr, int(n_columns), out.ptr, DEFAULT_STREAM)
