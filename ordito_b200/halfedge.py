"""Halfedge tables on the device (``ordito.halfedge``): twins and counter-clockwise one-rings.

Halfedge ``h = 3 f + k`` runs ``faces[3 f + k] -> faces[3 f + (k + 1) % 3]``. ``halfedge_twins``
pairs the two halfedges of every edge from the operator pattern's sorted key runs (each run lists
the corners opposite one vertex pair); ``vertex_one_rings`` walks ``twin(prev(h))`` from each
vertex's start halfedge (ordito/halfedge.py:59, :284). Both reject what the reference rejects:
an edge with three or more halfedges, an edge whose two halfedges run the same way, a pinched
vertex (``ValueError``).
"""

from __future__ import annotations

import ctypes
from typing import Any

import numpy as np

from ordito_b200 import _lib
from ordito_b200.device import DEFAULT_STREAM, DeviceArray, as_device
from ordito_b200.laplacian import MeshOperatorPattern, mesh_operator_pattern


def _faces(faces: Any) -> tuple[DeviceArray, int]:
    tri = as_device(faces, np.int32)
    if tri.size % 3:
        raise ValueError(f"faces must hold 3 * n_faces indices, got {tri.size}")
    return tri.reshape(tri.size), tri.size // 3


def _vertex_count(faces: DeviceArray, n_vertices: int | None) -> int:
    if n_vertices is not None:
        return int(n_vertices)
    # One read-back when the caller does not know the count (ordito/halfedge.py:405).
    host = faces.numpy()
    return int(host.max()) + 1 if host.size else 0


def corner_index(faces: DeviceArray, n_faces: int, n_vertices: int) -> tuple[DeviceArray, DeviceArray]:
    """``(corner_offsets[V + 1], corner_slots[3F])``: each vertex's corners (its outgoing
    halfedges) in ascending order (``ob_corner_index``)."""
    offsets = DeviceArray.empty(n_vertices + 1, np.int32)
    slots = DeviceArray.empty(max(3 * n_faces, 1), np.int32)
    size = ctypes.c_size_t(0)
    _lib.call("ob_corner_index_workspace", n_vertices, n_faces, ctypes.byref(size))
    workspace = DeviceArray.empty(int(size.value), np.uint8)
    _lib.call("ob_corner_index", faces.ptr, n_faces, n_vertices, offsets.ptr, slots.ptr, workspace.ptr,
              int(size.value), DEFAULT_STREAM)
    return offsets, slots


def twins_from_pattern(pattern: MeshOperatorPattern, faces: DeviceArray, n_faces: int,
                       *, validate: bool = True) -> DeviceArray:
    """The twin table of ``faces`` from its cotangent operator pattern (``ob_halfedge_twins``)."""
    twins = DeviceArray.empty(max(3 * n_faces, 1), np.int32)
    defects = DeviceArray.empty(2, np.int32)
    _lib.call("ob_halfedge_twins", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
              pattern.keys.ptr, pattern.n_keys, pattern.order.ptr, faces.ptr, n_faces, pattern.n_vertices,
              twins.ptr, defects.ptr, DEFAULT_STREAM)
    if validate:
        many, same_way = (int(x) for x in defects.numpy())
        if many:
            raise ValueError(f"halfedge_twins requires an edge-manifold mesh: {many} edge(s) carry three or more "
                             "halfedges")
        if same_way:
            raise ValueError(f"halfedge_twins requires consistently wound faces: {same_way} edge(s) have both "
                             "halfedges running the same way")
    return twins.view(0, 3 * n_faces) if n_faces else twins.view(0, 0)


def halfedge_twins(faces: Any, n_vertices: int | None = None, *, validate: bool = True) -> DeviceArray:
    """Opposite halfedge of every halfedge, ``-1`` on the boundary (ordito/halfedge.py:59).

    Raises ``ValueError`` (under ``validate``) for an edge carried by three or more halfedges or
    whose two halfedges run the same way (an inconsistently wound or non-orientable mesh)."""
    tri, n_faces = _faces(faces)
    n = _vertex_count(tri, n_vertices)
    if n_faces == 0:
        return DeviceArray.empty(0, np.int32)
    return twins_from_pattern(mesh_operator_pattern(tri, n), tri, n_faces, validate=validate)


def _check_twins(faces: DeviceArray, twins: DeviceArray) -> None:
    """``require_matching_twins`` (ordito/halfedge.py:175): every entry -1 or the opposite
    halfedge of the same edge, paired both ways."""
    f = faces.numpy().astype(np.int64)
    t = twins.numpy().astype(np.int64)
    if t.size != f.size:
        raise ValueError(f"twins must hold one entry per halfedge ({f.size}), got {t.size}")
    h = np.flatnonzero(t >= 0)
    tw = t[h]
    dest = lambda x: f[x - x % 3 + (x + 1) % 3]  # noqa: E731
    bad = (tw >= t.size)
    ok = ~bad
    bad[ok] |= (t[tw[ok]] != h[ok]) | (f[tw[ok]] != dest(h[ok])) | (f[h[ok]] != dest(tw[ok]))
    if bad.any():
        raise ValueError(f"twins is not a twin table for faces: {int(bad.sum())} mispaired entries")


def rings_from_twins(faces: DeviceArray, n_faces: int, n_vertices: int, twins: DeviceArray,
                     corners: tuple[DeviceArray, DeviceArray] | None = None, *, validate: bool = True
                     ) -> tuple[DeviceArray, DeviceArray, DeviceArray]:
    """``(ring_halfedges, offsets, is_boundary)`` over a twin table (``ob_vertex_one_rings``)."""
    if corners is None:
        corners = corner_index(faces, n_faces, n_vertices)
    offsets, slots = corners
    ring = DeviceArray.empty(max(3 * n_faces, 1), np.int32)
    boundary = DeviceArray.empty(max(n_vertices, 1), np.uint8)
    defects = DeviceArray.empty(1, np.int32)
    _lib.call("ob_vertex_one_rings", offsets.ptr, slots.ptr, twins.ptr, n_vertices, ring.ptr, boundary.ptr,
              defects.ptr, DEFAULT_STREAM)
    if validate:
        pinched = int(defects.numpy()[0])
        if pinched:
            raise ValueError(f"vertex_one_rings requires a vertex-manifold mesh: {pinched} vertex/vertices have "
                             "more than one fan of faces (a pinch point).")
    return ring.view(0, 3 * n_faces), offsets, boundary.view(0, n_vertices)


def vertex_one_rings(faces: Any, twins: Any = None, n_vertices: int | None = None, *, validate: bool = True,
                     return_twins: bool = False) -> tuple[DeviceArray, ...]:
    """Outgoing halfedges of every vertex counter-clockwise, as CSR ``(ring_halfedges, offsets,
    is_boundary)`` (ordito/halfedge.py:284): a rim vertex from its outgoing boundary halfedge, an
    interior one from its lowest-indexed outgoing halfedge; ``return_twins`` adds the twin table.
    ``is_boundary`` is uint8. Raises ``ValueError`` at a pinched vertex (under ``validate``) and
    for a supplied ``twins`` that is not a twin table of ``faces``."""
    tri, n_faces = _faces(faces)
    n = _vertex_count(tri, n_vertices)
    if twins is None:
        table = twins_from_pattern(mesh_operator_pattern(tri, n), tri, n_faces, validate=validate) \
            if n_faces else DeviceArray.empty(0, np.int32)
    else:
        table = as_device(twins, np.int32)
        _check_twins(tri, table)
    if n_faces == 0 or n == 0:
        rings = (DeviceArray.empty(0, np.int32), DeviceArray.zeros(n + 1, np.int32), DeviceArray.zeros(n, np.uint8))
    else:
        rings = rings_from_twins(tri, n_faces, n, table, validate=validate)
    return (*rings, table) if return_twins else rings
