"""Per-vertex tangent spaces on the device (``ordito.tangent_space``).

Polar angles of every outgoing halfedge (a vertex's corner angles rescaled to a full turn, half a
turn on a rim, from geometry-central's reference halfedge), the vertex frames those angles are
measured in (``basis_x`` fitted to the whole fan, the angle-weighted normal), and the rotation
that carries a tangent vector across each halfedge (ordito/tangent_space.py:38, :254, :363). The
gauge is the reference's, so frames, angles and every tangent vector built on them agree with it
element for element.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from ordito_b200 import _lib
from ordito_b200.device import DEFAULT_STREAM, DeviceArray, as_device
from ordito_b200.halfedge import vertex_one_rings


def _mesh(vertices: Any, faces: Any) -> tuple[DeviceArray, DeviceArray, int, int]:
    xyz = as_device(vertices, np.float32)
    tri = as_device(faces, np.int32)
    if xyz.size % 3 or tri.size % 3:
        raise ValueError("vertices must be (n_vertices, 3) and faces 3 * n_faces indices")
    return xyz.reshape(xyz.size), tri.reshape(tri.size), xyz.size // 3, tri.size // 3


def _checked_rings(rings: tuple[Any, Any, Any], n_vertices: int, n_faces: int
                   ) -> tuple[DeviceArray, DeviceArray, DeviceArray]:
    """A caller's ``(ring_halfedges, offsets, is_boundary)`` on the device, its sizes and offsets
    checked (the kernels index with them; a slot of -1 is skipped there)."""
    ring, offsets, boundary = (as_device(r, dt) for r, dt in zip(rings, (np.int32, np.int32, np.uint8)))
    if ring.size != 3 * n_faces or offsets.size != n_vertices + 1 or boundary.size != n_vertices:
        raise ValueError(f"rings must be ((3 * n_faces,), (n_vertices + 1,), (n_vertices,)) arrays, got sizes "
                         f"({ring.size}, {offsets.size}, {boundary.size})")
    host = offsets.numpy()
    if host[0] != 0 or host[-1] != 3 * n_faces or np.any(np.diff(host) < 0):
        raise ValueError("rings: offsets must ascend from 0 to 3 * n_faces")
    return ring.reshape(ring.size), offsets.reshape(offsets.size), boundary.reshape(boundary.size)


def tangent_angles_of(xyz: DeviceArray, faces: DeviceArray, n_faces: int, n_vertices: int,
                      rings: tuple[DeviceArray, DeviceArray, DeviceArray], face_angles: Any = None) -> DeviceArray:
    """``ob_halfedge_tangent_angles`` over known rings."""
    ring, offsets, boundary = rings
    angles = DeviceArray.empty(max(3 * n_faces, 1), np.float64)
    scratch = DeviceArray.empty(max(3 * n_faces, 1), np.float64)
    table = None
    if face_angles is not None:
        table = as_device(face_angles, np.float32)
        if table.size != 3 * n_faces:
            raise ValueError(f"face_angles must be (n_faces, 3), got {table.size} values")
    _lib.call("ob_halfedge_tangent_angles", xyz.ptr, faces.ptr, n_faces, n_vertices, offsets.ptr, ring.ptr,
              boundary.ptr, table.ptr if table is not None else None, scratch.ptr, angles.ptr, DEFAULT_STREAM)
    return angles.view(0, 3 * n_faces)


def frames_of(xyz: DeviceArray, faces: DeviceArray, n_vertices: int,
              rings: tuple[DeviceArray, DeviceArray, DeviceArray],
              normals: Any = None) -> tuple[DeviceArray, DeviceArray, DeviceArray]:
    """``ob_vertex_tangent_frames`` over known rings."""
    ring, offsets, boundary = rings
    basis_x = DeviceArray.empty((n_vertices, 3), np.float32)
    basis_y = DeviceArray.empty((n_vertices, 3), np.float32)
    given = None
    if normals is not None:
        given = as_device(normals, np.float32)
        if given.size != 3 * n_vertices:
            raise ValueError(f"normals must be (n_vertices, 3), got {given.size} values")
        out_normals = given.reshape(n_vertices, 3)
    else:
        out_normals = DeviceArray.empty((n_vertices, 3), np.float32)
    _lib.call("ob_vertex_tangent_frames", xyz.ptr, faces.ptr, faces.size // 3, n_vertices, offsets.ptr, ring.ptr,
              boundary.ptr,
              given.ptr if given is not None else None, basis_x.ptr, basis_y.ptr,
              None if given is not None else out_normals.ptr, DEFAULT_STREAM)
    return basis_x, basis_y, out_normals


def transport_of(twins: DeviceArray, tangent_angles: DeviceArray, n_halfedges: int, *, angles: bool = True,
                 rotations: bool = False) -> tuple[DeviceArray | None, DeviceArray | None]:
    """``ob_halfedge_transport``: the transport angles and / or their rotations ``(cos, sin)``."""
    rho = DeviceArray.empty(max(n_halfedges, 1), np.float64) if angles else None
    rot = DeviceArray.empty((max(n_halfedges, 1), 2), np.float64) if rotations else None
    if n_halfedges:
        _lib.call("ob_halfedge_transport", twins.ptr, tangent_angles.ptr, n_halfedges,
                  rho.ptr if rho is not None else None, rot.ptr if rot is not None else None, DEFAULT_STREAM)
    return (rho.view(0, n_halfedges) if rho is not None else None,
            rot.view(0, 2 * n_halfedges, (n_halfedges, 2)) if rot is not None else None)


def vertex_tangent_frames(vertices: Any, faces: Any, normals: Any = None,
                          rings: tuple[Any, Any, Any] | None = None
                          ) -> tuple[DeviceArray, DeviceArray, DeviceArray]:
    """``(basis_x, basis_y, normal)``, float32 ``(V, 3)`` each (ordito/tangent_space.py:38).

    ``normal`` is the angle-weighted vertex normal (or the caller's ``normals``); ``basis_x`` is
    where ``halfedge_tangent_angles`` puts polar angle 0, fitted to the whole fan;
    ``basis_y = normal x basis_x``. A vertex with no faces gets ``((1, 0, 0), (0, 1, 0))``."""
    xyz, tri, n, n_faces = _mesh(vertices, faces)
    if n == 0:
        empty = DeviceArray.empty((0, 3), np.float32)
        return (empty, DeviceArray.empty((0, 3), np.float32),
                DeviceArray.empty((0, 3), np.float32) if normals is None else as_device(normals, np.float32))
    rings = vertex_one_rings(tri, n_vertices=n) if rings is None else _checked_rings(rings, n, n_faces)
    return frames_of(xyz, tri, n, rings, normals)


def halfedge_tangent_angles(vertices: Any, faces: Any, face_angles: Any = None,
                            rings: tuple[Any, Any, Any] | None = None) -> DeviceArray:
    """Polar angle of every outgoing halfedge in its origin's frame, float64 ``(3F,)``
    (ordito/tangent_space.py:254): the corner angles from the reference halfedge rescaled to a full
    turn (half a turn on a rim). ``face_angles``: a float32 ``(F, 3)`` corner-angle table to use
    instead of the float64 angles formed from the positions."""
    xyz, tri, n, n_faces = _mesh(vertices, faces)
    if n_faces == 0 or n == 0:
        return DeviceArray.zeros(3 * n_faces, np.float64)
    rings = vertex_one_rings(tri, n_vertices=n) if rings is None else _checked_rings(rings, n, n_faces)
    return tangent_angles_of(xyz, tri, n_faces, n, rings, face_angles)


def halfedge_transport_angles(vertices: Any, faces: Any, twins: Any = None,
                              tangent_angles: Any = None) -> DeviceArray:
    """Rotation carrying a tangent vector across each halfedge, in ``(-pi, pi]``
    (ordito/tangent_space.py:363): ``theta_twin + pi - theta_h`` wrapped, ``pi`` standing in for a
    boundary edge's missing twin. Raises ``ValueError`` for a ``twins`` that is not ``faces``'."""
    xyz, tri, n, n_faces = _mesh(vertices, faces)
    if n_faces == 0:
        return DeviceArray.empty(0, np.float64)
    ring, offsets, boundary, table = vertex_one_rings(tri, twins, n_vertices=n, return_twins=True)
    if tangent_angles is None:
        tangent = tangent_angles_of(xyz, tri, n_faces, n, (ring, offsets, boundary))
    else:
        tangent = as_device(tangent_angles, np.float64)
        if tangent.size != 3 * n_faces:
            raise ValueError(f"tangent_angles must hold one angle per halfedge ({3 * n_faces}), got {tangent.size}")
    return transport_of(table, tangent, 3 * n_faces)[0]


def tangent_to_world(tangent: Any, basis_x: Any, basis_y: Any) -> DeviceArray:
    """A tangent field ``(V, 2)`` in each vertex's frame as world vectors ``(V, 3)``:
    ``a * basis_x + b * basis_y`` (ordito/heat.py ``tangent_to_world``, kernels/heat.py:583)."""
    t = as_device(tangent, np.float32)
    bx = as_device(basis_x, np.float32)
    by = as_device(basis_y, np.float32)
    n = t.size // 2
    if bx.size != 3 * n or by.size != 3 * n:
        raise ValueError("tangent_to_world: tangent (V, 2) and frames (V, 3) must agree in V")
    out = DeviceArray.empty((n, 3), np.float32)
    _lib.call("ob_tangent_to_world", t.ptr, bx.ptr, by.ptr, n, out.ptr, DEFAULT_STREAM)
    return out
