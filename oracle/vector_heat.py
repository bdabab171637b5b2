"""CPU restatement of ordito's vector heat method (TEST INFRASTRUCTURE: the checker only).

The halfedge tables, the tangent spaces (polar angles, vertex frames, transport angles), the
vector heat system ``M + t L_connection`` and the two solvers built on it,
``transport_tangent_vectors`` and ``log_map`` (both its ``"heat_geodesic"`` and its
``"potpourri3d"`` construction). Each function cites the reference file:line it follows (paths
within the ordito project). Per-vertex float32 arithmetic is done in ``np.float32`` in the
reference's operation order; the linear systems are solved directly in float64 (scipy SuperLU),
the exact solutions the reference's settled iterations approach.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

from oracle import heat_path as hp

F32 = np.float32
F64 = np.float64

TOLERANCE_MERGE = F32(1e-8)  # ordito/constants.py:13,40 (float32 constant)
TOLERANCE_ZERO = F32(1e-12)  # ordito/constants.py:15,42
RESOLVED_FRACTION = 1e-4  # ordito/heat.py:1726


# --------------------------------------------------------------------------------------------
# Halfedges: ordito/halfedge.py:59 (halfedge_twins), :284-452 (vertex_one_rings),
# kernels/halfedge.py:41-114 (next, prev, destination), :656-752 (ring start, walk).
# Halfedge 3 f + k runs faces[f, k] -> faces[f, (k + 1) % 3].
# --------------------------------------------------------------------------------------------


def prev_halfedge(h: np.ndarray | int) -> np.ndarray | int:
    return h - h % 3 + (h + 2) % 3


def destination(faces: np.ndarray, h: np.ndarray | int) -> np.ndarray | int:
    flat = np.asarray(faces).reshape(-1)
    return flat[h - h % 3 + (h + 1) % 3]


def halfedge_twins(faces: np.ndarray) -> np.ndarray:
    """Opposite halfedge of every halfedge, -1 on the boundary; ValueError on an edge with three
    or more halfedges or two running the same way (halfedge.py:59-172)."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1)
    nh = f.size
    origin = f
    target = destination(f, np.arange(nh))
    lo, hi = np.minimum(origin, target), np.maximum(origin, target)
    key = lo * (int(f.max()) + 1 if nh else 1) + hi
    order = np.argsort(key, kind="stable")
    twins = np.full(nh, -1, dtype=np.int64)
    sk = key[order]
    start = 0
    while start < nh:
        end = start + 1
        while end < nh and sk[end] == sk[start]:
            end += 1
        run = order[start:end]
        if run.size > 2:
            raise ValueError("halfedge_twins: an edge carries three or more halfedges")
        if run.size == 2:
            a, b = int(run[0]), int(run[1])
            if origin[a] == origin[b]:
                raise ValueError("halfedge_twins: two halfedges of an edge run the same way")
            twins[a], twins[b] = b, a
        start = end
    return twins


def vertex_one_rings(faces: np.ndarray, n_vertices: int,
                     twins: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """``(ring_halfedges, offsets, is_boundary)``: every vertex's outgoing halfedges counter-
    clockwise, from its outgoing boundary halfedge on a rim, else from its lowest-indexed one
    (halfedge.py:284-452, kernels/halfedge.py:656-752). ValueError at a pinched vertex."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1)
    if twins is None:
        twins = halfedge_twins(f)
    nh = f.size
    degree = np.bincount(f, minlength=n_vertices)[:n_vertices]
    offsets = np.zeros(n_vertices + 1, dtype=np.int64)
    np.cumsum(degree, out=offsets[1:])
    ring = np.full(nh, -1, dtype=np.int64)
    is_boundary = np.zeros(n_vertices, dtype=bool)
    interior_start = np.full(n_vertices, nh, dtype=np.int64)
    boundary_start = np.full(n_vertices, nh, dtype=np.int64)
    for h in range(nh):
        v = f[h]
        interior_start[v] = min(interior_start[v], h)
        if twins[h] < 0:
            boundary_start[v] = min(boundary_start[v], h)
    pinched = 0
    for v in range(n_vertices):
        if degree[v] == 0:
            continue
        is_boundary[v] = boundary_start[v] < nh
        start = boundary_start[v] if is_boundary[v] else interior_start[v]
        count, h = 0, start
        while h >= 0 and count < degree[v]:
            ring[offsets[v] + count] = h
            count += 1
            nxt = twins[prev_halfedge(h)]
            if nxt < 0 or nxt == start:
                break
            h = nxt
        if count != degree[v]:
            pinched += 1
    if pinched:
        raise ValueError(f"vertex_one_rings requires a vertex-manifold mesh: {pinched} pinched vertices")
    return ring, offsets, is_boundary


# --------------------------------------------------------------------------------------------
# Corner angles: kernels/triangles.py:427-493 (corner_angles_of_edges, face_corner_angles(_d),
# halfedge_corner_angle), kernels/predicates.py:458-472 (vector_angle = atan2(|a x b|, a . b)).
# --------------------------------------------------------------------------------------------


def _angle(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.arctan2(hp._length(hp._cross(a, b)), hp._dot(a, b))


def corner_angles(vertices: np.ndarray, faces: np.ndarray, dtype=F64) -> np.ndarray:
    """``(F, 3)`` interior angles from the corners in ``dtype`` (float64: ``face_corner_angles_d``,
    float32: ``face_corner_angles``); all three zero when any is below ``TOLERANCE_MERGE``."""
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3).astype(dtype)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    v0, v1, v2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    e01, e02, e12 = v1 - v0, v2 - v0, v2 - v1
    with np.errstate(all="ignore"):
        a0 = _angle(e01, e02).astype(dtype)
        a1 = _angle(-e01, e12).astype(dtype)
        a2 = (dtype(math.pi) - a0 - a1).astype(dtype)
    tol = dtype(TOLERANCE_MERGE)
    bad = (a0 < tol) | (a1 < tol) | (a2 < tol)
    out = np.stack((a0, a1, a2), axis=1)
    out[bad] = 0
    return out


def _reference_slot(ring: np.ndarray, boundary: bool) -> int:
    """kernels/tangent_space.py:48-61: slot 0 on a rim, else the slot of the largest halfedge."""
    return 0 if boundary else int(np.argmax(ring))


def _ring_scale(total, boundary: bool, dtype):
    """kernels/tangent_space.py:32-45 (ring_tangent_scale)."""
    if total > dtype(TOLERANCE_ZERO):
        return (dtype(math.pi) if boundary else dtype(2.0 * math.pi)) / total
    return dtype(0.0)


def halfedge_tangent_angles(vertices: np.ndarray, faces: np.ndarray,
                            rings: tuple[np.ndarray, np.ndarray, np.ndarray]) -> np.ndarray:
    """Every halfedge's polar angle in its origin's frame, float64 (tangent_space.py:254-360,
    kernels/tangent_space.py:102-133, 298-330: the one-lane ring walk)."""
    ring, offsets, is_boundary = rings
    angles = corner_angles(vertices, faces, F64).reshape(-1)
    out = np.zeros(angles.size, dtype=F64)
    for v in range(offsets.size - 1):
        r = ring[offsets[v]:offsets[v + 1]]
        if r.size == 0:
            continue
        total = F64(0.0)
        for h in r:
            total += angles[h]
        scale = _ring_scale(total, bool(is_boundary[v]), F64)
        start = _reference_slot(r, bool(is_boundary[v]))
        acc = F64(0.0)
        for t in range(r.size):
            h = r[(start + t) % r.size]
            out[h] = scale * acc
            acc += angles[h]
    return out


def halfedge_transport_angles(twins: np.ndarray, tangent_angles: np.ndarray) -> np.ndarray:
    """``wrap(theta_twin + pi - theta_h)``, ``pi`` standing in for a boundary edge's missing twin
    (tangent_space.py:363-466, kernels/tangent_space.py:700-730)."""
    opposite = np.where(twins >= 0, tangent_angles[np.maximum(twins, 0)], math.pi)
    a = opposite + math.pi - tangent_angles
    return np.arctan2(np.sin(a), np.cos(a))


# --------------------------------------------------------------------------------------------
# Vertex frames: tangent_space.py:38-163, kernels/tangent_space.py:335-480 (fan_anchor,
# anchored_basis_x, vertex_tangent_basis), kernels/normals.py:52-169 (angle-weighted normal),
# kernels/predicates.py:163-182, 627-682 (any_perpendicular, unit_tangent, world_to_tangent).
# --------------------------------------------------------------------------------------------


def _v3(x) -> np.ndarray:
    return np.asarray(x, dtype=F32).reshape(3)


def _dot3(a: np.ndarray, b: np.ndarray):
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]


def _cross3(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]],
                    dtype=a.dtype)


def _len3(a: np.ndarray):
    return np.sqrt(_dot3(a, a))


def _normalize3(a: np.ndarray) -> np.ndarray:
    length = _len3(a)
    if length > 0:
        return (a / length).astype(a.dtype)
    return np.zeros(3, dtype=a.dtype)


def any_perpendicular(normal: np.ndarray) -> np.ndarray:
    axis = np.array([1.0, 0.0, 0.0], dtype=normal.dtype)
    if abs(normal[0]) > abs(normal[1]):
        axis = np.array([0.0, 1.0, 0.0], dtype=normal.dtype)
    return _normalize3(_cross3(normal, axis))


def vertex_tangent_frames(vertices: np.ndarray, faces: np.ndarray,
                          rings: tuple[np.ndarray, np.ndarray, np.ndarray]
                          ) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """``(basis_x, basis_y, normal)`` float32 per vertex: the angle-weighted normal gathered over
    the ring, ``basis_x`` the fan-fitted polar angle 0 in geometry-central's gauge."""
    ring, offsets, is_boundary = rings
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    flat = f.reshape(-1)
    n = v.shape[0]
    normals_f, _ = hp.face_normals_and_areas(v, f)
    angles32 = corner_angles(v, f, F32).reshape(-1)
    bx_out = np.zeros((n, 3), dtype=F32)
    by_out = np.zeros((n, 3), dtype=F32)
    nrm_out = np.zeros((n, 3), dtype=F32)
    for vert in range(n):
        r = ring[offsets[vert]:offsets[vert + 1]]
        boundary = bool(is_boundary[vert])
        total = np.zeros(3, dtype=F64)
        angle_total = F32(0.0)
        for h in r:
            angle = angles32[h]
            total += (normals_f[h // 3] * angle).astype(F32).astype(F64)
            angle_total = F32(angle_total + angle)
        length = math.sqrt(total[0] * total[0] + total[1] * total[1] + total[2] * total[2])
        if length > 0:
            total = total / length
        normal = total.astype(F32)
        nrm_out[vert] = normal
        if _len3(normal) <= TOLERANCE_ZERO:
            bx_out[vert] = (1.0, 0.0, 0.0)
            by_out[vert] = (0.0, 1.0, 0.0)
            continue
        if r.size == 0:
            bx = any_perpendicular(normal)
            bx_out[vert], by_out[vert] = bx, _cross3(normal, bx)
            continue
        start = _reference_slot(r, boundary)
        origin = v[vert]
        direction = (v[destination(flat, r[start])] - origin).astype(F32)
        tangential = (direction - _dot3(direction, normal) * normal).astype(F32)
        ref_length = _len3(tangential)
        bx = any_perpendicular(normal)
        if ref_length > TOLERANCE_ZERO:
            bx = (tangential / ref_length).astype(F32)
        scale = _ring_scale(angle_total, boundary, F32)
        if scale > F32(0.0):
            fy = _cross3(normal, bx)
            ax = F32(0.0)
            ay = F32(0.0)
            acc = F32(0.0)
            for t in range(r.size):
                h = r[(start + t) % r.size]
                edge = (v[destination(flat, h)] - origin).astype(F32)
                e0, e1 = _dot3(edge, bx), _dot3(edge, fy)
                theta = F32(scale * acc)
                c, s = np.cos(theta, dtype=F32), np.sin(theta, dtype=F32)
                ax = F32(ax + F32(e0 * c + e1 * s))
                ay = F32(ay + F32(e1 * c - e0 * s))
                acc = F32(acc + angles32[h])
            if boundary:
                rim = (v[flat[prev_halfedge(r[-1])]] - origin).astype(F32)
                ax = F32(ax - _dot3(rim, bx))
                ay = F32(ay - _dot3(rim, fy))
            if F32(np.sqrt(F32(F32(ax * ax) + F32(ay * ay)))) > F32(TOLERANCE_ZERO * ref_length):
                bx = _normalize3((ax * bx + ay * fy).astype(F32))
        bx_out[vert] = bx
        by_out[vert] = _cross3(normal, bx)
    return bx_out, by_out, nrm_out


# --------------------------------------------------------------------------------------------
# The vector heat system: heat.py:1740-1955 (vector_heat_operators), kernels/heat.py:243-296
# (vector_heat_row / _diagonal), kernels/laplacian.py:1430-1465 (connection_offdiagonal),
# kernels/linalg.py:1625-1633 (shifted_block_entry), kernels/laplacian.py:130-136 (float64 cot).
# --------------------------------------------------------------------------------------------


def cotmatrix_entries_float64(vertices: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """``(F, 3)`` half-cotangents from the float32 corners widened to float64."""
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3).astype(F64)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    v0, v1, v2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    with np.errstate(all="ignore"):
        den = 2.0 * hp._length(hp.triangle_area_vector(v0, v1, v2))
        ok = den > 0
        safe = np.where(ok, den, 1.0)
        out = np.stack((hp._dot(v1 - v0, v2 - v0) / safe, hp._dot(v2 - v1, v0 - v1) / safe,
                        hp._dot(v0 - v2, v1 - v2) / safe), axis=1)
    out[~ok] = 0.0
    return out


def vector_heat_system(vertices: np.ndarray, faces: np.ndarray, ops: dict, transport: np.ndarray,
                       t: float) -> sp.csr_matrix:
    """``M + t L_connection`` as the real ``2n x 2n`` matrix, vertex v's tangent components in rows
    ``2v`` and ``2v + 1``: each off-diagonal block ``-t sum w R(+-rho)`` over the edge's faces in
    face order, each diagonal block ``(t sum w + m) I``."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1)
    pattern = ops["pattern"]
    offsets = pattern["offsets"]
    n = offsets.size - 1
    columns = pattern["columns"].astype(np.int64)
    rs = pattern["run_start"].astype(np.int64)
    ends = hp.run_ends(pattern["keys"], rs)
    order = pattern["order"].astype(np.int64)
    cot64 = cotmatrix_entries_float64(vertices, faces).reshape(-1)
    cos_r, sin_r = np.cos(transport), np.sin(transport)
    mass = ops["mass"]
    rows, cols, vals = [], [], []
    for i in range(n):
        weight = 0.0
        for k in range(offsets[i], offsets[i + 1]):
            j = int(columns[k])
            if j == i:
                continue
            block = np.zeros((2, 2))
            for p in range(rs[k], ends[k]):
                q = order[p]
                h = (q // 3) * 3 + (q % 3 + 1) % 3
                w = cot64[q]
                c = cos_r[h]
                s = -sin_r[h] if f[h] == i else sin_r[h]
                block += -w * np.array([[c, -s], [s, c]])
                weight += w
            block *= t
            for a in range(2):
                for b in range(2):
                    rows.append(2 * i + a)
                    cols.append(2 * j + b)
                    vals.append(block[a, b])
        if offsets[i + 1] > offsets[i]:
            d = t * weight + mass[i]
            rows += [2 * i, 2 * i + 1]
            cols += [2 * i, 2 * i + 1]
            vals += [d, d]
    return sp.csr_matrix((vals, (rows, cols)), shape=(2 * n, 2 * n))


class VectorHeat:
    """Everything the two vector solvers read for one mesh, at the potpourri3d discretization and
    the time step ``t`` (None: the squared unique-edge mean, lengthened on a fine mesh)."""

    def __init__(self, vertices: np.ndarray, faces: np.ndarray, t: float | None = None) -> None:
        self.vertices = np.asarray(vertices, dtype=F32).reshape(-1, 3)
        self.faces = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
        n = self.vertices.shape[0]
        self.n = n
        t_eff, _ = hp.vertex_time(self.vertices, self.faces, t, "potpourri3d")
        self.ops = hp.heat_operators(self.vertices, self.faces, t_eff, method="potpourri3d")
        self.t = float(self.ops["t"])
        self.twins = halfedge_twins(self.faces)
        self.rings = vertex_one_rings(self.faces, n, self.twins)
        self.tangent = halfedge_tangent_angles(self.vertices, self.faces, self.rings)
        self.transport = halfedge_transport_angles(self.twins, self.tangent)
        self.frames = vertex_tangent_frames(self.vertices, self.faces, self.rings)
        self.system = vector_heat_system(self.vertices, self.faces, self.ops, self.transport, self.t)
        self.heat = hp.csr_matrix(self.ops["pattern"], self.ops["H"])

    def diffuse_tangent(self, rhs: np.ndarray) -> np.ndarray:
        return hp.solve_heat(self.system, rhs)

    def diffuse(self, rhs: np.ndarray) -> np.ndarray:
        return hp.solve_heat(self.heat, rhs)


def _stable_normalize(v: np.ndarray) -> np.ndarray:
    """kernels/predicates.py:719-724, row-wise."""
    largest = np.abs(v).max(axis=-1, keepdims=True)
    with np.errstate(all="ignore"):
        w = v / np.where(largest > 0, largest, 1.0)
        length = np.sqrt((w * w).sum(axis=-1, keepdims=True))
        out = np.where(length > 0, w / np.where(length > 0, length, 1.0), 0.0)
    return np.where(largest > 0, out, 0.0)


def _stable_length(v: np.ndarray) -> np.ndarray:
    largest = np.abs(v).max(axis=-1)
    with np.errstate(all="ignore"):
        w = v / np.where(largest > 0, largest, 1.0)[..., None]
        return np.where(largest > 0, largest * np.sqrt((w * w).sum(axis=-1)), 0.0)


def transport_tangent_vectors(state: VectorHeat, sources: np.ndarray,
                              vectors: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """``(transported float32 (n, 2), resolved bool (n,))`` (heat.py:2526-2729,
    kernels/heat.py:3881-3901 seed, :3975-3996 transported_and_resolved)."""
    n = state.n
    src = np.asarray(sources, dtype=np.int64).reshape(-1)
    vec = np.asarray(vectors, dtype=F32).reshape(-1, 2).astype(F64)
    if src.size == 0:
        return np.zeros((n, 2), dtype=F32), np.zeros(n, dtype=bool)
    if np.any((src < 0) | (src >= n)):
        raise ValueError("transport_tangent_vectors: sources must be vertex indices in [0, n_vertices)")
    field_rhs = np.zeros(2 * n)
    scalar_rhs = np.zeros((n, 2))
    for s, v in zip(src, vec):
        field_rhs[2 * s] += v[0]
        field_rhs[2 * s + 1] += v[1]
        scalar_rhs[s, 0] += 1.0
        scalar_rhs[s, 1] += math.sqrt(v[0] * v[0] + v[1] * v[1])
    field = state.diffuse_tangent(field_rhs).reshape(n, 2)
    scalars = state.diffuse(scalar_rhs)
    indicator, magnitude = scalars[:, 0], scalars[:, 1]
    with np.errstate(all="ignore"):
        extended = np.where(indicator != 0.0, magnitude / np.where(indicator != 0, indicator, 1.0), 0.0)
    transported = (extended[:, None] * _stable_normalize(field)).astype(F32)
    resolved = _stable_length(field) > RESOLVED_FRACTION * magnitude
    return transported, resolved


def tangent_to_world(tangent: np.ndarray, basis_x: np.ndarray, basis_y: np.ndarray) -> np.ndarray:
    """kernels/heat.py:583-596."""
    return (tangent[:, :1] * basis_x + tangent[:, 1:2] * basis_y).astype(F32)


def _distance(state: VectorHeat, source: int, heat: np.ndarray) -> np.ndarray:
    """``heat_geodesic``'s tail at the potpourri3d discretization (heat.py:3052-3131)."""
    ops = state.ops
    neg_div = hp.unit_gradient_divergence(state.vertices, state.faces, ops["normals"], ops["areas"],
                                          heat, ops["cot"])
    phi = hp.solve_regularized_poisson(ops["pattern"], ops["P"], neg_div)
    return hp.shift_to_sources(phi, np.array([source]))


def _vertex_gradient(state: VectorHeat, distance: np.ndarray) -> np.ndarray:
    """Area-weighted face unit gradients summed onto vertices in float32, corners in ascending
    order (kernels/heat.py:3999-4027, kernels/triangles.py:835-894)."""
    v = state.vertices.astype(F64)
    f = state.faces
    ops = state.ops
    nrm = ops["normals"].astype(F64)
    area = ops["areas"].astype(F64)
    v0, v1, v2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    with np.errstate(all="ignore"):
        g = (distance[f[:, 0], None] * hp._cross(nrm, v2 - v1)
             + distance[f[:, 1], None] * hp._cross(nrm, v0 - v2)
             + distance[f[:, 2], None] * hp._cross(nrm, v1 - v0)) / (2.0 * np.where(area > 0, area, 1.0))[:, None]
    g = np.where((area > 0)[:, None], g, 0.0)
    x = _stable_normalize(g).astype(F32) * ops["areas"][:, None]
    out = np.zeros((state.n, 3), dtype=F32)
    np.add.at(out, f.reshape(-1), np.repeat(x.astype(F32), 3, axis=0))
    return out


def _stable_normalize32(v: np.ndarray) -> np.ndarray:
    largest = np.abs(v).max(axis=-1, keepdims=True)
    with np.errstate(all="ignore"):
        w = (v / np.where(largest > 0, largest, F32(1.0))).astype(F32)
        length = np.sqrt((w[:, :1] * w[:, :1] + w[:, 1:2] * w[:, 1:2])).astype(F32)
        out = np.where(length > 0, w / np.where(length > 0, length, F32(1.0)), F32(0.0))
    return np.where(largest > 0, out, F32(0.0)).astype(F32)


def log_map(state: VectorHeat, source: int, method: str = "heat_geodesic") -> np.ndarray:
    """``(n, 2)`` float32 log-map coordinates in the source's frame (heat.py:2745-3027)."""
    if method == "potpourri3d":
        return _log_map_vector_heat(state, source)
    n = state.n
    field_rhs = np.zeros(2 * n)
    field_rhs[2 * source] = 1.0
    heat_rhs = np.zeros(n)
    heat_rhs[source] = 1.0
    transported_raw = state.diffuse_tangent(field_rhs).reshape(n, 2)
    heat = state.diffuse(heat_rhs)
    distance = _distance(state, source, heat)
    gradient = _vertex_gradient(state, distance)
    bx, by, _ = state.frames
    reference = _stable_normalize(transported_raw).astype(F32)
    projected = np.stack((hp._dot(gradient, bx), hp._dot(gradient, by)), axis=1).astype(F32)
    outward = _stable_normalize32(projected)
    r = distance.astype(F32)
    ref_len = np.sqrt(reference[:, 0] ** 2 + reference[:, 1] ** 2)
    out_len = np.sqrt(outward[:, 0] ** 2 + outward[:, 1] ** 2)
    cross = reference[:, 0] * outward[:, 1] - reference[:, 1] * outward[:, 0]
    dot = reference[:, 0] * outward[:, 0] + reference[:, 1] * outward[:, 1]
    angle = np.arctan2(cross, dot).astype(F32)
    none = (ref_len <= TOLERANCE_ZERO) | (out_len <= TOLERANCE_ZERO)
    angle = np.where(none, F32(0.0), angle)
    return np.stack((r * np.cos(angle), r * np.sin(angle)), axis=1).astype(F32)


def _complex(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.stack((a[..., 0] * b[..., 0] - a[..., 1] * b[..., 1],
                     a[..., 0] * b[..., 1] + a[..., 1] * b[..., 0]), axis=-1)


def _polar(angle) -> np.ndarray:
    return np.stack((np.cos(angle), np.sin(angle)), axis=-1)


def outward_ball(state: VectorHeat, source: int) -> tuple[np.ndarray, np.ndarray]:
    """The potpourri3d log map's right-hand sides: the outward ball and the reference direction
    (kernels/heat.py:4088-4152, appendix A of the vector heat method)."""
    n = state.n
    v = state.vertices.astype(F64)
    flat = state.faces.reshape(-1)
    ring, offsets, _ = state.rings
    radial = np.zeros((n, 2))
    horizontal = np.zeros((n, 2))
    horizontal[source] = (1.0, 0.0)
    pa = v[source]
    for j in range(offsets[source], offsets[source + 1]):
        ab = int(ring[j])
        f, k = ab // 3, ab % 3
        bc = 3 * f + (k + 1) % 3
        ca = 3 * f + (k + 2) % 3
        b, c = int(flat[bc]), int(flat[ca])
        pb, pc = v[b], v[c]
        twice_area = float(np.linalg.norm(np.cross(pb - pa, pc - pa)))
        if twice_area == 0.0:
            continue
        theta = math.atan2(np.linalg.norm(np.cross(pb - pa, pc - pa)), np.dot(pb - pa, pc - pa))
        gamma = math.atan2(np.linalg.norm(np.cross(pa - pb, pc - pb)), np.dot(pa - pb, pc - pb))
        sine = math.sin(theta)
        swing = theta * math.cos(theta) - sine
        height_b = twice_area / float(np.linalg.norm(pc - pa))
        toward_b = np.array([-theta * sine, swing]) / (2.0 * height_b)
        reversed_angle = state.tangent[ab] + state.transport[ab] - math.pi
        radial[b] += _complex(toward_b, _polar(reversed_angle))
        height_c = twice_area / float(np.linalg.norm(pb - pa))
        toward_c = np.array([-theta * sine, -swing]) / (2.0 * height_c)
        radial[c] += _complex(toward_c, _polar(state.tangent[ca]))
        height_a = twice_area / float(np.linalg.norm(pc - pb))
        alpha = 0.5 * math.pi - gamma
        at_source = np.array([
            -(theta * math.cos(alpha) + math.cos(alpha - theta) * sine) / (2.0 * height_a),
            -(math.cos(alpha) - math.cos(alpha - 2.0 * theta) + 2.0 * theta * math.sin(alpha)) / (4.0 * height_a),
        ])
        radial[source] += _complex(at_source, _polar(state.tangent[ab]))
    return radial, horizontal


def _unit_radial(radial_raw: np.ndarray, source: int) -> np.ndarray:
    out = _stable_normalize(radial_raw)
    out[source] = 0.0
    return out


def radial_divergence(state: VectorHeat, radial_raw: np.ndarray, source: int) -> np.ndarray:
    """``-sum_j w_ij <X_ij, e_ij>`` of the unit radial field (kernels/heat.py:4163-4225)."""
    v = state.vertices.astype(F64)
    f = state.faces
    flat = f.reshape(-1)
    cot = state.ops["cot"].astype(F64)
    unit = _unit_radial(radial_raw, source)

    def flux(h: np.ndarray, nh: np.ndarray, w: np.ndarray) -> np.ndarray:
        i, j = flat[h], flat[nh]
        back = _complex(unit[j], _polar(-state.transport[h]))
        length = np.linalg.norm(v[j] - v[i], axis=1)
        edge = length[:, None] * _polar(state.tangent[h])
        return w * (0.5 * (unit[i] + back) * edge).sum(axis=1)

    base = 3 * np.arange(f.shape[0])
    f01 = flux(base, base + 1, cot[:, 2])
    f12 = flux(base + 1, base + 2, cot[:, 0])
    f20 = flux(base + 2, base, cot[:, 1])
    out = np.zeros(state.n)
    np.add.at(out, flat, np.stack((f20 - f01, f01 - f12, f12 - f20), axis=1).reshape(-1))
    return out


def _log_map_vector_heat(state: VectorHeat, source: int) -> np.ndarray:
    """``log_map(method="potpourri3d")`` (heat.py:2952-3027, kernels/heat.py:4228-4243)."""
    radial_rhs, horizontal_rhs = outward_ball(state, source)
    radial_raw = state.diffuse_tangent(radial_rhs.reshape(-1)).reshape(-1, 2)
    horizontal_raw = state.diffuse_tangent(horizontal_rhs.reshape(-1)).reshape(-1, 2)
    divergence = radial_divergence(state, radial_raw, source)
    distance = hp.PoissonFactor(hp.csr_matrix(state.ops["pattern"], state.ops["P"])).solve(divergence)
    radial = _unit_radial(radial_raw, source)
    horizontal = _stable_normalize(horizontal_raw)
    conjugate = np.stack((horizontal[:, 0], -horizontal[:, 1]), axis=1)
    return ((distance - distance[source])[:, None] * _complex(radial, conjugate)).astype(F32)
