"""CPU restatement of ordito's heat-method geodesic path (TEST INFRASTRUCTURE: the checker only).

Each function restates one step of the reference and cites the file:line it follows (paths are
within the ordito project). Per-face geometry is computed in float32 exactly as the reference's
kernels do (``np.float32`` arithmetic, one rounding per operation), sums and operator values in
float64, and both linear solves are *direct* float64 solves (scipy SuperLU), so this is the
"same discretisation factored and solved in float64 on the host".
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.csgraph as csgraph
import scipy.sparse.linalg as spla

F32 = np.float32
F64 = np.float64


# --------------------------------------------------------------------------------------------
# Pattern: ordito/kernels/laplacian.py:707-748 (store_operator_keys), kernels/array.py:1163-1167
# (csr_key), array.py:1688-1807 (csr_from_keys), laplacian.py:1212-1299 (directed build).
# --------------------------------------------------------------------------------------------


def key_bits(value: int) -> int:
    """Bits a radix sort needs to order keys below ``value`` (``_launch.key_bits``)."""
    return max(1, int(value - 1).bit_length())


def csr_key(row: np.ndarray, col: np.ndarray, n_rows: int, n_cols: int) -> np.ndarray:
    """``row * n_cols + col`` as uint64, the sentinel ``n_rows * n_cols`` outside (array.py:1163)."""
    row = np.asarray(row, dtype=np.int64)
    col = np.asarray(col, dtype=np.int64)
    inside = (row >= 0) & (row < n_rows) & (col >= 0) & (col < n_cols)
    key = np.where(inside, row * n_cols + col, n_rows * n_cols)
    return key.astype(np.uint64)


def operator_keys(faces: np.ndarray, n_vertices: int) -> tuple[np.ndarray, np.ndarray]:
    """The directed ``"cotmatrix"`` keys and corner payloads (kernels/laplacian.py:707-748).

    Slots ``6 f + 2 e`` and ``+1`` hold edge ``(i, j)`` and ``(j, i)`` opposite corner ``e``
    (``i`` = corner ``e+1``, ``j`` = corner ``e+2``), payload ``3 f + e``; the tail of
    ``n_vertices`` slots holds the diagonal key of every referenced vertex, the sentinel
    otherwise (laplacian.py:1263-1266). The tail payload is never read by the reference; it is
    defined here as ``-1``.
    """
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    n_faces = f.shape[0]
    count = 6 * n_faces + n_vertices
    keys = np.empty(count, dtype=np.uint64)
    order = np.empty(count, dtype=np.int32)
    for e in range(3):
        i = f[:, (e + 1) % 3]
        j = f[:, (e + 2) % 3]
        keys[2 * e : 6 * n_faces : 6] = csr_key(i, j, n_vertices, n_vertices)
        keys[2 * e + 1 : 6 * n_faces : 6] = csr_key(j, i, n_vertices, n_vertices)
        slot = (3 * np.arange(n_faces) + e).astype(np.int32)
        order[2 * e : 6 * n_faces : 6] = slot
        order[2 * e + 1 : 6 * n_faces : 6] = slot
    tail = np.full(n_vertices, n_vertices * n_vertices, dtype=np.uint64)
    referenced = f.ravel()
    referenced = referenced[(referenced >= 0) & (referenced < n_vertices)]
    tail[referenced] = (referenced * n_vertices + referenced).astype(np.uint64)
    keys[6 * n_faces :] = tail
    order[6 * n_faces :] = -1
    return keys, order


def csr_from_keys(
    keys: np.ndarray, order: np.ndarray, n_rows: int, n_cols: int
) -> dict[str, np.ndarray]:
    """Stable sort of the keys, runs of equal in-range keys -> CSR (array.py:1688-1807).

    Returns the sorted ``keys`` and ``order``, ``offsets`` (``n_rows + 1``), the ``nnz`` entries'
    ``columns`` and ``run_start`` (first sorted position of each entry's run).
    """
    perm = np.argsort(keys, kind="stable")
    skeys = keys[perm]
    sorder = order[perm]
    sentinel = np.uint64(n_rows * n_cols)
    count = skeys.size
    inside = skeys < sentinel
    start = np.ones(count, dtype=bool)
    if count > 1:
        start[1:] = skeys[1:] != skeys[:-1]
    flags = inside & start
    run_start = np.flatnonzero(flags).astype(np.int32)
    entry_keys = skeys[flags]
    rows = (entry_keys // np.uint64(n_cols)).astype(np.int64)
    columns = (entry_keys % np.uint64(n_cols)).astype(np.int32)
    offsets = np.zeros(n_rows + 1, dtype=np.int32)
    np.add.at(offsets, rows + 1, 1)
    offsets = np.cumsum(offsets).astype(np.int32)
    return {
        "keys": skeys,
        "order": sorder,
        "offsets": offsets,
        "columns": columns,
        "run_start": run_start,
        "count": count,
    }


def mesh_operator_pattern(faces: np.ndarray, n_vertices: int) -> dict[str, np.ndarray]:
    """``mesh_operator_pattern(faces, n_vertices)`` for the ``"cotmatrix"`` operator.

    laplacian.py:1071 / 1212: every edge both ways plus every referenced vertex's diagonal.
    """
    keys, order = operator_keys(faces, n_vertices)
    pattern = csr_from_keys(keys, order, n_vertices, n_vertices)
    pattern["n_vertices"] = n_vertices
    return pattern


def run_ends(skeys: np.ndarray, run_start: np.ndarray) -> np.ndarray:
    """One past each run's last sorted position (kernels/array.py:1320 sorted_run_end)."""
    count = skeys.size
    boundary = np.ones(count + 1, dtype=bool)
    if count > 1:
        boundary[1:count] = skeys[1:] != skeys[:-1]
    starts = np.flatnonzero(boundary)
    idx = np.searchsorted(starts, run_start, side="right")
    return starts[idx].astype(np.int64)


# --------------------------------------------------------------------------------------------
# Per-face geometry in float32: kernels/predicates.py:106-130 (triangle_area_vector), :186
# (triangle_double_area), kernels/laplacian.py:94-108 (half_cotangents_of),
# kernels/triangles.py:333-359 (face_normals_and_area).
# --------------------------------------------------------------------------------------------


def _dot(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]) + a[:, 2] * b[:, 2]


def _cross(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.stack(
        (
            a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
            a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
            a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0],
        ),
        axis=1,
    )


def _length(a: np.ndarray) -> np.ndarray:
    return np.sqrt(_dot(a, a))


def triangle_area_vector(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """``cross`` at the corner opposite the longest edge (kernels/predicates.py:106-130)."""
    ab = b - a
    bc = c - b
    ca = a - c
    l_ab = _dot(ab, ab)
    l_bc = _dot(bc, bc)
    l_ca = _dot(ca, ca)
    at_a = (l_bc >= l_ca) & (l_bc >= l_ab)
    at_b = ~at_a & (l_ca >= l_ab)
    out = _cross(ca, -bc)
    out = np.where(at_b[:, None], _cross(bc, -ab), out)
    out = np.where(at_a[:, None], _cross(ab, -ca), out)
    return out


def face_corners(vertices: np.ndarray, faces: np.ndarray) -> tuple[np.ndarray, ...]:
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    return v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]


def cotmatrix_entries(vertices: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """``(n_faces, 3)`` float32 half-cotangents, column e opposite corner e (laplacian.py:94-108)."""
    with np.errstate(all="ignore"):
        v0, v1, v2 = face_corners(vertices, faces)
        dbl = _length(triangle_area_vector(v0, v1, v2))
        den = F32(2.0) * dbl
        ok = den > 0
        safe = np.where(ok, den, F32(1.0))
        c0 = _dot(v1 - v0, v2 - v0) / safe
        c1 = _dot(v2 - v1, v0 - v1) / safe
        c2 = _dot(v0 - v2, v1 - v2) / safe
        out = np.stack((c0, c1, c2), axis=1).astype(F32)
        out[~ok] = 0
    return out


TOLERANCE_MOLLIFY = 1e-5  # ordito/constants.py:31


def mollified_lengths(vertices: np.ndarray, faces: np.ndarray,
                      epsilon: float = TOLERANCE_MOLLIFY) -> tuple[np.ndarray, float]:
    """``laplacian.mollify_intrinsic`` (ordito/laplacian.py:779-874, kernels/laplacian.py:1585-1627):
    each face's float32 side lengths (column e opposite corner e) plus the one constant
    ``delta = max(epsilon * mean - min margin, 0)`` that gives every triangle a margin of
    ``epsilon`` times the mean edge length (float32; the mean summed in float64 here)."""
    v0, v1, v2 = face_corners(vertices, faces)
    with np.errstate(all="ignore"):
        lengths = np.stack([_length(v1 - v2), _length(v2 - v0), _length(v0 - v1)], axis=1).astype(F32)
    if lengths.shape[0] == 0:
        return lengths, 0.0
    a, b, c = lengths[:, 0], lengths[:, 1], lengths[:, 2]
    margin = np.min(np.minimum(np.minimum(a + b - c, b + c - a), c + a - b))
    mean = float(lengths.astype(F64).sum()) / lengths.size
    eps = F32(epsilon * mean)
    delta = max(F32(eps - margin), F32(0.0))
    if delta <= 0.0:
        return lengths, 0.0
    return (lengths + F32(delta)).astype(F32), float(delta)


def cot_from_lengths(lengths: np.ndarray) -> np.ndarray:
    """``cotmatrix_entries_intrinsic`` in float32 (kernels/laplacian.py:56-90, 225-249;
    kernels/predicates.py:194-210): the law of cosines over Kahan's Heron double area, the
    largest side first; a zero-area face weighs nothing."""
    L = np.asarray(lengths, dtype=F32)
    srt = np.sort(L, axis=1)
    c, b, a = srt[:, 0], srt[:, 1], srt[:, 2]
    with np.errstate(all="ignore"):
        arg = (a + (b + c)) * (c - (a - b)) * (c + (a - b)) * (a + (b - c))
        dbl = F32(0.5) * np.sqrt(np.maximum(arg, F32(0.0)))
        dbl = np.where(np.isnan(dbl), F32(0.0), dbl).astype(F32)
        den = F32(4.0) * dbl
        sq = L * L
        c0 = (sq[:, 1] + sq[:, 2] - sq[:, 0]) / den
        c1 = (sq[:, 2] + sq[:, 0] - sq[:, 1]) / den
        c2 = (sq[:, 0] + sq[:, 1] - sq[:, 2]) / den
    cot = np.stack([c0, c1, c2], axis=1).astype(F32)
    cot[den <= 0] = 0.0
    return cot


def face_normals_and_areas(vertices: np.ndarray, faces: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Unit normals (zero if degenerate) and areas, float32 (kernels/triangles.py:333-359)."""
    with np.errstate(all="ignore"):
        v0, v1, v2 = face_corners(vertices, faces)
        n = triangle_area_vector(v0, v1, v2)
        norm = _length(n)
        ok = norm > 0
        unit = np.where(ok[:, None], n / np.where(ok, norm, F32(1.0))[:, None], n)
        area = F32(0.5) * norm
    return unit.astype(F32), area.astype(F32)


def area_sums(faces: np.ndarray, areas: np.ndarray, n_vertices: int) -> np.ndarray:
    """Each corner's f32 face area added in float64 (kernels/heat.py:128-131, scatter.py:700)."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    out = np.zeros(n_vertices, dtype=F64)
    a = areas.astype(F64)
    for e in range(3):
        np.add.at(out, f[:, e], a)
    return out


def voronoi_area_sums(vertices: np.ndarray, faces: np.ndarray, n_vertices: int) -> np.ndarray:
    """Each corner's Voronoi share of its face, added in float64: the ``method="igl"`` lumped mass
    (kernels/triangles.py:276-330 face_voronoi_areas, kernels/heat.py:128-129).

    Shares are formed in float64 from the float32 corners (Meyer et al.'s mixed areas: the
    circumcentric split of a non-obtuse face, half to an obtuse corner and a quarter to each other,
    an even split of a face with a zero-length edge or zero circumcentre weights) and rounded once
    to float32.
    """
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    p0, p1, p2 = (v[f[:, e]].astype(F64) for e in range(3))

    def length(a: np.ndarray) -> np.ndarray:
        return np.sqrt(a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1] + a[:, 2] * a[:, 2])

    l0, l1, l2 = length(p1 - p2), length(p2 - p0), length(p0 - p1)
    area = 0.5 * length(np.cross(p1 - p0, p2 - p0))
    q = np.repeat((area / 3.0)[:, None], 3, axis=1)
    with np.errstate(all="ignore"):
        ok = (l0 > 0) & (l1 > 0) & (l2 > 0)
        c0 = (l2 * l2 + l1 * l1 - l0 * l0) / (2.0 * l1 * l2)
        c1 = (l0 * l0 + l2 * l2 - l1 * l1) / (2.0 * l2 * l0)
        c2 = (l1 * l1 + l0 * l0 - l2 * l2) / (2.0 * l0 * l1)
        b0, b1, b2 = c0 * l0, c1 * l1, c2 * l2
        weight = b0 + b1 + b2
        split = ok & (weight != 0.0)
        p_0, p_1, p_2 = b0 / weight * area, b1 / weight * area, b2 / weight * area
        circ = np.stack([0.5 * (p_1 + p_2), 0.5 * (p_2 + p_0), 0.5 * (p_0 + p_1)], axis=1)
    q[split] = circ[split]
    half, quarter = 0.5 * area, 0.25 * area
    for corner, c in enumerate((c0, c1, c2)):
        obtuse = ok & (c < 0.0)
        if corner > 0:
            obtuse &= ~np.any(np.stack([c0, c1, c2][:corner], axis=1) < 0.0, axis=1)
        share = np.repeat(quarter[:, None], 3, axis=1)
        share[:, corner] = half
        q[obtuse] = share[obtuse]
    q = q.astype(F32).astype(F64)
    out = np.zeros(n_vertices, dtype=F64)
    for e in range(3):
        np.add.at(out, f[:, e], q[:, e])
    return out


# --------------------------------------------------------------------------------------------
# Time step: kernels/heat.py:143-237 (upper_edge_length_sum_and_count), kernels/linalg.py:1594
# (shift_factor), heat.py:3714-3736 (_vertex_time), :5228-5243 (_diffusion_floor, _settle_window).
# --------------------------------------------------------------------------------------------

HEAT_CHECK_ROUNDS = 16  # heat.py:142
HEAT_CHANGE_TOLERANCE = 1e-6  # heat.py:146
HEAT_SETTLE_ROUNDS = 192  # heat.py:147
DIFFUSION_DECAY = 400.0  # heat.py:158
CG_TOLERANCE = 1e-8  # heat.py:108


def edge_length_sums(
    vertices: np.ndarray, pattern: dict[str, np.ndarray], face_edges: bool = True
) -> tuple[float, float]:
    """Sum and count of the strict-upper-triangle edge lengths, meshlab weights (heat.py:173-237).

    Each length is the float32 ``length(v_col - v_row)`` widened to float64; with ``face_edges``
    each edge weighs its run length (the number of faces holding it).
    """
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
    offsets = pattern["offsets"]
    columns = pattern["columns"].astype(np.int64)
    rows = np.repeat(np.arange(offsets.size - 1), np.diff(offsets))
    upper = columns > rows
    d = v[columns[upper]] - v[rows[upper]]
    lengths = _length(d).astype(F64)
    if face_edges:
        rs = pattern["run_start"][upper].astype(np.int64)
        weight = (run_ends(pattern["keys"], rs) - rs).astype(F64)
    else:
        weight = np.ones(lengths.size, dtype=F64)
    return float(np.sum(weight * lengths)), float(np.sum(weight))


def mean_face_edge_length(vertices: np.ndarray, faces: np.ndarray) -> float:
    """Mean over all ``3 n_faces`` per-face edges (mesh.py:1179), float32 lengths in float64."""
    v0, v1, v2 = face_corners(vertices, faces)
    if v0.shape[0] == 0:
        return 0.0
    total = (
        _length(v1 - v0).astype(F64).sum()
        + _length(v2 - v1).astype(F64).sum()
        + _length(v0 - v2).astype(F64).sum()
    )
    return float(total / (3 * v0.shape[0]))


def diffusion_floor(vertices: np.ndarray) -> float:
    """``(|bbox diagonal| / 400) ** 2`` (heat.py:5228-5231)."""
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
    low, high = v.min(axis=0).astype(F64), v.max(axis=0).astype(F64)
    return (math.dist(low, high) / DIFFUSION_DECAY) ** 2


def settle_window(t: float | None, default: float) -> int:
    """heat.py:5234-5243."""
    if t is None or not t > default > 0.0:
        return HEAT_SETTLE_ROUNDS
    return math.ceil(HEAT_SETTLE_ROUNDS * math.sqrt(t / default))


def vertex_time(vertices: np.ndarray, faces: np.ndarray, t: float | None,
                method: str = "meshlab") -> tuple[float | None, int]:
    """``HeatSolver._vertex_time`` (heat.py:3714-3736): the mean over every face's three edges for
    ``"meshlab"``, over the unique edges for ``"igl"`` and ``"potpourri3d"``."""
    if method == "meshlab":
        mean = mean_face_edge_length(vertices, faces)
    else:
        v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
        f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
        total, count = edge_length_sums(v, mesh_operator_pattern(f, v.shape[0]), face_edges=False)
        mean = total / count if count > 0 else 0.0
    default = mean**2
    if t is None:
        floor = diffusion_floor(vertices)
        t = floor if floor > default else None
    return t, settle_window(t, default)


# --------------------------------------------------------------------------------------------
# Operators: kernels/heat.py:299-465 (heat_system_rows), kernels/laplacian.py:971-989
# (cotmatrix_offdiagonal), kernels/linalg.py:1594-1621 (shift_factor, shifted_scalar_entry).
# --------------------------------------------------------------------------------------------


def heat_operators(
    vertices: np.ndarray, faces: np.ndarray, t: float | None = None, *, mass_divisor: float = 3.0,
    method: str = "meshlab", use_robust: bool = False, cot: np.ndarray | None = None,
    area_sums: np.ndarray | None = None,
) -> dict[str, object]:
    """The heat operators over the cotmatrix pattern (heat.py:2015-2245): barycentric mass and
    the face-edge time step for ``"meshlab"``, the unique-edge time step for ``"potpourri3d"``,
    the Voronoi mass (divisor 1) and the unique-edge time step for ``"igl"`` (heat.py:2002-2012).
    ``cot`` replaces the half-cotangent table the rows are summed from (a caller's own weights,
    as ``cotmatrix(cot_entries=...)`` takes them, laplacian.py:371); ``area_sums`` the per-vertex
    area sums the lumped mass divides (the intrinsic cover's, heat.py:3783-3784).

    Returns the pattern, the float32 cot table, normals, areas, area sums, ``L``, ``H = M - t L``,
    ``P = -L`` (float64 values over the pattern), the lumped mass and the time ``t`` used.
    """
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    n = v.shape[0]
    pattern = mesh_operator_pattern(f, n)
    # use_robust: the half-cotangents of the mollified lengths (heat.py:2043-2056); the mass, the
    # normals and the areas stay the positions' own.
    if cot is None:
        cot = cot_from_lengths(mollified_lengths(v, f)[0]) if use_robust else cotmatrix_entries(v, f)
    normals, areas = face_normals_and_areas(v, f)
    if area_sums is not None:
        sums = np.asarray(area_sums, dtype=F64)
    elif method == "igl":
        sums = voronoi_area_sums(v, f, n)
        mass_divisor = 1.0
    else:
        sums = globals()["area_sums"](f, areas, n)
    if t is None:
        total, count = edge_length_sums(v, pattern, face_edges=method == "meshlab")
        h = total / count if count > 0 else 0.0
        factor = -1.0 * (h * h)
        t_used = h * h
    else:
        factor = -float(t)
        t_used = float(t)
    offsets = pattern["offsets"]
    columns = pattern["columns"].astype(np.int64)
    nnz = int(offsets[-1])
    rows = np.repeat(np.arange(n), np.diff(offsets))
    diag = columns == rows
    rs = pattern["run_start"].astype(np.int64)
    ends = run_ends(pattern["keys"], rs)
    flat_cot = cot.reshape(-1).astype(F64)
    order = pattern["order"]
    L = np.zeros(nnz, dtype=F64)
    # Off-diagonal entries: the run's half-cotangents in sorted (face) order.
    lengths = ends - rs
    off = np.flatnonzero(~diag)
    max_len = int(lengths[off].max()) if off.size else 0
    for k in range(max_len):
        sel = off[lengths[off] > k]
        L[sel] = L[sel] + flat_cot[order[rs[sel] + k]]
    # Diagonal: minus the row's off-diagonal sum, in row order.
    mass = sums / mass_divisor
    offdiag_vals = np.where(diag, 0.0, L)
    row_len = np.diff(offsets)
    max_row = int(row_len.max()) if n else 0
    totals = np.zeros(n, dtype=F64)
    for k in range(max_row):
        rsel = np.flatnonzero(row_len > k)
        totals[rsel] = totals[rsel] + offdiag_vals[offsets[rsel] + k]
    diag_idx = np.flatnonzero(diag)
    L[diag_idx] = -totals[rows[diag_idx]]
    H = factor * L
    H[diag_idx] = H[diag_idx] + mass[rows[diag_idx]]
    P = -L
    return {
        "pattern": pattern,
        "cot": cot,
        "normals": normals,
        "areas": areas,
        "area_sums": sums,
        "mass": mass,
        "L": L,
        "H": H,
        "P": P,
        "t": t_used,
        "factor": factor,
    }


def csr_matrix(pattern: dict[str, np.ndarray], values: np.ndarray) -> sp.csr_matrix:
    n = pattern["offsets"].size - 1
    nnz = int(pattern["offsets"][-1])
    return sp.csr_matrix(
        (values[:nnz], pattern["columns"][:nnz], pattern["offsets"]), shape=(n, n)
    )


# --------------------------------------------------------------------------------------------
# Per-query: kernels/heat.py:613-623 (seed), :626-687 (unit_gradient_divergence),
# kernels/triangles.py:834-894 (face_gradient_given), kernels/predicates.py:719-724
# (stable_normalize), kernels/heat.py:3383-3424 (source_and_global_sums, shift_and_orient).
# --------------------------------------------------------------------------------------------


def seed(sources: np.ndarray, n_vertices: int) -> np.ndarray:
    src = np.asarray(sources, dtype=np.int64)
    if np.any((src < 0) | (src >= n_vertices)):
        raise ValueError("heat_geodesic: sources must be vertex indices in [0, n_vertices)")
    u0 = np.zeros(n_vertices, dtype=F64)
    u0[src] = 1.0
    return u0


def unit_gradient_divergence(
    vertices: np.ndarray,
    faces: np.ndarray,
    normals: np.ndarray,
    areas: np.ndarray,
    u: np.ndarray,
    cot: np.ndarray,
) -> np.ndarray:
    """Accumulated ``-div(X)`` of the face unit gradients (kernels/heat.py:626-687)."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3).astype(F64)
    v0, v1, v2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    nrm = normals.astype(F64)
    area = areas.astype(F64)
    with np.errstate(all="ignore"):
        g = (
            u[f[:, 0], None] * _cross(nrm, v2 - v1)
            + u[f[:, 1], None] * _cross(nrm, v0 - v2)
            + u[f[:, 2], None] * _cross(nrm, v1 - v0)
        ) / (2.0 * np.where(area > 0, area, 1.0))[:, None]
        g = np.where((area > 0)[:, None], g, 0.0)
        largest = np.abs(g).max(axis=1)
        w = g / np.where(largest > 0, largest, 1.0)[:, None]
        length = _length(w)
        x = np.where((length > 0)[:, None], w / np.where(length > 0, length, 1.0)[:, None], 0.0)
        x = np.where((largest > 0)[:, None], x, 0.0)
    c = cot.astype(F64)
    c0, c1, c2 = c[:, 0], c[:, 1], c[:, 2]
    d0 = c2 * _dot(v1 - v0, x) + c1 * _dot(v2 - v0, x)
    d1 = c0 * _dot(v2 - v1, x) + c2 * _dot(v0 - v1, x)
    d2 = c1 * _dot(v0 - v2, x) + c0 * _dot(v1 - v2, x)
    out = np.zeros(v.shape[0], dtype=F64)
    np.add.at(out, f[:, 0], d0)
    np.add.at(out, f[:, 1], d1)
    np.add.at(out, f[:, 2], d2)
    return out


def shift_to_sources(phi: np.ndarray, sources: np.ndarray) -> np.ndarray:
    """Zero mean over the sources, oriented positive (kernels/heat.py:3383-3424)."""
    src = np.asarray(sources, dtype=np.int64)
    offset = float(np.sum(phi[src])) / src.size
    shifted = phi - offset
    if float(np.sum(phi)) / phi.size - offset < 0.0:
        shifted = offset - phi
    return shifted


# --------------------------------------------------------------------------------------------
# Direct float64 solves: the oracle's stand-in for the settled heat PCG (linalg.py:2490) and the
# Poisson PCG (linalg.py:1356): the exact solutions those iterations approach.
# --------------------------------------------------------------------------------------------


def _active_rows(matrix: sp.csr_matrix) -> np.ndarray:
    return np.flatnonzero(np.diff(matrix.indptr) > 0)


def solve_heat(H: sp.csr_matrix, rhs: np.ndarray) -> np.ndarray:
    """Solve ``(M - t L) u = rhs`` directly; empty rows keep zero (their unknown is untouched)."""
    active = _active_rows(H)
    out = np.zeros(H.shape[0], dtype=F64)
    if active.size == 0:
        return out
    sub = H[active][:, active].tocsc()
    lu = spla.splu(sub, permc_spec="COLAMD")
    rhs2 = np.asarray(rhs, dtype=F64)
    if rhs2.ndim == 1:
        out[active] = lu.solve(rhs2[active])
        return out
    out2 = np.zeros((H.shape[0], rhs2.shape[1]), dtype=F64)
    out2[active] = lu.solve(np.ascontiguousarray(rhs2[active]))
    return out2


class PoissonFactor:
    """``-L`` with the lowest vertex of each connected component pinned, factored once (with
    ``vertices``, in a geometric nested-dissection ordering, as ``HeatFactor``)."""

    def __init__(self, P: sp.csr_matrix, vertices: np.ndarray | None = None) -> None:
        active = _active_rows(P)
        n_comp, labels = csgraph.connected_components(P[active][:, active], directed=False)
        pinned = np.zeros(active.size, dtype=bool)
        seen: set[int] = set()
        for local, label in enumerate(labels):
            if label not in seen:
                seen.add(int(label))
                pinned[local] = True
        self.n = P.shape[0]
        self.free = active[~pinned]
        sub = P[self.free][:, self.free].tocsc()
        if not self.free.size:
            self.lu = None
        elif vertices is not None:
            order = dissection_order(np.asarray(vertices).reshape(-1, 3)[self.free], sub.tocsr())
            self.lu = _Ordered(sub, order)
        else:
            self.lu = spla.splu(sub, permc_spec="COLAMD")

    def solve(self, rhs: np.ndarray) -> np.ndarray:
        out = np.zeros(self.n, dtype=F64)
        if self.lu is not None:
            out[self.free] = self.lu.solve(np.asarray(rhs, dtype=F64)[self.free])
        return out


def rim_vertices(pattern: dict[str, np.ndarray]) -> np.ndarray:
    """1 where a vertex has an edge on a single face: one of its off-diagonal entries' runs holds
    one key (kernels/heat.py:469-485, kernels/laplacian.py:1286-1321)."""
    offsets = pattern["offsets"]
    n = offsets.size - 1
    columns = pattern["columns"][: offsets[-1]].astype(np.int64)
    rows = np.repeat(np.arange(n), np.diff(offsets))
    rs = pattern["run_start"][: offsets[-1]].astype(np.int64)
    single = (run_ends(pattern["keys"], rs) - rs) == 1
    rim = np.zeros(n, dtype=np.int32)
    rim[rows[(columns != rows) & single]] = 1
    return rim


def pinned_heat_values(pattern: dict[str, np.ndarray], H: np.ndarray, rim: np.ndarray) -> np.ndarray:
    """The heat system pinned to zero on the rim: rim rows the identity's, rim columns dropped
    (kernels/heat.py:488-509)."""
    offsets = pattern["offsets"]
    n = offsets.size - 1
    columns = pattern["columns"][: offsets[-1]].astype(np.int64)
    rows = np.repeat(np.arange(n), np.diff(offsets))
    out = np.asarray(H[: offsets[-1]], dtype=F64).copy()
    out[rim[columns] != 0] = 0.0
    on = rim[rows] != 0
    out[on] = np.where(columns[on] == rows[on], 1.0, 0.0)
    return out


GEOMETRY_CENTRAL_POISSON_SHIFT = 1e-6  # heat.py:4090 (the +1e-6 I of HeatMethodDistanceSolver)


def solve_regularized_poisson(pattern: dict[str, np.ndarray], P: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """``(-L + 1e-6 I) phi = rhs`` directly (heat.py:4086-4116); empty rows stay zero."""
    offsets = pattern["offsets"]
    n = offsets.size - 1
    columns = pattern["columns"][: offsets[-1]].astype(np.int64)
    rows = np.repeat(np.arange(n), np.diff(offsets))
    values = np.asarray(P[: offsets[-1]], dtype=F64) + np.where(columns == rows, GEOMETRY_CENTRAL_POISSON_SHIFT, 0.0)
    return solve_heat(csr_matrix(pattern, values), rhs)


def heat_geodesic(
    vertices: np.ndarray,
    faces: np.ndarray,
    sources: np.ndarray,
    t: float | None = None,
    *,
    operators: dict[str, object] | None = None,
    factors: tuple[object, PoissonFactor] | None = None,
    method: str = "meshlab",
    use_robust: bool = False,
) -> np.ndarray:
    """``heat_geodesic(vertices, faces, sources, method=...)`` (heat.py:391-588).

    Both solves are direct. ``"igl"`` averages the Neumann heat with the heat pinned to zero on
    the rim when the mesh has one (heat.py:594-597, 4153-4198); ``"potpourri3d"`` solves
    geometry-central's regularized Poisson system (heat.py:3124-3129). ``operators``/``factors``
    may be passed to reuse them across queries (``factors`` for ``"meshlab"`` only).
    """
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    n = v.shape[0]
    src = np.asarray(sources, dtype=np.int64)
    if n == 0 or f.shape[0] == 0 or src.size == 0:
        return np.zeros(n, dtype=F64)
    u0 = seed(src, n)
    if operators is None:
        t_eff, _ = vertex_time(v, f, t, method)
        operators = heat_operators(v, f, t_eff, method=method, use_robust=use_robust)
    ops = operators
    pattern = ops["pattern"]
    if factors is None:
        H = csr_matrix(pattern, ops["H"])
        P = csr_matrix(pattern, ops["P"])
        heat_lu = HeatFactor(H)
        factors = (heat_lu, PoissonFactor(P) if method != "potpourri3d" else None)
    heat = factors[0].solve(u0)
    if method == "igl":
        rim = rim_vertices(pattern)
        if rim.any():
            pinned = solve_heat(csr_matrix(pattern, pinned_heat_values(pattern, ops["H"], rim)),
                                np.where(rim != 0, 0.0, u0))
            heat = 0.5 * (heat + pinned)
    neg_div = unit_gradient_divergence(v, f, ops["normals"], ops["areas"], heat, ops["cot"])
    if method == "potpourri3d":
        phi = solve_regularized_poisson(pattern, ops["P"], neg_div)
    else:
        phi = factors[1].solve(neg_div)
    return shift_to_sources(phi, src)


def dissection_order(vertices: np.ndarray, matrix: sp.csr_matrix, leaf: int = 64) -> np.ndarray:
    """A geometric nested-dissection ordering (new -> old) of a mesh operator's rows, for direct
    solves of meshes too large for SuperLU's own column ordering (the fallback of the float64
    oracle on the 2.6 M-vertex sphere).

    Level by level every part larger than ``leaf`` is split at the median of its widest
    coordinate; the vertices of the first half adjacent to the second form the part's separator,
    ordered after both halves (a one-sided vertex separator, the kind the reference's ordering
    takes, cholesky.py:2227). The ordering changes only the fill and the rounding of the exact
    factorisation, not what it solves.
    """
    v = np.asarray(vertices, dtype=F64).reshape(-1, 3)
    n = v.shape[0]
    coo = matrix.tocoo()
    off = coo.row != coo.col
    ei, ej = coo.row[off].astype(np.int64), coo.col[off].astype(np.int64)
    part = np.zeros(n, dtype=np.int64)  # the part of every still-undecided vertex
    # Every vertex's path, one base-3 digit a level (0 / 1 the halves, 2 the separator; a
    # decided vertex appends 0), so sorting the keys puts each subtree before its separator.
    key = np.zeros(n, dtype=np.int64)
    done = np.zeros(n, dtype=bool)
    while True:
        live = np.flatnonzero(~done)
        if live.size:
            labels, counts = np.unique(part[live], return_counts=True)
            done[live[~np.isin(part[live], labels[counts > leaf])]] = True
            live = np.flatnonzero(~done)
        if live.size == 0:
            break
        live = live[np.argsort(part[live], kind="stable")]
        p = part[live]
        starts = np.flatnonzero(np.r_[True, p[1:] != p[:-1]])
        sizes = np.diff(np.r_[starts, live.size])
        lo = np.minimum.reduceat(v[live], starts, axis=0)
        hi = np.maximum.reduceat(v[live], starts, axis=0)
        axis = np.argmax(hi - lo, axis=1)
        group = np.repeat(np.arange(starts.size), sizes)
        order = np.lexsort((live, v[live, axis[group]], group))
        live, group = live[order], group[order]
        side = ((np.arange(live.size) - starts[group]) >= sizes[group] // 2).astype(np.int64)
        side_of = np.full(n, -1, dtype=np.int64)
        side_of[live] = side
        cut = (side_of[ei] == 0) & (side_of[ej] == 1) & (part[ei] == part[ej])
        sep = np.zeros(n, dtype=bool)
        sep[ei[cut]] = True
        key *= 3
        key[live] += np.where(sep[live], 2, side)
        done[live[sep[live]]] = True
        part[live] = part[live] * 2 + side
    return np.lexsort((np.arange(n), key))


class _Ordered:
    """SuperLU over rows renumbered by ``order`` (new -> old) with no column reordering of its own
    and no pivoting (the operators are symmetric positive definite on the rows factored)."""

    def __init__(self, sub: sp.csc_matrix, order: np.ndarray) -> None:
        self.order = order
        permuted = sub[order][:, order].tocsc()
        self.lu = spla.splu(permuted, permc_spec="NATURAL", diag_pivot_thresh=0.0,
                            options={"SymmetricMode": True})

    def solve(self, rhs: np.ndarray) -> np.ndarray:
        out = np.empty_like(rhs)
        out[self.order] = self.lu.solve(rhs[self.order])
        return out


class HeatFactor:
    """``M - t L`` factored once (empty rows excluded); ``vertices`` given, in a geometric
    nested-dissection ordering (``dissection_order``), else in SuperLU's COLAMD ordering."""

    def __init__(self, H: sp.csr_matrix, vertices: np.ndarray | None = None) -> None:
        self.n = H.shape[0]
        self.active = _active_rows(H)
        sub = H[self.active][:, self.active].tocsc()
        if not self.active.size:
            self.lu = None
        elif vertices is not None:
            order = dissection_order(np.asarray(vertices).reshape(-1, 3)[self.active], sub.tocsr())
            self.lu = _Ordered(sub, order)
        else:
            self.lu = spla.splu(sub, permc_spec="COLAMD")

    def solve(self, rhs: np.ndarray) -> np.ndarray:
        out = np.zeros(self.n, dtype=F64)
        if self.lu is not None:
            out[self.active] = self.lu.solve(np.asarray(rhs, dtype=F64)[self.active])
        return out


def relative_linf(value: np.ndarray, reference: np.ndarray) -> float:
    """``max |value - reference| / max |reference|``: the error measure stated for distances."""
    scale = float(np.max(np.abs(reference))) if reference.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(value))) if value.size else 0.0
    return float(np.max(np.abs(np.asarray(value, dtype=F64) - reference)) / scale)


def extend_scalar(vertices: np.ndarray, faces: np.ndarray, sources: np.ndarray, values: np.ndarray,
                  t: float | None = None) -> tuple[np.ndarray, float]:
    """``extend_scalar`` (heat.py:2321-2500, kernels/heat.py:3858 and :3933): the indicator of the
    sources and the values they carry diffused through ``M - t L`` (the solver's default
    discretization, potpourri3d's unique-edge time step) in one exact solve, the extension their
    quotient (0 where the indicator is exactly 0). Returns the field and its largest excess over
    the source values' range at vertices the indicator reaches."""
    v = np.asarray(vertices, dtype=F32).reshape(-1, 3)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    n = v.shape[0]
    src = np.asarray(sources, dtype=np.int64)
    vals = np.asarray(values, dtype=F64)
    t_eff, _ = vertex_time(v, f, t, "potpourri3d")
    ops = heat_operators(v, f, t_eff, method="potpourri3d")
    rhs = np.zeros((n, 2), dtype=F64)
    np.add.at(rhs[:, 0], src, 1.0)
    np.add.at(rhs[:, 1], src, vals)
    diffused = solve_heat(csr_matrix(ops["pattern"], ops["H"]), rhs)
    reached = diffused[:, 0] != 0.0
    extended = np.zeros(n, dtype=F64)
    extended[reached] = diffused[reached, 1] / diffused[reached, 0]
    excess = 0.0
    if reached.any():
        excess = float(max(0.0, np.max(np.maximum(extended[reached] - vals.max(), vals.min() - extended[reached]))))
    return extended, excess
