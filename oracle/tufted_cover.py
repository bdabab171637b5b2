"""CPU restatement of the intrinsic tufted cover (TEST INFRASTRUCTURE: the checker only).

``heat_geodesic(method="potpourri3d", use_robust=True)`` runs the heat method on geometry-central's
intrinsic Delaunay tufted cover of the mesh (ordito/heat.py:5084 ``_tufted_intrinsic_delaunay``,
:3749 ``_cover_operators``; ordito/kernels/heat.py:710-1204): every face doubled into a front and a
reversed back copy, edges glued into a closed surface, lengths mollified and flipped to intrinsic
Delaunay in rounds of independent sets, and the mass, Laplacian, time step, gradient and
divergence all formed from the flipped float64 lengths.

Every float64 expression is evaluated in the order the device kernels evaluate it, one rounding
per operation (no fused multiply-adds), so the flips this module makes are the device's flip for
flip, and the lengths agree bit for bit wherever the mollification adds nothing.
"""

from __future__ import annotations

import numpy as np

from . import heat_path as hp

F64 = np.float64
INT32_MAX = 2**31 - 1
TOLERANCE_MOLLIFY = 1e-5           # ordito/constants.py:31
DELAUNAY_EPSILON = 1e-6            # ordito/heat.py:194 (_GEOMETRY_CENTRAL_DELAUNAY_EPSILON)
FLIP_ROUNDS = 4096                 # ordito/heat.py:197 (_COVER_FLIP_ROUNDS)


def _next(h: np.ndarray) -> np.ndarray:
    """``halfedge_next`` (ordito/kernels/halfedge.py:41)."""
    return h - h % 3 + (h + 1) % 3


def _prev(h: np.ndarray) -> np.ndarray:
    """``halfedge_prev`` (ordito/kernels/halfedge.py:48)."""
    return h - h % 3 + (h + 2) % 3


def _back_corner(e: np.ndarray) -> np.ndarray:
    """``cover_back_corner`` (ordito/kernels/heat.py:736): the back copy of ``(c0, c1, c2)`` is
    ``(c0, c2, c1)``."""
    return np.where(e == 0, 0, 3 - e)


def halfedge_mates(faces: np.ndarray) -> np.ndarray:
    """Every halfedge's partner on its undirected edge (ordito/halfedge.py:609-669): the other
    halfedge when exactly two span the edge, ``-1`` for one, ``-2 - lowest`` for three or more.
    Halfedge ``3 f + k`` runs corner ``k`` to corner ``k + 1``."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1)
    n_h = f.size
    h = np.arange(n_h)
    a, b = f[h], f[_next(h)]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    order = np.lexsort((h, hi, lo))
    lo_s, hi_s = lo[order], hi[order]
    starts = np.flatnonzero(np.r_[True, (lo_s[1:] != lo_s[:-1]) | (hi_s[1:] != hi_s[:-1])])
    sizes = np.diff(np.r_[starts, n_h])
    mates = np.full(n_h, -1, dtype=np.int64)
    for start, size in zip(starts, sizes):
        run = order[start:start + size]
        if size == 2:
            mates[run[0]], mates[run[1]] = run[1], run[0]
        elif size >= 3:
            mates[run] = -2 - int(run.min())
    return mates


def tufted_cover(vertices: np.ndarray, faces: np.ndarray, mates: np.ndarray) -> tuple[np.ndarray, ...]:
    """The tufted cover before mollification (ordito/kernels/heat.py:749-798 ``tufted_cover``,
    :841-873 ``glue_nonmanifold_cover_edges``): ``(cover_faces (6F,), lengths (2F, 3), twin
    (6F,))``. Cover face ``f`` is face ``f``'s front copy, ``F + f`` its back copy; slot ``3 g + e``
    is the edge of cover face ``g`` opposite its corner ``e``."""
    v = np.asarray(vertices, dtype=np.float32).reshape(-1, 3).astype(F64)
    f = np.asarray(faces, dtype=np.int64).reshape(-1)
    n_faces = f.size // 3
    h = np.arange(3 * n_faces)
    face, e = h // 3, h % 3
    back = 3 * (n_faces + face) + _back_corner(e)
    cover = np.empty(6 * n_faces, dtype=np.int64)
    cover[h] = f[h]
    cover[back] = f[h]
    tail, tip = f[_next(h)], f[_prev(h)]
    d = v[tip] - v[tail]
    length = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    lengths = np.empty((2 * n_faces, 3), dtype=F64)
    lengths[face, e] = length
    lengths[n_faces + face, _back_corner(e)] = length
    twin = np.full(6 * n_faces, -1, dtype=np.int64)
    mate = np.asarray(mates, dtype=np.int64)[_next(h)]
    rim = mate == -1
    twin[h[rim]] = back[rim]
    twin[back[rim]] = h[rim]
    pair = mate >= 0
    hp_, bp, mp = h[pair], back[pair], mate[pair]
    front_mate = _prev(mp)
    back_mate = 3 * (n_faces + front_mate // 3) + _back_corner(front_mate % 3)
    same_way = f[mp] == tail[pair]
    twin[hp_] = np.where(same_way, back_mate, front_mate)
    twin[bp] = np.where(same_way, front_mate, back_mate)
    # Edges of three or more faces: each edge's halfedges in index order, each one's copy running
    # against the lowest glued to its predecessor's (the lowest's: the highest's) copy running along.
    many = np.flatnonzero(np.asarray(mates, dtype=np.int64) <= -2)
    if many.size:
        lowest = -2 - np.asarray(mates, dtype=np.int64)[many]
        order = np.lexsort((many, lowest))
        hs, ls = many[order], lowest[order]
        starts = np.flatnonzero(np.r_[True, ls[1:] != ls[:-1]])
        ends = np.r_[starts[1:], hs.size]

        def copy_of(x: int, forward: bool) -> int:
            front = int(_prev(np.int64(x)))
            if forward:
                return front
            return 3 * (n_faces + x // 3) + int(_back_corner(np.int64(front % 3)))

        for s, t in zip(starts, ends):
            run = hs[s:t]
            tail0 = f[run[0]]
            for p in range(run.size):
                x = int(run[p])
                sib = int(run[p - 1]) if p > 0 else int(run[-1])
                backward = copy_of(x, bool(f[x] != tail0))
                forward = copy_of(sib, bool(f[sib] == tail0))
                twin[backward] = forward
                twin[forward] = backward
    return cover, lengths, twin


def length_sums(lengths: np.ndarray) -> tuple[float, float, float]:
    """``(sum, count, worst)`` of a length table (ordito/kernels/heat.py:876-905): the sum and
    count of its entries and its largest triangle-inequality violation ``c - a - b``."""
    a, b, c = lengths[:, 0], lengths[:, 1], lengths[:, 2]
    worst = np.maximum(a - b - c, np.maximum(b - c - a, c - a - b))
    return float(np.sum(lengths)), float(lengths.size), float(worst.max()) if worst.size else -np.inf


def mollify(lengths: np.ndarray, n_faces: int, epsilon: float = TOLERANCE_MOLLIFY) -> np.ndarray:
    """``mollifyIntrinsic`` (ordito/kernels/heat.py:908-921, heat.py:5135-5138): every length grows
    by ``max(0, worst + epsilon * mean)`` over the front copies' table."""
    total, count, worst = length_sums(lengths[:n_faces])
    delta = epsilon * total / count
    return lengths + max(0.0, worst + delta)


def heron(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """``heron_area_float64`` (ordito/kernels/heat.py:924-928)."""
    s = ((a + b) + c) / 2.0
    return np.sqrt(np.maximum(0.0, ((s * (s - a)) * (s - b)) * (s - c)))


def half_cotangent(lengths: np.ndarray, face: np.ndarray, e: np.ndarray, area: np.ndarray) -> np.ndarray:
    """``cover_half_cotangent`` (ordito/kernels/heat.py:931-941): ``(b^2 + c^2 - a^2) / (8 A)``."""
    a = lengths[face, e]
    b = lengths[face, (e + 1) % 3]
    c = lengths[face, (e + 2) % 3]
    with np.errstate(divide="ignore", invalid="ignore"):
        return ((b * b + c * c) - a * a) / (8.0 * area)


def slot_half_cotangent(lengths: np.ndarray, h: np.ndarray) -> np.ndarray:
    face = h // 3
    area = heron(lengths[face, 0], lengths[face, 1], lengths[face, 2])
    return half_cotangent(lengths, face, h % 3, area)


def unfolded_diagonal(ab, bc, ca, bd, dc):
    """``unfolded_diagonal`` (ordito/kernels/heat.py:952-964): the quad's other diagonal ``|ad|``."""
    with np.errstate(divide="ignore", invalid="ignore"):
        ax = ((ab * ab + bc * bc) - ca * ca) / (2.0 * bc)
        ay = np.sqrt(np.maximum(0.0, ab * ab - ax * ax))
        dx = ((bd * bd + bc * bc) - dc * dc) / (2.0 * bc)
        dy = -np.sqrt(np.maximum(0.0, bd * bd - dx * dx))
        x, y = ax - dx, ay - dy
        return np.sqrt(x * x + y * y)


def flip_round(cover: np.ndarray, lengths: np.ndarray, twin: np.ndarray,
               epsilon: float = DELAUNAY_EPSILON) -> tuple[np.ndarray, np.ndarray, np.ndarray, int]:
    """One round of ``flipToDelaunay`` (ordito/kernels/heat.py:967-1130: ``cover_flip_candidates``,
    ``cover_flip_commit``, ``cover_flip_fixup``): every edge failing the Euclidean Delaunay test
    is a candidate; the lowest candidate slot of each face claims it, and a candidate owning both
    of its faces flips. Returns the new faces, lengths and twins and the number of flips."""
    n_slots = twin.size
    n_cover = n_slots // 3
    h = np.arange(n_slots)
    t = twin
    live = (t > h) & (h // 3 != t // 3)
    hs, ts = h[live], t[live]
    weight = slot_half_cotangent(lengths, hs) + slot_half_cotangent(lengths, ts)
    fail = weight < -epsilon
    hs, ts = hs[fail], ts[fail]
    f0, f1 = hs // 3, ts // 3
    e0, e1 = hs % 3, ts % 3
    new_length = unfolded_diagonal(lengths[f0, (e0 + 2) % 3], lengths[f0, e0], lengths[f0, (e0 + 1) % 3],
                                   lengths[f1, (e1 + 1) % 3], lengths[f1, (e1 + 2) % 3])
    ok = np.isfinite(new_length)
    hs, ts, f0, f1, e0, e1, new_length = hs[ok], ts[ok], f0[ok], f1[ok], e0[ok], e1[ok], new_length[ok]
    claim = np.full(n_cover, np.iinfo(np.int64).max, dtype=np.int64)
    np.minimum.at(claim, f0, hs)
    np.minimum.at(claim, f1, hs)
    won = (claim[f0] == hs) & (claim[f1] == hs)
    hs, ts, f0, f1, e0, e1, new_length = (x[won] for x in (hs, ts, f0, f1, e0, e1, new_length))
    faces_new, lengths_new = cover.copy(), lengths.copy()
    pending = np.full(n_slots, -1, dtype=np.int64)
    remap = np.full(n_slots, -1, dtype=np.int64)
    flipped = np.zeros(n_cover, dtype=bool)
    for x, y, g0, g1, c0, c1, ad in zip(hs, ts, f0, f1, e0, e1, new_length):
        a, b, c, d = cover[x], cover[_next(x)], cover[_prev(x)], cover[y]
        ca, ab = lengths[g0, (c0 + 1) % 3], lengths[g0, (c0 + 2) % 3]
        bd, dc = lengths[g1, (c1 + 1) % 3], lengths[g1, (c1 + 2) % 3]
        for old, new in ((_next(y), 3 * g0), (_prev(x), 3 * g0 + 2), (_next(x), 3 * g1),
                         (_prev(y), 3 * g1 + 2)):
            pending[new] = twin[old]
            remap[old] = new
        pending[3 * g0 + 1] = -2 - (3 * g1 + 1)
        pending[3 * g1 + 1] = -2 - (3 * g0 + 1)
        faces_new[3 * g0:3 * g0 + 3] = (a, b, d)
        faces_new[3 * g1:3 * g1 + 3] = (d, c, a)
        lengths_new[g0] = (bd, ad, ab)
        lengths_new[g1] = (ca, ad, dc)
        flipped[g0] = flipped[g1] = True
    other = np.where(flipped[h // 3], pending, twin)
    final = other <= -2
    twin_new = np.where(final, -2 - other, np.where(remap[np.maximum(other, 0)] >= 0, remap[np.maximum(other, 0)], other))
    return faces_new, lengths_new, twin_new, int(hs.size)


def intrinsic_delaunay(vertices: np.ndarray, faces: np.ndarray,
                       max_rounds: int = FLIP_ROUNDS) -> tuple[np.ndarray, np.ndarray, np.ndarray, int]:
    """``_tufted_intrinsic_delaunay`` (ordito/heat.py:5084-5160): the mollified tufted cover
    flipped to intrinsic Delaunay. Returns ``(cover_faces, lengths, twin, rounds)``."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1)
    n_faces = f.size // 3
    cover, lengths, twin = tufted_cover(vertices, f, halfedge_mates(f))
    lengths = mollify(lengths, n_faces)
    rounds = 0
    for _ in range(max_rounds):
        cover, lengths, twin, flips = flip_round(cover, lengths, twin)
        rounds += 1
        if flips == 0:
            break
    return cover, lengths, twin, rounds


def cover_face_terms(cover: np.ndarray, lengths: np.ndarray, n_vertices: int) -> tuple[np.ndarray, np.ndarray]:
    """``cover_face_terms`` (ordito/kernels/heat.py:1133-1151): each cover face's three
    half-cotangents (float64) and each vertex's corner area sum, corners in ascending order."""
    n_cover = lengths.shape[0]
    g = np.arange(n_cover)
    area = heron(lengths[:, 0], lengths[:, 1], lengths[:, 2])
    cot = np.stack([half_cotangent(lengths, g, np.full(n_cover, e), area) for e in range(3)], axis=1)
    sums = np.zeros(n_vertices, dtype=F64)
    np.add.at(sums, np.asarray(cover, dtype=np.int64), np.repeat(area, 3))
    return cot, sums


def cover_operators(vertices: np.ndarray, faces: np.ndarray, t: float | None = None) -> dict[str, object]:
    """``HeatSolver._cover_operators`` (ordito/heat.py:3749-3830): the heat operators over the
    cover's own cotmatrix pattern, from its flipped lengths; with ``t`` None the time is the
    squared mean cover edge (every cover slot's length, each edge counted from both sides)."""
    v = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
    n = v.shape[0]
    cover, lengths, twin, rounds = intrinsic_delaunay(v, faces)
    cot, sums = cover_face_terms(cover, lengths, n)
    if t is None:
        total, count, _ = length_sums(lengths)
        mean = total / count if count > 0 else 0.0
        t = mean * mean
    ops = hp.heat_operators(v, cover.reshape(-1, 3), float(t), method="potpourri3d", cot=cot,
                            area_sums=sums)
    ops.update(cover_faces=cover, lengths=lengths, twin=twin, rounds=rounds)
    return ops


def cover_divergence(cover: np.ndarray, lengths: np.ndarray, cot: np.ndarray, u: np.ndarray,
                     n_vertices: int) -> np.ndarray:
    """``cover_unit_gradient_divergence`` (ordito/kernels/heat.py:1154-1204): each cover face laid
    out in the plane from its lengths, the field's gradient direction there, and each slot's term
    ``cot * dot(edge, x)`` added to its tail and taken from its tip; positive divergence."""
    c = np.asarray(cover, dtype=np.int64).reshape(-1, 3)
    l0, l1, l2 = lengths[:, 0], lengths[:, 1], lengths[:, 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        x2 = ((l2 * l2 + l1 * l1) - l0 * l0) / (2.0 * l2)
        y2 = np.sqrt(np.maximum(0.0, l1 * l1 - x2 * x2))
        e0 = np.stack([x2 - l2, y2], axis=1)
        e1 = np.stack([-x2, -y2], axis=1)
        e2 = np.stack([l2, np.zeros_like(l2)], axis=1)
        perp = lambda e: np.stack([-e[:, 1], e[:, 0]], axis=1)  # noqa: E731
        g = perp(e0) * u[c[:, 0], None] + perp(e1) * u[c[:, 1], None] + perp(e2) * u[c[:, 2], None]
        largest = np.abs(g).max(axis=1)
        w = g / np.where(largest > 0, largest, 1.0)[:, None]
        norm = np.sqrt(w[:, 0] * w[:, 0] + w[:, 1] * w[:, 1])
        x = np.where((largest > 0)[:, None], w / np.where(norm > 0, norm, 1.0)[:, None], 0.0)
    t0 = cot[:, 0] * (e0[:, 0] * x[:, 0] + e0[:, 1] * x[:, 1])
    t1 = cot[:, 1] * (e1[:, 0] * x[:, 0] + e1[:, 1] * x[:, 1])
    t2 = cot[:, 2] * (e2[:, 0] * x[:, 0] + e2[:, 1] * x[:, 1])
    out = np.zeros(n_vertices, dtype=F64)
    corner = np.stack([t2 - t1, t0 - t2, t1 - t0], axis=1)
    np.add.at(out, c.reshape(-1), corner.reshape(-1))
    return out


def heat_geodesic_robust(vertices: np.ndarray, faces: np.ndarray, sources: np.ndarray,
                         t: float | None = None, *, operators: dict[str, object] | None = None) -> np.ndarray:
    """``heat_geodesic(method="potpourri3d", use_robust=True)`` (ordito/heat.py:391, 3632-3660,
    3052-3131): heat and regularized Poisson solves on the cover's operators, both direct."""
    v = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
    n = v.shape[0]
    src = np.asarray(sources, dtype=np.int64)
    if operators is None:
        t_eff, _ = hp.vertex_time(v, np.asarray(faces, dtype=np.int64).reshape(-1, 3), t, "potpourri3d")
        operators = cover_operators(v, faces, t_eff)
    ops = operators
    pattern = ops["pattern"]
    heat = hp.solve_heat(hp.csr_matrix(pattern, ops["H"]), hp.seed(src, n))
    div = cover_divergence(ops["cover_faces"], ops["lengths"], ops["cot"], heat, n)
    phi = hp.solve_regularized_poisson(pattern, ops["P"], div)
    return hp.shift_to_sources(phi, src)
