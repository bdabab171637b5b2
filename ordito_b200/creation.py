"""Synthetic mesh generators for the heat-geodesic workloads (host numpy; float32 xyz, int32 faces).

``icosphere`` follows ordito's construction (``ordito/creation.py:641-712``): the geometry of the
recursive projected-midpoint refinement of an icosahedron (the same points ``trimesh`` builds), and
the vertex numbering ordito documents -- the 12 base corners first, then the interior points of each
base edge, then the interior points of each base face. Within an edge or a face the points are
numbered by their barycentric coordinates, which is this module's own choice. ``torus`` is a
revolved ``cols x rows`` quad grid split into triangles (``ordito/creation.py:1383``).
"""

from __future__ import annotations

import numpy as np

_PHI = (1.0 + 5.0**0.5) / 2.0
_ICO_VERTICES = np.array(
    [
        [-1, _PHI, 0], [1, _PHI, 0], [-1, -_PHI, 0], [1, -_PHI, 0],
        [0, -1, _PHI], [0, 1, _PHI], [0, -1, -_PHI], [0, 1, -_PHI],
        [_PHI, 0, -1], [_PHI, 0, 1], [-_PHI, 0, -1], [-_PHI, 0, 1],
    ],
    dtype=np.float64,
)  # fmt: skip
_ICO_FACES = np.array(
    [
        [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
        [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
        [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
        [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
    ],
    dtype=np.int64,
)  # fmt: skip


def icosphere(subdivisions: int = 3, radius: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    """Return ``(vertices float32 (V, 3), faces int32 (F, 3))`` of a refined icosahedron.

    ``V = 10 * 4**s + 2``, ``F = 20 * 4**s``. Each level splits every triangle into four at the
    edge midpoints, projected back onto the unit sphere (computed in float64, stored as float32).
    """
    levels = max(0, int(subdivisions))
    verts = _ICO_VERTICES / np.linalg.norm(_ICO_VERTICES, axis=1, keepdims=True)
    faces = _ICO_FACES.copy()
    scale = 1 << levels
    # Each face corner's integer barycentric coordinates in its base face, at resolution ``scale``.
    bary = np.zeros((20, 3, 3), dtype=np.int64)
    for c in range(3):
        bary[:, c, c] = scale
    base = np.arange(20, dtype=np.int64)
    for _ in range(levels):
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        ends = np.concatenate((np.stack((a, b), 1), np.stack((b, c), 1), np.stack((c, a), 1)))
        lo, hi = ends.min(axis=1), ends.max(axis=1)
        keys, first, inverse = np.unique(lo * verts.shape[0] + hi, return_index=True,
                                         return_inverse=True)
        p = verts[lo[first]] + verts[hi[first]]
        mid_ids = verts.shape[0] + inverse.reshape(3, -1)
        verts = np.concatenate((verts, p / np.linalg.norm(p, axis=1, keepdims=True)))
        m0, m1, m2 = mid_ids
        w0, w1, w2 = bary[:, 0], bary[:, 1], bary[:, 2]
        wm0, wm1, wm2 = (w0 + w1) // 2, (w1 + w2) // 2, (w2 + w0) // 2
        faces = np.stack(
            (np.stack((a, m0, m2), 1), np.stack((m0, b, m1), 1),
             np.stack((m2, m1, c), 1), np.stack((m0, m1, m2), 1)), axis=1,
        ).reshape(-1, 3)
        bary = np.stack(
            (np.stack((w0, wm0, wm2), 1), np.stack((wm0, w1, wm1), 1),
             np.stack((wm2, wm1, w2), 1), np.stack((wm0, wm1, wm2), 1)), axis=1,
        ).reshape(-1, 3, 3)
        base = np.repeat(base, 4)
    # Canonical numbering: corners, then edge interiors (by base edge, then position along it),
    # then face interiors (by base face, then barycentric (w1, w2)).
    n = verts.shape[0]
    edge_ids = {}
    for tri in _ICO_FACES:
        for e in range(3):
            u, v = int(tri[e]), int(tri[(e + 1) % 3])
            edge_ids.setdefault((min(u, v), max(u, v)), len(edge_ids))
    edge_table = np.full((12, 12), -1, dtype=np.int64)
    for (u, v), k in edge_ids.items():
        edge_table[u, v] = edge_table[v, u] = k
    corner_bary = bary.reshape(-1, 3)
    corner_vertex = faces.reshape(-1)
    corner_base = np.repeat(base, 3)
    tri = _ICO_FACES[corner_base]
    nonzero = (corner_bary != 0).sum(axis=1)
    dim = np.where(nonzero == 1, 0, np.where(nonzero == 2, 1, 2))
    # On an edge: the two base corners with weight, position = weight at the higher-numbered one.
    first_zero = np.argmin(corner_bary != 0, axis=1)
    ca = tri[np.arange(tri.shape[0]), (first_zero + 1) % 3]
    cb = tri[np.arange(tri.shape[0]), (first_zero + 2) % 3]
    wa = corner_bary[np.arange(tri.shape[0]), (first_zero + 1) % 3]
    wb = corner_bary[np.arange(tri.shape[0]), (first_zero + 2) % 3]
    edge_pos = np.where(ca > cb, wa, wb)
    simplex = np.where(dim == 0, corner_vertex, np.where(dim == 1, edge_table[ca, cb], corner_base))
    k1 = np.where(dim == 1, edge_pos, np.where(dim == 2, corner_bary[:, 1], 0))
    k2 = np.where(dim == 2, corner_bary[:, 2], 0)
    key = np.zeros((n, 4), dtype=np.int64)
    key[corner_vertex] = np.stack((dim, simplex, k1, k2), axis=1)
    perm = np.lexsort((key[:, 3], key[:, 2], key[:, 1], key[:, 0]))
    relabel = np.empty(n, dtype=np.int64)
    relabel[perm] = np.arange(n)
    vertices = (verts[perm] * radius).astype(np.float32)
    return vertices, relabel[faces].astype(np.int32)


def torus(
    cols: int = 512, rows: int = 256, major: float = 1.0, minor: float = 0.3
) -> tuple[np.ndarray, np.ndarray]:
    """A revolved torus grid: ``cols`` sections around the axis, ``rows`` around the tube.

    Vertex ``(i, j)`` is ``i * rows + j`` at angles ``u = 2 pi i / cols``, ``v = 2 pi j / rows``;
    each grid quad is split into two triangles along its ``(i, j) - (i+1, j+1)`` diagonal, wound
    so the normals point out of the tube.
    """
    i, j = np.meshgrid(np.arange(cols), np.arange(rows), indexing="ij")
    u = 2.0 * np.pi * i / cols
    v = 2.0 * np.pi * j / rows
    ring = major + minor * np.cos(v)
    vertices = np.stack((ring * np.cos(u), ring * np.sin(u), minor * np.sin(v)), axis=-1)
    a = (i * rows + j).ravel()
    b = (((i + 1) % cols) * rows + j).ravel()
    c = (((i + 1) % cols) * rows + (j + 1) % rows).ravel()
    d = (i * rows + (j + 1) % rows).ravel()
    faces = np.empty((2 * a.size, 3), dtype=np.int64)
    faces[0::2] = np.stack((a, b, c), axis=1)
    faces[1::2] = np.stack((a, c, d), axis=1)
    return vertices.reshape(-1, 3).astype(np.float32), faces.astype(np.int32)


def mean_face_edge_length(vertices: np.ndarray, faces: np.ndarray) -> float:
    v = np.asarray(vertices, dtype=np.float64)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    total = 0.0
    for e in range(3):
        total += np.linalg.norm(v[f[:, (e + 1) % 3]] - v[f[:, e]], axis=1).sum()
    return float(total / (3 * f.shape[0]))


def jittered_torus(
    cols: int = 512,
    rows: int = 256,
    major: float = 1.0,
    minor: float = 0.3,
    sigma_edges: float = 0.1,
    seed: int = 0,
) -> tuple[np.ndarray, np.ndarray]:
    """``torus`` with i.i.d. ``N(0, (sigma_edges * h)^2)`` noise per coordinate, ``h`` the clean
    torus's mean edge length, drawn from ``numpy.random.default_rng(seed)``."""
    vertices, faces = torus(cols, rows, major, minor)
    h = mean_face_edge_length(vertices, faces)
    rng = np.random.default_rng(seed)
    noisy = vertices.astype(np.float64) + rng.normal(0.0, sigma_edges * h, size=vertices.shape)
    return noisy.astype(np.float32), faces


def radial_noise(vertices: np.ndarray, fraction: float, seed: int) -> np.ndarray:
    """Scale each vertex's radius by ``1 + N(0, fraction^2)`` (seeded), for the large sphere."""
    rng = np.random.default_rng(seed)
    scale = 1.0 + rng.normal(0.0, fraction, size=(vertices.shape[0], 1))
    return (vertices.astype(np.float64) * scale).astype(np.float32)


def grid(count: tuple[int, int] = (2, 2)) -> tuple[np.ndarray, np.ndarray]:
    """A unit-square ``nx x ny`` vertex grid in the z = 0 plane, two triangles per cell.

    Cell ``(x, y)`` with lower-left vertex ``a`` is split as ``(a, a+1, a+nx+1)`` and
    ``(a, a+nx+1, a+nx)``, which for ``(2, 2)`` gives the half-cotangent table ordito's
    ``cotmatrix_entries`` docstring states (``ordito/laplacian.py:240-249``).
    """
    nx, ny = count
    xs = np.linspace(0.0, 1.0, nx)
    ys = np.linspace(0.0, 1.0, ny)
    x, y = np.meshgrid(xs, ys, indexing="xy")
    vertices = np.stack((x.ravel(), y.ravel(), np.zeros(x.size)), axis=1).astype(np.float32)
    faces = []
    for cy in range(ny - 1):
        for cx in range(nx - 1):
            a = cy * nx + cx
            faces += [[a, a + 1, a + nx + 1], [a, a + nx + 1, a + nx]]
    return vertices, np.asarray(faces, dtype=np.int32)


def flat_grid(count: tuple[int, int] = (10, 10), extents: tuple[float, float] = (1.0, 1.0),
              center: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """ordito's ``creation.grid`` patch (``ordito/creation.py:385``, ``kernels/creation.py:70``):
    ``nx x ny`` vertices in the z = 0 plane numbered ``i * ny + j`` (X the slow axis) at
    ``origin + extent * (k / (n - 1))``, cell ``(i, j)`` split into ``(c, c + ny, c + ny + 1)`` and
    ``(c, c + ny + 1, c + 1)``, both wound counter-clockwise seen from +Z. Vertex and face
    numbering matter to the tangent frames (their gauge starts at each vertex's highest face)."""
    nx, ny = int(count[0]), int(count[1])
    if nx < 2 or ny < 2:
        raise ValueError(f"count must be at least 2 along each axis, got {count}")
    width, height = float(extents[0]), float(extents[1])
    x0 = -0.5 * width if center else 0.0
    y0 = -0.5 * height if center else 0.0
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    x = x0 + width * (i.astype(np.float64) / (nx - 1))
    y = y0 + height * (j.astype(np.float64) / (ny - 1))
    vertices = np.stack((x.ravel(), y.ravel(), np.zeros(nx * ny)), axis=1).astype(np.float32)
    corner = (i[:-1, :-1] * ny + j[:-1, :-1]).ravel()
    faces = np.empty((2 * corner.size, 3), dtype=np.int32)
    faces[0::2] = np.stack((corner, corner + ny, corner + ny + 1), axis=1)
    faces[1::2] = np.stack((corner, corner + ny + 1, corner + 1), axis=1)
    return vertices, faces


def octahedron() -> tuple[np.ndarray, np.ndarray]:
    """The unit octahedron: vertices +x, +y, +z, -x, -y, -z and the 8 outward faces in ordito's
    numbering (``ordito/creation.py:215-229``; the ring and frame known answers depend on it)."""
    vertices = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]],
                        dtype=np.float32)
    # Faces around +x (vertex 0), then around -x (vertex 3), each counter-clockwise from outside.
    faces = np.array([[0, 1, 2], [0, 2, 4], [0, 4, 5], [0, 5, 1],
                      [3, 1, 5], [3, 5, 4], [3, 4, 2], [3, 2, 1]], dtype=np.int32)
    return vertices, faces


def box() -> tuple[np.ndarray, np.ndarray]:
    """The unit cube ``[0, 1]^3`` as 8 vertices and 12 outward-wound triangles."""
    vertices = np.array(
        [[x, y, z] for z in (0.0, 1.0) for y in (0.0, 1.0) for x in (0.0, 1.0)], dtype=np.float32
    )
    quads = [
        (0, 2, 3, 1),  # z = 0
        (4, 5, 7, 6),  # z = 1
        (0, 1, 5, 4),  # y = 0
        (2, 6, 7, 3),  # y = 1
        (0, 4, 6, 2),  # x = 0
        (1, 3, 7, 5),  # x = 1
    ]
    faces = []
    for a, b, c, d in quads:
        faces += [[a, b, c], [a, c, d]]
    return vertices, np.asarray(faces, dtype=np.int32)
