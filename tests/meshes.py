"""Test meshes: small generated fixtures with the properties the reference's tests rely on.

``saddle_graded`` restates ordito's fixture (tests/conftest.py:471-502: a k x k grid on the saddle
z = 0.35 (x^2 - 0.6 y^2), x spacing graded as |t|^e). ``sphere_irregular`` and
``torus_irregular`` restate ordito's irregular closed fixtures (tests/conftest.py:536-639 and
:981-1004: the hull of 500 random directions on a bumpy, longitude-squeezed sphere; 500 random
points Delaunay-triangulated on a flat torus and mapped onto a bumpy, squeezed torus; both
scrambled -- vertex and face order, each face's first corner -- and placed off-axis by a uniform
random rotation, Shoemake's quaternion method). ``bumpy_sphere`` is this suite's own variant.
"""

from __future__ import annotations

import functools

import numpy as np
from scipy.spatial import ConvexHull, Delaunay

from ordito_b200 import creation


@functools.cache
def saddle_graded(resolution: int = 34, exponent: float = 3.4) -> tuple[np.ndarray, np.ndarray]:
    k = resolution
    step = np.linspace(-1.0, 1.0, k)
    u, v = np.meshgrid(np.sign(step) * np.abs(step) ** exponent, step, indexing="ij")
    vertices = np.column_stack((u.ravel(), v.ravel(), 0.35 * (u * u - 0.6 * v * v).ravel()))
    i, j = np.meshgrid(np.arange(k - 1), np.arange(k - 1), indexing="ij")
    corner = (i * k + j).ravel()
    faces = np.vstack(
        (
            np.column_stack((corner, corner + k, corner + k + 1)),
            np.column_stack((corner, corner + k + 1, corner + 1)),
        )
    )
    return vertices.astype(np.float32), faces.astype(np.int32)


@functools.cache
def bumpy_sphere(n: int = 500, seed: int = 5) -> tuple[np.ndarray, np.ndarray]:
    """Convex hull of random directions (a Delaunay sphere), squeezed in longitude and pushed out
    to a bumpy radius; vertex order and face starting corners shuffled."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    hull = ConvexHull(d)
    faces = hull.simplices.copy()
    # Orient outward.
    centers = d[faces].mean(axis=1)
    normals = np.cross(d[faces[:, 1]] - d[faces[:, 0]], d[faces[:, 2]] - d[faces[:, 0]])
    flip = np.einsum("ij,ij->i", normals, centers) < 0
    faces[flip] = faces[flip][:, ::-1]
    theta = np.arccos(np.clip(d[:, 2], -1, 1))
    phi = np.arctan2(d[:, 1], d[:, 0])
    phi = phi - 0.97 * np.sin(phi)
    radius = 1.0 + 0.35 * np.sin(3 * theta) * np.cos(2 * phi) + 0.15 * np.cos(5 * theta)
    vertices = np.column_stack(
        (radius * np.sin(theta) * np.cos(phi), radius * np.sin(theta) * np.sin(phi),
         radius * np.cos(theta))
    )
    perm = rng.permutation(n)
    inverse = np.empty(n, dtype=np.int64)
    inverse[perm] = np.arange(n)
    vertices = vertices[perm]
    faces = inverse[faces]
    faces = np.roll(faces, rng.integers(0, 3), axis=1)[rng.permutation(faces.shape[0])]
    return vertices.astype(np.float32), faces.astype(np.int32)


def _uniform_rotation(u: np.ndarray) -> np.ndarray:
    """The rotation of the unit quaternion Shoemake's method draws from three uniform numbers
    (K. Shoemake, "Uniform random rotations", Graphics Gems III, 1992): components
    (w, x, y, z) = (sqrt(u0) cos 2 pi u2, sqrt(1 - u0) sin 2 pi u1, sqrt(1 - u0) cos 2 pi u1,
    sqrt(u0) sin 2 pi u2), turned into its 3 x 3 matrix."""
    a, b = np.sqrt(1.0 - u[0]), np.sqrt(u[0])
    w, x, y, z = b * np.cos(2 * np.pi * u[2]), a * np.sin(2 * np.pi * u[1]), a * np.cos(2 * np.pi * u[1]), \
        b * np.sin(2 * np.pi * u[2])
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _scramble(vertices: np.ndarray, faces: np.ndarray, rng: np.random.Generator) -> tuple[np.ndarray, np.ndarray]:
    """Shuffle vertex and face order, rotate each face's corners, place the mesh off-axis (scaled
    1.7, a uniform random rotation, shifted by (0.3, -2.1, 1.4)), rounded to float32."""
    order = rng.permutation(vertices.shape[0])
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    faces = rank[faces][rng.permutation(faces.shape[0])]
    shift = rng.integers(0, 3, faces.shape[0])
    faces = np.take_along_axis(faces, (np.arange(3)[None, :] + shift[:, None]) % 3, axis=1)
    vertices = vertices[order]
    rotation = _uniform_rotation(rng.random(3))
    vertices = 1.7 * vertices @ rotation.T + np.array([0.3, -2.1, 1.4])
    return vertices.astype(np.float32), faces.astype(np.int32)


def _hull_sphere(rng: np.random.Generator, n_points: int, squeeze: float) -> tuple[np.ndarray, np.ndarray]:
    """The hull of random directions, wound outward, pushed to radius 1 + 0.35 sin 3 theta cos 2 phi
    + 0.15 cos 5 theta with the longitude squeezed by phi - squeeze sin phi."""
    directions = rng.normal(size=(n_points, 3))
    directions /= np.linalg.norm(directions, axis=1)[:, None]
    faces = ConvexHull(directions).simplices
    corners = directions[faces]
    normals = np.cross(corners[:, 1] - corners[:, 0], corners[:, 2] - corners[:, 0])
    inward = np.einsum("ij,ij->i", normals, corners.mean(axis=1)) < 0.0
    faces[inward] = faces[inward][:, [0, 2, 1]]
    theta = np.arccos(np.clip(directions[:, 2], -1.0, 1.0))
    phi = np.arctan2(directions[:, 1], directions[:, 0])
    phi = phi - squeeze * np.sin(phi)
    radius = 1.0 + 0.35 * np.sin(3.0 * theta) * np.cos(2.0 * phi) + 0.15 * np.cos(5.0 * theta)
    vertices = radius[:, None] * np.column_stack(
        (np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)))
    return vertices, faces


def _periodic_delaunay(uv: np.ndarray, period: tuple[float, float]) -> np.ndarray:
    """Delaunay triangulation of points on a flat torus: the 3 x 3 tiling's triangles whose
    centroid lies in the central tile, indices taken modulo the point count."""
    n = uv.shape[0]
    shifts = [(i * period[0], j * period[1]) for i in (-1, 0, 1) for j in (-1, 0, 1)]
    tiled = np.vstack([uv + np.array(shift) for shift in shifts])
    faces = Delaunay(tiled).simplices
    centroids = tiled[faces].mean(axis=1)
    central = ((centroids[:, 0] >= 0.0) & (centroids[:, 0] < period[0]) & (centroids[:, 1] >= 0.0)
               & (centroids[:, 1] < period[1]))
    return faces[central] % n


@functools.cache
def sphere_irregular() -> tuple[np.ndarray, np.ndarray]:
    """ordito's ``sphere_irregular`` (tests/conftest.py:624): 500 directions, squeeze 0.97, seed 5;
    vertex degree 3-12, needles up to aspect ~300, three quarters of the faces obtuse."""
    rng = np.random.default_rng(5)
    vertices, faces = _hull_sphere(rng, 500, 0.97)
    return _scramble(vertices, faces, rng)


@functools.cache
def torus_irregular() -> tuple[np.ndarray, np.ndarray]:
    """ordito's ``torus_irregular`` (tests/conftest.py:981): 500 random points (seed 7) on the flat
    torus of radii 1 and 0.45, Delaunay in the periodic domain, mapped onto a bumpy torus with the
    angle u squeezed by u - 0.97 sin u (needles up to aspect ~540)."""
    rng = np.random.default_rng(7)
    major, minor = 1.0, 0.45
    period = (2.0 * np.pi * major, 2.0 * np.pi * minor)
    uv = rng.random((500, 2)) * np.array(period)
    faces = _periodic_delaunay(uv, period)
    u = uv[:, 0] / major
    v = uv[:, 1] / minor
    u = u - 0.97 * np.sin(u)
    radius = minor * (1.0 + 0.25 * np.sin(3.0 * u) * np.cos(2.0 * v))
    ring = major + radius * np.cos(v)
    vertices = np.column_stack((ring * np.cos(u), ring * np.sin(u), radius * np.sin(v)))
    return _scramble(vertices, faces, rng)


def small_torus(cols: int = 48, rows: int = 24, seed: int = 3) -> tuple[np.ndarray, np.ndarray]:
    return creation.jittered_torus(cols, rows, 1.0, 0.3, 0.1, seed)


def with_unreferenced_vertex() -> tuple[np.ndarray, np.ndarray]:
    """icosphere(2) plus one vertex no face references (its row stays empty)."""
    v, f = creation.icosphere(2)
    v = np.vstack((v, [[3.0, 0.0, 0.0]])).astype(np.float32)
    return v, f


def with_degenerate_face() -> tuple[np.ndarray, np.ndarray]:
    """icosphere(1) plus a zero-area face with a repeated vertex (self-edge keys)."""
    v, f = creation.icosphere(1)
    f = np.vstack((f, [[0, 0, 1]])).astype(np.int32)
    return v, f


ALL = {
    "ico3": lambda: creation.icosphere(3),
    "saddle_graded": saddle_graded,
    "bumpy_sphere": bumpy_sphere,
    "sphere_irregular": sphere_irregular,
    "torus_irregular": torus_irregular,
    "small_torus": small_torus,
    "grid": lambda: creation.grid((5, 4)),
    "unreferenced": with_unreferenced_vertex,
    "degenerate": with_degenerate_face,
}
