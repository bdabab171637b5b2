"""Test meshes: small generated fixtures with the properties the reference's tests rely on.

``saddle_graded`` restates ordito's fixture (tests/conftest.py:471-502: a k x k grid on the saddle
z = 0.35 (x^2 - 0.6 y^2), x spacing graded as |t|^e). ``bumpy_sphere`` and ``irregular_torus``
are this suite's own irregular closed meshes (random Delaunay sampling, needles and obtuse faces)
in the spirit of the reference's ``sphere_irregular`` / ``torus_irregular``.
"""

from __future__ import annotations

import functools

import numpy as np
from scipy.spatial import ConvexHull

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
    "small_torus": small_torus,
    "grid": lambda: creation.grid((5, 4)),
    "unreferenced": with_unreferenced_vertex,
    "degenerate": with_degenerate_face,
}
