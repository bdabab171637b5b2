"""Cotangent Laplacian, lumped mass and the operator pattern (``ordito.laplacian``'s path subset).

Signatures follow ordito/laplacian.py: ``mesh_operator_pattern`` (:1071), ``cotmatrix_entries``
(:189), ``cotmatrix`` (:371) and ``mass_matrix_entries`` (:1930). Arrays in are device arrays
(``__cuda_array_interface__``) or host NumPy arrays; arrays out are ``DeviceArray``. Every value
is computed by the CUDA kernels of ``libordito_b200.so``.
"""

from __future__ import annotations

import ctypes
from typing import Any, NamedTuple

import numpy as np

from ordito_b200 import _lib
from ordito_b200.array import CsrMatrix
from ordito_b200.device import DEFAULT_STREAM, DeviceArray, as_device, element_count


class MeshOperatorPattern(NamedTuple):
    """The sparsity of a vertex operator on one face buffer, with each entry's contributing corners.

    Fields as ordito/laplacian.py:1022-1068: ``offsets`` (``n_vertices + 1``), ``columns`` and
    ``run_start`` (capacity ``n_keys``, ``offsets[-1]`` used), the sorted ``keys`` and their corner
    payloads ``order`` (``3 f + e``; -1 for a diagonal slot).
    """

    operator: str
    n_vertices: int
    offsets: DeviceArray
    columns: DeviceArray
    run_start: DeviceArray
    keys: DeviceArray
    n_keys: int
    order: DeviceArray


def mesh_arrays(vertices: Any, faces: Any) -> tuple[DeviceArray, DeviceArray, int, int]:
    """``(xyz float32 (V, 3), faces int32 (3F,), V, F)`` on the device, validating shapes."""
    xyz = as_device(vertices, np.float32)
    if xyz.size % 3:
        raise ValueError(f"vertices must hold (n_vertices, 3) float32 positions, got {xyz.shape}")
    tri = as_device(faces, np.int32)
    if tri.size % 3:
        raise ValueError(f"faces must hold 3 * n_faces indices, got {tri.shape}")
    return xyz, tri, xyz.size // 3, tri.size // 3


def mesh_operator_pattern(
    faces: Any, n_vertices: int, *, operator: str = "cotmatrix"
) -> MeshOperatorPattern:
    """Sparsity of the cotangent operator on ``faces``: every edge both ways plus the diagonal of
    every referenced vertex (an unreferenced vertex keeps an empty row).

    Raises ``ValueError`` for an unknown ``operator``; the ``"laplacian_*"`` patterns serve
    operators outside the heat-geodesic path and are not built here.
    """
    if operator not in ("cotmatrix", "laplacian_symmetric", "laplacian_directed"):
        raise ValueError(
            "operator must be one of ['cotmatrix', 'laplacian_symmetric', 'laplacian_directed'], "
            f"got {operator!r}"
        )
    if operator != "cotmatrix":
        raise NotImplementedError(f"the {operator!r} pattern is not part of the heat-geodesic path")
    tri = as_device(faces, np.int32)
    n_faces = tri.size // 3
    n_vertices = int(n_vertices)
    count = 6 * n_faces + n_vertices
    offsets = DeviceArray.empty(n_vertices + 1, np.int32)
    columns = DeviceArray.empty(count, np.int32)
    run_start = DeviceArray.empty(count, np.int32)
    keys = DeviceArray.empty(count, np.uint64)
    order = DeviceArray.empty(count, np.int32)
    nbytes = ctypes.c_size_t(0)
    _lib.call("ob_pattern_workspace", n_vertices, n_faces, ctypes.byref(nbytes))
    workspace = DeviceArray.empty(int(nbytes.value), np.uint8)
    _lib.call(
        "ob_pattern_build", tri.ptr, n_faces, n_vertices, offsets.ptr, columns.ptr, run_start.ptr,
        keys.ptr, order.ptr, workspace.ptr, int(nbytes.value), DEFAULT_STREAM,
    )  # fmt: skip
    return MeshOperatorPattern("cotmatrix", n_vertices, offsets, columns, run_start, keys, count, order)


class FaceTerms(NamedTuple):
    cot: DeviceArray  # (F, 3) float32
    normals: DeviceArray  # (F, 3) float32
    areas: DeviceArray  # (F,) float32
    area_sums: DeviceArray  # (V,) float64


def face_terms(xyz: DeviceArray, tri: DeviceArray, n_vertices: int, n_faces: int,
               cot_entries: Any = None) -> FaceTerms:
    """One pass over the faces (ordito/kernels/heat.py:92 heat_face_terms)."""
    write_cot = cot_entries is None
    cot = DeviceArray.empty((n_faces, 3), np.float32) if write_cot else as_device(cot_entries, np.float32)
    if not write_cot and cot.size != 3 * n_faces:
        raise ValueError(f"cot_entries must have shape (n_faces, 3) = ({n_faces}, 3), got {cot.shape}")
    normals = DeviceArray.empty((n_faces, 3), np.float32)
    areas = DeviceArray.empty(n_faces, np.float32)
    area_sums = DeviceArray.empty(n_vertices, np.float64)
    _lib.call(
        "ob_face_terms", xyz.ptr, tri.ptr, n_faces, n_vertices, cot.ptr if write_cot else None,
        normals.ptr, areas.ptr, area_sums.ptr, DEFAULT_STREAM,
    )  # fmt: skip
    return FaceTerms(cot, normals, areas, area_sums)


def cotmatrix_entries(vertices: Any, faces: Any, dtype: Any = np.float32, *,
                      nonnegative_weights: bool = False) -> DeviceArray:
    """``(n_faces, 3)`` half-cotangent weights, column ``e`` for the edge opposite corner ``e``.

    Computed in float32 (the vertex precision) as ordito/laplacian.py:189 does; ``dtype`` float64
    widens the float32 values. ``nonnegative_weights`` clamps an obtuse angle's negative weight to
    zero (kernels/laplacian.py:146-163).
    """
    xyz, tri, n_vertices, n_faces = mesh_arrays(vertices, faces)
    terms = face_terms(xyz, tri, n_vertices, n_faces)
    if nonnegative_weights:
        _lib.call("ob_floor_f32", terms.cot.ptr, terms.cot.size, 0.0, DEFAULT_STREAM)
    return cast(terms.cot, dtype)


def mass_matrix_entries(vertices: Any, faces: Any, dtype: Any = np.float32) -> DeviceArray:
    """Barycentric lumped mass: a third of each vertex's faces' float32 areas, summed exactly in
    float64 (ordito/laplacian.py:1930, kernels/scatter.py:860)."""
    xyz, tri, n_vertices, n_faces = mesh_arrays(vertices, faces)
    terms = face_terms(xyz, tri, n_vertices, n_faces)
    return cast(terms.area_sums, dtype, 1.0 / 3.0)


class Assembled(NamedTuple):
    laplacian: CsrMatrix
    heat: CsrMatrix
    poisson: CsrMatrix
    mass: DeviceArray
    edge_sums: DeviceArray | None


def assemble_rows(
    pattern: MeshOperatorPattern,
    xyz: DeviceArray,
    cot: DeviceArray,
    area_sums: DeviceArray,
    *,
    t: float | None,
    face_edges: bool,
    mass_divisor: float = 3.0,
) -> Assembled:
    """``L``, ``M - t L`` and ``-L`` over the pattern plus the lumped mass (kernels/heat.py:361).

    With ``t`` None the time step is the device-formed ``h ** 2`` from the pattern's edge sums
    (``face_edges`` weighs each edge by the faces holding it: MeshLab's mean over every face's
    three edges; otherwise the unique-edge mean).
    """
    n = pattern.n_vertices
    capacity = max(pattern.n_keys, 1)
    values = DeviceArray.empty(3 * capacity, np.float64)
    L = values.view(0, capacity)
    H = values.view(capacity, 2 * capacity)
    P = values.view(2 * capacity, 3 * capacity)
    mass = DeviceArray.empty(n, np.float64)
    edge_sums = None
    if t is None:
        edge_sums = DeviceArray.empty(2, np.float64)
        _lib.call(
            "ob_edge_sums", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
            pattern.keys.ptr, pattern.n_keys, n, xyz.ptr, int(face_edges), edge_sums.ptr,
            DEFAULT_STREAM,
        )  # fmt: skip
    _lib.call(
        "ob_heat_rows", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
        pattern.keys.ptr, pattern.n_keys, pattern.order.ptr, n, cot.ptr,
        -1.0 if t is None else -float(t), edge_sums.ptr if edge_sums is not None else None,
        1 if t is None else 0, area_sums.ptr, float(mass_divisor), L.ptr, H.ptr, P.ptr, mass.ptr,
        DEFAULT_STREAM,
    )  # fmt: skip
    laplacian = CsrMatrix(n, n, pattern.offsets, pattern.columns, L)
    return Assembled(laplacian, laplacian.with_values(H), laplacian.with_values(P), mass, edge_sums)


def cotmatrix(
    vertices: Any,
    faces: Any,
    cot_entries: Any = None,
    dtype: Any = np.float32,
    *,
    pattern: MeshOperatorPattern | None = None,
    nonnegative_weights: bool = False,
) -> CsrMatrix:
    """The cotangent stiffness ``L`` (igl sign convention: negative diagonal).

    ordito/laplacian.py:371; off-diagonal ``L_ij`` sums the entry's half-cotangents in face order,
    the diagonal is minus the row's off-diagonal sum. The weights are the float32 half-cotangent
    table (or ``cot_entries``); the rows are summed in float64, and ``dtype`` float32 (the
    reference's default) rounds those float64 sums once (the reference sums in float32: the two
    agree within float32 rounding). ``nonnegative_weights`` assembles from the weights clamped at
    zero (only for weights computed here).
    """
    dtype = np.dtype(dtype)
    if dtype not in (np.dtype(np.float32), np.dtype(np.float64)):
        raise ValueError(f"cotmatrix: dtype must be float32 or float64, got {dtype}")
    if nonnegative_weights and cot_entries is not None:
        raise ValueError(
            "cotmatrix: nonnegative_weights clamps the weights it computes; pass cot_entries from "
            "cotmatrix_entries(..., nonnegative_weights=True) instead"
        )
    xyz, tri, n_vertices, n_faces = mesh_arrays(vertices, faces)
    if pattern is None:
        pattern = mesh_operator_pattern(tri, n_vertices)
    elif pattern.n_vertices != n_vertices or pattern.operator != "cotmatrix":
        raise ValueError("pattern was built for another operator or vertex count")
    terms = face_terms(xyz, tri, n_vertices, n_faces, cot_entries)
    if nonnegative_weights:
        _lib.call("ob_floor_f32", terms.cot.ptr, terms.cot.size, 0.0, DEFAULT_STREAM)
    laplacian = assemble_rows(pattern, xyz, terms.cot, terms.area_sums, t=0.0, face_edges=False).laplacian
    if dtype == np.float64:
        return laplacian
    return laplacian.with_values(cast(laplacian.values, dtype))


def cast(array: DeviceArray, dtype: Any, scale: float = 1.0) -> DeviceArray:
    """``array * scale`` as ``dtype`` (float32 or float64), formed on the device."""
    dtype = np.dtype(dtype)
    if dtype == array.dtype and scale == 1.0:
        return array
    codes = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}
    if dtype not in codes or array.dtype not in codes:
        raise ValueError(f"dtype must be float32 or float64, got {dtype}")
    out = DeviceArray.empty(array.shape, dtype)
    _lib.call("ob_cast_scale", array.ptr, codes[array.dtype], out.ptr, codes[dtype], array.size,
              float(scale), DEFAULT_STREAM)
    return out


def faces_count(faces: Any) -> int:
    return element_count(faces) // 3
