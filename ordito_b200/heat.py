"""The heat-method geodesic distance (Crane et al.), ``ordito.heat``'s path subset.

``heat_geodesic`` (ordito/heat.py:391), ``heat_operators`` (:200) and ``HeatSolver`` (:3491) with
the reference's signatures, defaults and errors. A query is: seed the source indicator, diffuse it
by the heat system ``M - t L`` (Jacobi CG to settled entries, or the held Cholesky factor),
integrate the face-wise unit gradient's divergence, solve the Poisson system ``-L`` (Chebyshev-
preconditioned CG to relative residual 1e-8, or the held factor), and shift to the sources. Every
step is a CUDA kernel of ``libordito_b200.so``; the host only reads back the documented scalars
(an invalid-source flag, solver counts, and -- once per solver -- the mean edge length and bounds).
"""

from __future__ import annotations

import contextlib
import ctypes
import gc
import logging
import math
import warnings
from typing import Any, NamedTuple

import numpy as np

from ordito_b200 import _lib
from ordito_b200 import linalg as twl
from ordito_b200.array import CsrMatrix
from ordito_b200.device import DEFAULT_STREAM, DeviceArray, as_device, device_pointer
from ordito_b200.laplacian import (
    MeshOperatorPattern,
    assemble_rows,
    face_terms,
    mesh_arrays,
    mesh_operator_pattern,
)
from ordito_b200.mesh import Trimesh, mesh_arguments

_LOGGER = logging.getLogger(__name__)

_CG_TOLERANCE = 1e-8  # ordito/heat.py:108
# The relative residual the mixed-precision multigrid Poisson solve of the batched path reaches.
_MULTIGRID_POISSON_TOLERANCE = 1e-10
_HEAT_CHECK_ROUNDS = 16  # :142
_HEAT_CHANGE_TOLERANCE = 1e-6  # :146
_HEAT_SETTLE_ROUNDS = 192  # :147
_DIFFUSION_DECAY = 400.0  # :158
_GEOMETRY_CENTRAL_POISSON_SHIFT = 1e-6  # :193 (geometry-central's Poisson system -L + 1e-6 I)
_TOLERANCE_MOLLIFY = 1e-5  # ordito/constants.py:31 (use_robust's margin, of the mean edge length)


class HeatOperators(NamedTuple):
    """What ``heat_operators`` returns (ordito/heat.py:169-178)."""

    heat_system: CsrMatrix
    heat_preconditioner: twl.Preconditioner
    laplacian: CsrMatrix
    poisson_system: CsrMatrix
    poisson_preconditioner: twl.Preconditioner
    cot_entries: DeviceArray
    face_normals: DeviceArray
    face_areas: DeviceArray


def _heat_method_choices(method: str) -> tuple[str, str]:
    """``(mass, timestep)`` of a discretization (ordito/heat.py:2002-2012)."""
    if method == "potpourri3d":
        return "barycentric", "unique_edges"
    if method == "meshlab":
        return "barycentric", "face_edges"
    if method == "igl":
        return "voronoi", "unique_edges"
    raise ValueError(f"method must be 'potpourri3d', 'meshlab' or 'igl', got {method!r}")


def _supported(method: str, use_robust: bool) -> None:
    _heat_method_choices(method)


def _robust_cot(mesh: Trimesh) -> DeviceArray:
    """The use_robust half-cotangent table: the law of cosines over the face side lengths with one
    constant added to every length so that no triangle is degenerate (ordito/laplacian.py:779,
    :276; heat.py:2043-2056). The mass, normals and areas stay the positions' own."""
    lengths = DeviceArray.empty((max(mesh.n_faces, 1), 3), np.float32)
    cot = DeviceArray.empty((max(mesh.n_faces, 1), 3), np.float32)
    delta = ctypes.c_double(0.0)
    _lib.call("ob_mollified_cot", mesh.vertices.ptr, mesh.faces.ptr, mesh.n_faces, _TOLERANCE_MOLLIFY,
              lengths.ptr, cot.ptr, ctypes.byref(delta), DEFAULT_STREAM)
    return cot if mesh.n_faces else DeviceArray.empty((0, 3), np.float32)


def _assemble(mesh: Trimesh, t: float | None, method: str, cot_entries: Any = None,
              pattern: MeshOperatorPattern | None = None,
              use_robust: bool = False) -> tuple[HeatOperators, Any]:
    mass, timestep = _heat_method_choices(method)
    if use_robust:
        cot_entries = _robust_cot(mesh)
    if pattern is None:
        pattern = mesh.mesh_operator_pattern
    elif pattern.n_vertices != mesh.n_vertices or pattern.operator != "cotmatrix":
        raise ValueError("pattern was built for another operator or vertex count")
    if cot_entries is None:
        terms = mesh.face_terms
    else:
        terms = face_terms(mesh.vertices, mesh.faces, mesh.n_vertices, mesh.n_faces, cot_entries)
    area_sums, mass_divisor = terms.area_sums, 3.0
    if mass == "voronoi":
        # ``method="igl"``: each corner's Voronoi share, the lumped mass itself (heat.py:2116,2169).
        area_sums = DeviceArray.empty(mesh.n_vertices, np.float64)
        _lib.call("ob_voronoi_area_sums", mesh.vertices.ptr, mesh.faces.ptr, mesh.n_faces,
                  mesh.n_vertices, area_sums.ptr, DEFAULT_STREAM)
        mass_divisor = 1.0
    built = assemble_rows(
        pattern, mesh.vertices, terms.cot, area_sums, t=t, face_edges=timestep == "face_edges",
        mass_divisor=mass_divisor,
    )
    operators = HeatOperators(
        built.heat,
        twl.jacobi_preconditioner(built.heat),
        built.laplacian,
        built.poisson,
        twl.chebyshev_preconditioner(built.poisson),
        terms.cot,
        terms.normals,
        terms.areas,
    )
    return operators, built


def heat_operators(
    vertices: Any,
    faces: Any,
    t: float | None = None,
    *,
    use_robust: bool = False,
    cot_entries: Any = None,
    pattern: MeshOperatorPattern | None = None,
    method: str = "potpourri3d",
) -> HeatOperators:
    """Assemble the source-independent operators the heat method solves against.

    ``t`` None takes ``h ** 2`` formed on the device, ``h`` the mean edge length ``method`` names
    (unique edges for ``"potpourri3d"`` and ``"igl"``, every face's three edges for ``"meshlab"``);
    ``"igl"`` lumps the mass by Voronoi areas, the others barycentrically (ordito/heat.py:2002-2012).
    """
    if cot_entries is not None and use_robust:
        raise ValueError(
            "cot_entries and use_robust are mutually exclusive: use_robust rebuilds the "
            "half-cotangent table from mollified edge lengths."
        )
    _supported(method, use_robust)
    mesh = Trimesh(vertices, faces)
    return _assemble(mesh, t, method, cot_entries, pattern, use_robust)[0]


def _diffusion_floor(mesh: Trimesh) -> float:
    """``(|bounding-box diagonal| / 400) ** 2`` (ordito/heat.py:5228)."""
    low, high = mesh.bounds
    return (math.dist(low, high) / _DIFFUSION_DECAY) ** 2


def _bounds_floor_length(low: np.ndarray, high: np.ndarray) -> float:
    """``|bounding-box diagonal| / 400`` of a box's float32 corners: the square root of the floor
    above (the float32 extremes widened to float64, exactly as the device's bounds)."""
    return math.dist(low.astype(np.float64), high.astype(np.float64)) / _DIFFUSION_DECAY


def _settle_window(t: float | None, default: float) -> int:
    """ordito/heat.py:5234: the settle window grows like ``sqrt(t / h^2)``."""
    if t is None or not t > default > 0.0:
        return _HEAT_SETTLE_ROUNDS
    return math.ceil(_HEAT_SETTLE_ROUNDS * math.sqrt(t / default))


class HeatSolver:
    """A mesh's heat-method state for one ``(t, use_robust, method)`` (ordito/heat.py:3491).

    Holds the operators, the native solver states, and -- on a system's second solve (rent or
    buy, ordito/heat.py:4394) or when a settled iterate fails its check -- its sparse Cholesky
    factorization, which later solves go through directly.
    """

    def __init__(self, mesh: Trimesh, t: float | None = None, *, use_robust: bool = False,
                 method: str = "potpourri3d") -> None:
        _supported(method, use_robust)
        self._mesh = mesh
        self.t = t
        self.use_robust = use_robust
        self.method = method
        self._operators: HeatOperators | None = None
        self._cover = None  # the intrinsic tufted cover (use_robust at method="potpourri3d")
        self._resolved: tuple[float | None, int] | None = None
        self._systems: dict[str, Any] = {}
        self._ill_conditioned = False
        self._unfactorable = False
        self.factor_on_second_solve = True

    # -- time and operators ------------------------------------------------------------------
    def _vertex_time(self) -> tuple[float | None, int]:
        """The time the systems are built at (``None``: the device's ``h ** 2``) and the settle
        window (ordito/heat.py:3714-3736)."""
        if self._resolved is None:
            t = self.t
            mesh = self._mesh
            if self.method == "meshlab":
                mean = mesh.mean_edge_length
            else:
                mean = self._unique_mean_edge_length()
            default = mean**2
            if t is None:
                floor = _diffusion_floor(mesh)
                t = floor if floor > default else None
            self._resolved = (t, _settle_window(t, default))
        return self._resolved

    def _unique_mean_edge_length(self) -> float:
        mesh = self._mesh
        pattern = mesh.mesh_operator_pattern
        sums = DeviceArray.empty(2, np.float64)
        _lib.call(
            "ob_edge_sums", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
            pattern.keys.ptr, pattern.n_keys, mesh.n_vertices, mesh.vertices.ptr, 0, sums.ptr,
            DEFAULT_STREAM,
        )  # fmt: skip
        total, count = sums.numpy()
        return float(total / count) if count > 0 else 0.0

    @property
    def operators(self) -> HeatOperators:
        """``heat_operators`` for the mesh at ``t``; at ``method="potpourri3d"`` with
        ``use_robust``, the same systems on the mesh's intrinsic tufted cover (ordito/heat.py:3651-
        3663), whose per-face tables are empty: the cover's faces are not the mesh's."""
        if self._operators is None:
            t, _ = self._vertex_time()
            if self.use_robust and self.method == "potpourri3d":
                self._operators, self._built = self._cover_operators(t)
            else:
                self._operators, self._built = _assemble(self._mesh, t, self.method,
                                                         use_robust=self.use_robust)
        return self._operators

    @property
    def cover(self) -> Any:
        """The intrinsic tufted cover the operators are built on (``None`` unless ``use_robust``
        at ``method="potpourri3d"``)."""
        if self.use_robust and self.method == "potpourri3d":
            self.operators  # noqa: B018 -- builds the cover with the operators
            return self._cover
        return None

    def _cover_operators(self, t: float | None) -> tuple[HeatOperators, Any]:
        """geometry-central's ``HeatMethodDistanceSolver`` with ``useRobustLaplacian``
        (ordito/heat.py:3749-3830): the mass, the Laplacian and the default time's mean edge all
        from the cover's flipped float64 lengths."""
        from ordito_b200 import cover as gcover  # noqa: PLC0415

        self._cover, area_sums, edge_sums = gcover.build_cover(self._mesh)
        built = gcover.cover_rows(self._mesh, self._cover, area_sums, edge_sums, t)
        empty32 = DeviceArray.empty((0, 3), np.float32)
        operators = HeatOperators(
            built.heat,
            twl.jacobi_preconditioner(built.heat),
            built.laplacian,
            built.poisson,
            twl.chebyshev_preconditioner(built.poisson),
            empty32,
            empty32,
            DeviceArray.empty(0, np.float32),
        )
        return operators, built

    # -- the vector heat method (ordito/heat.py:3677, 3952-4060) -------------------------------
    def _require_vector_discretization(self, what: str) -> None:
        """The vector heat method is defined on the potpourri3d discretization (heat.py:4443)."""
        if self.use_robust:
            raise ValueError(f"HeatSolver: no use_robust variant of {what}")
        if self.method != "potpourri3d":
            raise ValueError(f"HeatSolver: no method={self.method!r} variant of {what}")

    @property
    def vector_operators(self) -> "VectorHeatOperators":
        """``vector_heat_operators`` for the mesh at this solver's ``t`` (ordito/heat.py:3677): its
        scalar bundle is ``operators``, one assembly."""
        self._require_vector_discretization("the vector heat operators")
        if getattr(self, "_vector_operators", None) is None:
            operators = self.operators
            mesh = self._mesh
            t, _ = self._vertex_time()
            system = _vector_system(mesh, mesh.mesh_operator_pattern, mesh.halfedge_transport[1],
                                    self._built.mass, t, self._built.edge_sums)
            self._vector_operators = VectorHeatOperators(system, operators, mesh.vertex_tangent_frames,
                                                         twl.jacobi_preconditioner(system))
        return self._vector_operators

    def diffuse_tangent(self, rhs: Any, solution: Any) -> None:
        """Solve the vector heat system ``(M + t L_connection) X = rhs`` to settled entries, in place:
        ``rhs`` and ``solution`` hold ``2 V`` rows (vertex v's tangent components in rows ``2v`` and
        ``2v + 1``), one column or several row-interleaved (ordito/heat.py:3952-4060). Factored on
        its second solve, as the heat system is; past the budget the band march answers."""
        system = self.vector_operators.vector_system
        kept = self._kept("vector")
        twl.solve_spd_settled(
            system,
            rhs,
            solution,
            check_rounds=_HEAT_CHECK_ROUNDS,
            change_tolerance=_HEAT_CHANGE_TOLERANCE,
            settle_rounds=self._vertex_time()[1],
            factorization=kept["factorization"],
            narrow_values=True,
        )

    # -- solves --------------------------------------------------------------------------------
    def _system(self, role: str) -> Any:
        from ordito_b200.cholesky import OperatorFactorization  # noqa: PLC0415

        kept = self._systems.get(role)
        if kept is None:
            matrix = {
                "heat": lambda: self.operators.heat_system,
                "poisson": lambda: self.operators.poisson_system,
                "pinned": lambda: self._pinned_system()[0],
                "poisson_regularized": lambda: self._regularized_system()[0],
                "vector": lambda: self.vector_operators.vector_system,
            }[role]()
            kept = self._systems[role] = {
                # The vector system's two tangent rows a vertex are analysed as one (block 2).
                "factorization": OperatorFactorization(
                    matrix, self._mesh.vertices, singular=role == "poisson",
                    block=2 if role == "vector" else 1,
                ),
                "solves": 0,
            }
        return kept

    def _kept(self, role: str) -> Any:
        """Count a solve of ``role``'s system, factoring it on its second (rent or buy)."""
        kept = self._system(role)
        kept["solves"] += 1
        factorization = kept["factorization"]
        if (self.factor_on_second_solve and kept["solves"] >= 2
                and factorization.factorization is None and not factorization.refused):
            if factorization.factor(self._sharing(role)):
                _LOGGER.debug("HeatSolver: factored the %s system on its second solve", role)
        return kept

    def _sharing(self, role: str) -> Any:
        # Every other scalar system is stored over the heat system's pattern: its analysis serves
        # them (the vector system's expanded pattern has an analysis of its own).
        heat = self._systems.get("heat")
        return heat["factorization"] if role not in ("heat", "vector") and heat is not None else None

    def _pinned_system(self) -> tuple[Any, DeviceArray] | tuple[()]:
        """``diffuse_pinned``'s system and rim mask, built on first use; ``()`` with no rim
        (ordito/heat.py:4200-4233)."""
        if getattr(self, "_pinned", None) is None:
            mesh, heat = self._mesh, self.operators.heat_system
            pattern = mesh.mesh_operator_pattern
            rim = DeviceArray.empty(max(mesh.n_vertices, 1), np.int32)
            n_rim = DeviceArray.empty(1, np.int32)
            _lib.call("ob_rim_vertices", pattern.offsets.ptr, pattern.columns.ptr,
                      pattern.run_start.ptr, pattern.keys.ptr, pattern.n_keys, mesh.n_vertices,
                      rim.ptr, n_rim.ptr, DEFAULT_STREAM)
            # One read-back per solver: a closed mesh has no rim and so no second solve.
            if int(n_rim.numpy()[0]) == 0:
                self._pinned = ()
            else:
                values = DeviceArray.empty(max(heat.nnz, 1), np.float64)
                _lib.call("ob_pinned_rows", heat.offsets.ptr, heat.columns.ptr, rim.ptr,
                          heat.values.ptr, mesh.n_vertices, values.ptr, DEFAULT_STREAM)
                self._pinned = (heat.with_values(values), rim)
        return self._pinned

    def _regularized_system(self) -> tuple[Any, Any]:
        """geometry-central's Poisson system ``-L + 1e-6 I`` and its Chebyshev preconditioner,
        built over the Poisson operator's pattern on first use (ordito/heat.py:4086-4114)."""
        if getattr(self, "_regularized", None) is None:
            poisson = self.operators.poisson_system
            values = DeviceArray.empty(max(poisson.nnz, 1), np.float64)
            _lib.call("ob_add_to_diagonal", poisson.offsets.ptr, poisson.columns.ptr,
                      poisson.values.ptr, poisson.nrow, _GEOMETRY_CENTRAL_POISSON_SHIFT, values.ptr,
                      DEFAULT_STREAM)
            system = poisson.with_values(values)
            self._regularized = (system, twl.chebyshev_preconditioner(system))
        return self._regularized

    def factor(self, roles: tuple[str, ...] = ("heat", "poisson")) -> bool:
        """Factor both systems now (ordito/heat.py:3863); False if either could not be."""
        ok = True
        for role in roles:
            kept = self._system(role)
            if kept["factorization"].factorization is None:
                ok = kept["factorization"].factor(self._sharing(role)) and ok
        return ok

    def tune(self, k: int) -> dict:
        """Tune both factors' pass schedules for batches of ``k`` columns (``tuning.tune_pass``);
        factors them first if needed. Returns each system's tuning report."""
        from ordito_b200.tuning import tune_shared  # noqa: PLC0415

        if not self.factor():
            raise RuntimeError("HeatSolver.tune: the systems could not be factored (over budget)")
        # The two factors share the heat system's analysis: one search serves both (tune_shared).
        return tune_shared({"heat": self.heat_factor, "poisson": self.poisson_factor}, k)

    def single_query(self, sources: DeviceArray) -> DeviceArray:
        """Distances for one validated source set with both factors held (``_SingleQuery``)."""
        query = getattr(self, "_single_query", None)
        if query is None or sources.size > query.capacity:
            if query is not None:
                query.close()
            query = self._single_query = _SingleQuery(self._mesh, self, max(64, sources.size))
        return query(sources)

    @property
    def gradient_terms(self) -> DeviceArray:
        """The divergence's per-face terms ``[F][18]`` (``ob_face_gradient_terms``), built once."""
        if getattr(self, "_gradient_terms", None) is None:
            mesh, ops = self._mesh, self.operators
            terms = DeviceArray.empty((max(mesh.n_faces, 1), 18), np.float64)
            _lib.call("ob_face_gradient_terms", mesh.vertices.ptr, mesh.faces.ptr, mesh.n_faces,
                      ops.face_normals.ptr, ops.face_areas.ptr, ops.cot_entries.ptr, terms.ptr,
                      DEFAULT_STREAM)
            self._gradient_terms = terms
        return self._gradient_terms

    @property
    def poisson_multigrid(self) -> Any:
        """The Poisson system's smoothed-aggregation hierarchy, built on first use and kept."""
        if getattr(self, "_poisson_multigrid", None) is None:
            self._poisson_multigrid = twl.multigrid_preconditioner(self.operators.poisson_system)
        return self._poisson_multigrid

    def scratch_flag(self) -> DeviceArray:
        """A device int32 the batched seeding writes its (host-prevalidated) range flag into."""
        if getattr(self, "_flag", None) is None:
            self._flag = DeviceArray.empty(1, np.int32)
        return self._flag

    @property
    def heat_factor(self):
        """The heat system's held ``SparseCholesky`` (``None`` before ``factor``)."""
        return self._system("heat")["factorization"].factorization

    @property
    def poisson_factor(self):
        """The Poisson system's held ``SparseCholesky`` (``None`` before ``factor``)."""
        return self._system("poisson")["factorization"].factorization

    def diffuse(self, rhs: Any, solution: Any) -> None:
        """Solve the heat system ``(M - t L) u = rhs`` to settled entries, in place."""
        operators = self.operators
        kept = self._kept("heat")
        held = kept["factorization"].factorization is not None
        twl.solve_spd_settled(
            operators.heat_system,
            rhs,
            solution,
            check_rounds=_HEAT_CHECK_ROUNDS,
            change_tolerance=_HEAT_CHANGE_TOLERANCE,
            settle_rounds=self._vertex_time()[1],
            factorization=kept["factorization"],
            narrow_values=True,
        )
        # A rejected settled iterate (answered by the factor or, past the budget, the march)
        # marks the mesh ill-conditioned for its Poisson solve (ordito/heat.py:4394-4404).
        if not held and (kept["factorization"].factorization is not None
                         or getattr(kept["factorization"], "iterate_rejected", False)):
            self._ill_conditioned = True

    def diffuse_pinned(self, rhs: Any, solution: Any) -> bool:
        """Solve the heat system with the heat pinned to zero on the mesh's rim, in place
        (ordito/heat.py:4153-4198): ``(M - t L) u = rhs`` on the interior, ``u = 0`` on every
        vertex with an edge on a single face, settled as ``diffuse``. Returns whether the mesh has
        a rim (without one ``solution`` is left as it was)."""
        if self.method == "potpourri3d" and self.use_robust:
            raise ValueError(
                "HeatSolver.diffuse_pinned: no use_robust variant at method='potpourri3d', whose "
                "intrinsic cover has no rim"
            )
        pinned = self._pinned_system()
        if not pinned:
            return False
        system, rim = pinned
        n = self._mesh.n_vertices
        rhs_ptr, keep_rhs = device_pointer(rhs, np.float64)
        pinned_rhs = DeviceArray.empty(n, np.float64)
        _lib.call("ob_off_rim", rhs_ptr, rim.ptr, n, pinned_rhs.ptr, DEFAULT_STREAM)
        del keep_rhs
        kept = self._kept("pinned")
        twl.solve_spd_settled(
            system,
            pinned_rhs,
            solution,
            check_rounds=_HEAT_CHECK_ROUNDS,
            change_tolerance=_HEAT_CHANGE_TOLERANCE,
            settle_rounds=self._vertex_time()[1],
            factorization=kept["factorization"],
            narrow_values=True,
        )
        return True

    def solve_regularized_poisson(self, rhs: Any, solution: Any) -> None:
        """Solve geometry-central's ``(-L + 1e-6 I) phi = rhs``, warm-started from ``solution``, in
        place (ordito/heat.py:4086-4150): factored when the heat system is, else by CG under its
        Chebyshev polynomial."""
        system, preconditioner = self._regularized_system()
        kept = self._kept("poisson_regularized")
        factorization = kept["factorization"]
        heat = self._systems.get("heat")
        if (factorization.factorization is None and heat is not None
                and heat["factorization"].factorization is not None):
            factorization.factor(self._sharing("poisson_regularized"))
        if factorization.factorization is not None:
            factorization.solve(rhs, solution, tol=twl.SETTLE_DIRECT_TOLERANCE)
            return
        twl.solve_spd(system, rhs, solution, tol=_CG_TOLERANCE, preconditioner=preconditioner,
                      name="heat_geodesic")

    def solve_poisson(self, rhs: Any, solution: Any) -> None:
        """Solve ``(-L) phi = rhs`` (consistent), warm-started from ``solution``, in place."""
        operators = self.operators
        kept = self._kept("poisson")
        factorization = kept["factorization"]
        if factorization.factorization is None and self._ill_conditioned:
            factorization.factor(self._sharing("poisson"))
        if factorization.factorization is not None:
            factorization.solve(rhs, solution, tol=twl.SETTLE_DIRECT_TOLERANCE)
            return
        # An unfactorable (over the budget) or ill-conditioned system takes the multigrid
        # preconditioner, otherwise the Chebyshev polynomial (ordito/heat.py:4118-4150).
        unfactorable = factorization.refused or self._ill_conditioned
        twl.solve_spd(
            operators.poisson_system,
            rhs,
            solution,
            tol=_CG_TOLERANCE,
            preconditioner=self.poisson_multigrid if unfactorable else operators.poisson_preconditioner,
            name="heat_geodesic",
        )

    def dispose(self) -> None:
        """Release this solver's device state now: its factorizations and recorded passes, its
        multigrid hierarchy, and its operators (whose CG states go back to the pool kept by
        shape for the next operators of this shape). The solver is unusable afterwards."""
        self.release_factorizations()
        multigrid = getattr(self, "_poisson_multigrid", None)
        if multigrid is not None:
            multigrid.close()
            self._poisson_multigrid = None
        extra = []
        if getattr(self, "_pinned", None):
            extra.append(self._pinned[0])
        if getattr(self, "_regularized", None) is not None:
            extra.append(self._regularized[0])
        self._pinned = self._regularized = None
        if getattr(self, "_vector_operators", None) is not None:
            self._vector_operators.vector_system.release()
            self._vector_operators = None
        if self._operators is not None:
            for matrix in (self._operators.heat_system, self._operators.poisson_system,
                           self._operators.laplacian, *extra):
                matrix.release()
            self._operators = None
        self._systems.clear()
        self._gradient_terms = None
        self._mesh = None

    def release_factorizations(self) -> None:
        query = getattr(self, "_single_query", None)
        if query is not None:  # its graph names the factors' buffers
            query.close()
            self._single_query = None
        for kept in self._systems.values():
            kept["factorization"].release()

    @property
    def nbytes(self) -> int:
        total = 0
        for kept in self._systems.values():
            total += kept["factorization"].nbytes
        return total


def _require_sources(sources: Any, n_vertices: int) -> DeviceArray:
    src = as_device(sources, np.int32)
    return src.reshape(src.size)


# The divergence's form: per corner (ob_grad_div_terms, the default: measured faster -- 3.7 against
# 10.4 ms on icosphere(9) at 64 columns -- since a tile of 32 vertices still forms 1.7-2 times as
# many face gradients as there are faces and its shared-memory passes hold fewer warps) or face by
# face over vertex tiles (ob_grad_div_tiled).
_TILED_DIVERGENCE = False


def divergence_tiles(corner_offsets: DeviceArray, corner_slots: DeviceArray, n: int,
                     n_faces: int) -> tuple[DeviceArray, DeviceArray, DeviceArray]:
    """``(tile_faces, tile_counts, corner_codes)`` of a corner index (``ob_divergence_tiles``):
    the distinct faces of every tile of 32 consecutive vertices, for ``ob_grad_div_tiled``."""
    corners = max(3 * n_faces, 1)
    tile_faces = DeviceArray.empty(corners, np.int32)
    tile_counts = DeviceArray.empty(max((n + 31) // 32, 1), np.int32)
    corner_codes = DeviceArray.empty(corners, np.int32)
    _lib.call("ob_divergence_tiles", corner_offsets.ptr, corner_slots.ptr, n, tile_faces.ptr,
              tile_counts.ptr, corner_codes.ptr, DEFAULT_STREAM)
    return tile_faces, tile_counts, corner_codes


def corner_records(terms: DeviceArray, faces: DeviceArray, corner_slots: DeviceArray,
                   n_faces: int) -> tuple[DeviceArray, DeviceArray]:
    """``(records, ids)`` of a corner index (``ob_corner_records``): each corner's twelve divergence
    terms and its face's vertices, in the index's order, for ``ob_grad_div_records``."""
    corners = max(3 * n_faces, 1)
    records = DeviceArray.empty(12 * corners, np.float64)
    ids = DeviceArray.empty(4 * corners, np.int32)
    _lib.call("ob_corner_records", terms.ptr, faces.ptr, corner_slots.ptr, n_faces, records.ptr, ids.ptr,
              DEFAULT_STREAM)
    return records, ids


def _grad_div(solver: "HeatSolver", faces: DeviceArray, index: tuple, n: int, k: int, u: int,
              u_stride: int, u_iperm: Any, out: int, out_stride: int, out_iperm: Any, out_pinned: Any,
              stream: Any) -> None:
    _grad_div_index(solver.gradient_terms, faces, index, n, k, u, u_stride, u_iperm, out,
                    out_stride, out_iperm, out_pinned, stream)


def _grad_div_index(terms: DeviceArray, faces: DeviceArray, index: tuple, n: int, k: int, u: int,
                    u_stride: int, u_iperm: Any, out: int, out_stride: int, out_iperm: Any,
                    out_pinned: Any, stream: Any) -> None:
    """``-div`` of the per-face unit gradients of ``k`` heat columns over a corner index and its
    tiles ``(offsets, slots, tile_faces, tile_counts, codes)``, from per-face terms: each vertex's
    corners summed in ascending slot order (no atomics: the same bits on every run, the reference's
    deterministic mode, ordito/heat.py:3170-3232, as the only mode), per corner
    (``ob_grad_div_terms``) or face by face over the tiles (``ob_grad_div_tiled``)."""
    corner_offsets, corner_slots, tile_faces, tile_counts, codes = index
    if _TILED_DIVERGENCE:
        _lib.call(
            "ob_grad_div_tiled", terms.ptr, faces.ptr, corner_offsets.ptr,
            corner_slots.ptr, tile_faces.ptr, tile_counts.ptr, codes.ptr, n, k, u, u_stride, u_iperm,
            out, out_stride, out_iperm, out_pinned, stream,
        )  # fmt: skip
        return
    _lib.call(
        "ob_grad_div_terms", terms.ptr, faces.ptr, corner_offsets.ptr,
        corner_slots.ptr, n, k, u, u_stride, u_iperm, out, out_stride, out_iperm, out_pinned,
        stream,
    )  # fmt: skip


def _divergence(mesh: Trimesh, solver: "HeatSolver", k: int, u: int, u_stride: int, u_iperm: Any,
                out: int, out_stride: int, out_iperm: Any, out_pinned: Any, stream: Any) -> None:
    """``_grad_div`` over the mesh's own numbering (its corner index and tiles, made once)."""
    _grad_div(solver, mesh.faces, mesh.corner_tiles, mesh.n_vertices, k, u, u_stride, u_iperm, out,
              out_stride, out_iperm, out_pinned, stream)


def _corners_in_factor_rows(mesh: Trimesh, solver: "HeatSolver", h_iperm: int,
                            p_iperm: int) -> tuple[DeviceArray, tuple, tuple] | None:
    """The face buffer and the corner index renumbered into the factors' shared ordering (built
    once per solver and ordering, outside any recording: the first eager pass builds it), with
    the index's corner records (``corner_records``), so the served divergence reads the heat rows
    and writes the Poisson rows with no inverse permutation per corner; None when the two
    factors' orderings differ. A vertex's corners keep their ascending slot order, so the sums
    are the same bits as in the vertex numbering."""
    # Kept on the heat factor (its lifetime is the ordering's), keyed by both orderings.
    holder = solver.heat_factor
    key = (h_iperm, p_iperm, id(solver.poisson_factor))
    cached = getattr(holder, "_factor_row_corners", None)
    if cached is not None and cached[0] == key:
        return cached[1]
    n = mesh.n_vertices
    same = h_iperm == p_iperm or np.array_equal(
        DeviceArray(h_iperm, (n,), np.int32, owned=False).numpy(),
        DeviceArray(p_iperm, (n,), np.int32, owned=False).numpy())
    result = None
    if same:
        corners = 3 * mesh.n_faces
        faces = DeviceArray.empty(max(corners, 1), np.int32)
        _lib.call("ob_renumber", mesh.faces.ptr, corners, h_iperm, faces.ptr, DEFAULT_STREAM)
        offsets = DeviceArray.empty(n + 1, np.int32)
        slots = DeviceArray.empty(max(corners, 1), np.int32)
        size = ctypes.c_size_t(0)
        _lib.call("ob_corner_index_workspace", n, mesh.n_faces, ctypes.byref(size))
        workspace = DeviceArray.empty(int(size.value), np.uint8)
        _lib.call("ob_corner_index", faces.ptr, mesh.n_faces, n, offsets.ptr, slots.ptr,
                  workspace.ptr, int(size.value), DEFAULT_STREAM)
        tiles = divergence_tiles(offsets, slots, n, mesh.n_faces)
        records = corner_records(solver.gradient_terms, faces, slots, mesh.n_faces)
        _lib.call("ob_stream_synchronize", DEFAULT_STREAM)  # the arrays serve other streams
        result = (faces, (offsets, slots) + tiles, records)
    holder._factor_row_corners = (key, result)
    return result


def _distance_from_heat(mesh: Trimesh, solver: HeatSolver, sources: DeviceArray,
                        heat: DeviceArray, n_columns: int = 1,
                        source_offsets: DeviceArray | None = None) -> DeviceArray:
    """Divergence, Poisson solve and shift (ordito/heat.py:3052-3131); ``method="potpourri3d"``
    solves geometry-central's regularized Poisson system (:3124-3129)."""
    n = mesh.n_vertices
    neg_div = DeviceArray.empty(n * n_columns, np.float64)
    cover = solver.cover
    if cover is not None:
        # The divergence on the cover, from its lengths (ordito/heat.py:3080-3097): positive, the
        # same right-hand side as the extrinsic kernel's negated sum.
        from ordito_b200 import cover as gcover  # noqa: PLC0415

        gcover.cover_divergence(cover, heat, neg_div, n_columns)
    else:
        _divergence(mesh, solver, n_columns, heat.ptr, n_columns, None, neg_div.ptr, n_columns, None,
                    None, DEFAULT_STREAM)
    phi = DeviceArray.zeros(n * n_columns, np.float64)
    if solver.method == "potpourri3d":
        solver.solve_regularized_poisson(neg_div, phi)
    else:
        solver.solve_poisson(neg_div, phi)
    _lib.call(
        "ob_shift", phi.ptr, n, sources.ptr, sources.size,
        source_offsets.ptr if source_offsets is not None else None, n_columns, 1, DEFAULT_STREAM,
    )  # fmt: skip
    return phi


def _source_columns(source_sets: Any, n: int) -> tuple[DeviceArray, DeviceArray, int]:
    """Concatenated int32 sources and their column offsets (device), from a list of sets."""
    sets = [np.asarray(s, dtype=np.int64).reshape(-1) for s in source_sets]
    if not sets:
        raise ValueError("heat_geodesic_batch: no source sets")
    if any(s.size == 0 for s in sets):
        raise ValueError("heat_geodesic_batch: every source set needs at least one vertex")
    if any(((s < 0) | (s >= n)).any() for s in sets):
        raise ValueError(
            "heat_geodesic_batch: every source must be a vertex index in [0, n_vertices)"
        )
    offsets = np.zeros(len(sets) + 1, dtype=np.int32)
    offsets[1:] = np.cumsum([s.size for s in sets])
    flat = np.concatenate(sets).astype(np.int32)
    return DeviceArray.from_host(flat), DeviceArray.from_host(offsets), len(sets)


def heat_geodesic_batch(
    mesh: Trimesh,
    source_sets: Any,
    *,
    t: float | None = None,
    method: str = "meshlab",
    refine: int = 1,
    transpose: bool = True,
    poisson: str = "factor",
) -> DeviceArray:
    """Distances for many source sets on one resident mesh, solved together.

    The served form of ``heat_geodesic(trimesh, sources)``: both systems are factored once and
    kept on the mesh's solver, and each batch of ``k`` source sets (ragged) is one pass of the
    path over ``k`` right-hand sides -- seeding, the two factored solves (``refine`` float64
    refinement steps each), the divergence and the shift all run as batched kernels over the
    interleaved ``[V][k]`` columns. Returns ``(k, V)`` (or ``(V, k)`` with ``transpose=False``).
    Each column equals ``heat_geodesic(mesh, source_sets[c])`` up to the solves' rounding.

    ``poisson="multigrid"`` solves the Poisson system by the mixed-precision multigrid solve
    (float32 CG and V-cycle inside float64 refinement to a relative residual of 1e-10) instead of
    its factorisation; the heat system stays factored, because its far-field entries (down to
    ``exp(-d/h)``, below float32's range on a large mesh) need the float64 direct solve.
    """
    if not isinstance(mesh, Trimesh):
        raise TypeError("heat_geodesic_batch: serves a resident Trimesh")
    n = mesh.n_vertices
    _supported(method, False)
    if method != "meshlab":
        raise NotImplementedError(
            "heat_geodesic_batch serves method='meshlab' (the batched pass has no rim-pinned heat "
            "or regularized Poisson system); use heat_geodesic for 'igl' and 'potpourri3d'"
        )
    if poisson not in ("factor", "multigrid"):
        raise ValueError(f"poisson must be 'factor' or 'multigrid', got {poisson!r}")
    src, offsets, k = _source_columns(source_sets, n)
    if n == 0 or mesh.n_faces == 0:
        return DeviceArray.zeros((k, n) if transpose else (n, k), np.float64)
    solver = mesh.heat_solver(t, method=method)
    if poisson == "multigrid":
        if not solver.factor(("heat",)):
            raise RuntimeError("heat_geodesic_batch: the heat system could not be factored (over budget)")
        return _batch_multigrid(mesh, solver, src, offsets, k, refine, transpose)
    if not solver.factor():
        raise RuntimeError("heat_geodesic_batch: the systems could not be factored (over budget)")
    return _batch_columns(mesh, solver, src, offsets, k, refine, transpose)


def _batch_multigrid(mesh: Trimesh, solver: "HeatSolver", src: DeviceArray, offsets: DeviceArray,
                     k: int, refine: int, transpose: bool) -> DeviceArray:
    """The batched pass with the Poisson system on the mixed-precision multigrid solve."""
    n = mesh.n_vertices
    heat_factor = solver.heat_factor
    neg_div = DeviceArray.empty(n * k, np.float64)
    if refine == 0:
        h_rhs, h_sol, h_stride, h_iperm, h_pinned = heat_factor.work(k)
        _lib.call("ob_seed_permuted", src.ptr, offsets.ptr, k, n, h_iperm, h_pinned, h_stride,
                  h_rhs, DEFAULT_STREAM)
        heat_factor.solve_in_place(k)
        heat_sol, heat_stride, heat_iperm = h_sol, h_stride, h_iperm
    else:
        heat_rhs, heat_sol = heat_factor.buffers(k)
        invalid = solver.scratch_flag()
        _lib.call("ob_seed_columns", src.ptr, offsets.ptr, k, n, heat_rhs, invalid.ptr, DEFAULT_STREAM)
        heat_factor.solve_pointers(0, 0, k, refine)
        heat_stride, heat_iperm = k, None
    _divergence(mesh, solver, k, heat_sol, heat_stride, heat_iperm, neg_div.ptr, k, None, None,
                DEFAULT_STREAM)
    phi = DeviceArray.zeros(n * k, np.float64)
    cycle = solver.poisson_multigrid
    iters, residual, status = cycle.solve(neg_div.ptr, phi.ptr, k, _MULTIGRID_POISSON_TOLERANCE,
                                          twl.CG_MAXITER_FACTOR * n)
    if np.any(residual > _MULTIGRID_POISSON_TOLERANCE):
        warnings.warn(
            f"heat_geodesic_batch: multigrid Poisson solve stopped at relative residual "
            f"{float(residual.max()):.3g} (tolerance {_MULTIGRID_POISSON_TOLERANCE:.3g})",
            UserWarning, stacklevel=3,
        )
    _lib.call("ob_shift", phi.ptr, n, src.ptr, src.size, offsets.ptr, k, 1, DEFAULT_STREAM)
    if not transpose:
        return phi.reshape((n, k))
    return _transposed(phi, n, k)


def _batch_columns(mesh: Trimesh, solver: "HeatSolver", src: DeviceArray, offsets: DeviceArray,
                   k: int, refine: int, transpose: bool, *, stream: Any = None,
                   out: DeviceArray | None = None, work_set: int = 0) -> DeviceArray:
    """The batched pass over resident, validated source columns.

    Without refinement the pass stays in the factors' shared ordering from the seeds to the shift:
    the seeds go straight into the heat factor's right-hand side, the divergence (gathered per
    vertex, no atomics) reads the heat solution and writes the Poisson right-hand side through
    the inverse permutation, and the shift reads the Poisson solution the same way and writes the
    ``(k, V)`` distances -- no permutation, copy or transpose passes. With ``refine`` each solve
    instead runs in the caller's numbering with that many float64 refinement steps.

    ``stream`` (refinement-free pass only) enqueues the whole pass on that stream, and ``out`` (a
    ``(k, V)`` float64 device buffer) receives the distances instead of a new array: the served
    loop runs each batch this way, on its slot's stream, without allocating.
    """
    n = mesh.n_vertices
    heat_factor, poisson_factor = solver.heat_factor, solver.poisson_factor
    if refine == 0:
        st = stream if stream is not None else DEFAULT_STREAM
        h_rhs, h_sol, h_stride, h_iperm, h_pinned = heat_factor.work(k, st, work_set)
        p_rhs, p_sol, p_stride, p_iperm, p_pinned = poisson_factor.work(k, st, work_set)
        _lib.call("ob_seed_permuted", src.ptr, offsets.ptr, k, n, h_iperm, h_pinned, h_stride,
                  h_rhs, st)
        heat_factor.solve_in_place_sources(k, src, offsets, st, work_set)
        rows = _corners_in_factor_rows(mesh, solver, h_iperm, p_iperm)
        if rows is None:
            _divergence(mesh, solver, k, h_sol, h_stride, h_iperm, p_rhs, p_stride, p_iperm,
                        p_pinned, st)
        else:
            _, index, (records, ids) = rows
            _lib.call("ob_grad_div_records", records.ptr, ids.ptr, index[0].ptr, n, k, h_sol, h_stride, None,
                      p_rhs, p_stride, None, p_pinned, st)
        poisson_factor.solve_in_place(k, st, work_set)
        if out is None:
            out = DeviceArray.empty((k, n), np.float64)
        _lib.call("ob_shift_permuted", p_sol, n, p_stride, p_iperm, src.ptr, offsets.ptr, k, 1,
                  out.ptr, st)
        return out if transpose else _transposed(out, k, n)
    if stream is not None or out is not None or work_set != 0:
        raise ValueError("_batch_columns: stream/out/work_set serve the refinement-free pass only")
    heat_rhs, heat_sol = heat_factor.buffers(k)
    poisson_rhs, phi = poisson_factor.buffers(k)
    invalid = solver.scratch_flag()
    _lib.call("ob_seed_columns", src.ptr, offsets.ptr, k, n, heat_rhs, invalid.ptr, DEFAULT_STREAM)
    heat_factor.solve_pointers(0, 0, k, refine)
    _divergence(mesh, solver, k, heat_sol, k, None, poisson_rhs, k, None, None, DEFAULT_STREAM)
    poisson_factor.solve_pointers(0, 0, k, refine)
    _lib.call("ob_shift", phi, n, src.ptr, src.size, offsets.ptr, k, 1, DEFAULT_STREAM)
    if not transpose:
        out = DeviceArray.empty((n, k), np.float64)
        _lib.call("ob_memcpy", out.ptr, phi, out.nbytes, 2, DEFAULT_STREAM, 0)
        return out
    out = DeviceArray.empty((k, n), np.float64)
    _lib.call("ob_transpose", n, k, phi, out.ptr, DEFAULT_STREAM)
    return out


@contextlib.contextmanager
def capture_guard():
    """No garbage collection while this thread records a graph: a collection there would run
    destructors (device frees, solver teardown) inside the capture, which the capture forbids."""
    enabled = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if enabled:
            gc.enable()


class BatchStep:
    """One served batch pass recorded as a CUDA graph and replayed with a single launch.

    The refinement-free batched pass of ``_batch_columns`` -- seeding, the two factored
    triangular passes, the gathered divergence and the shift -- over ``k`` columns, bound to fixed
    device buffers: ``sources`` / ``offsets`` (read at every replay, so a caller rewrites their
    contents between batches) and ``out`` (``(k, V)`` float64, rewritten by every replay). Built by
    running the pass once eagerly on ``stream`` (a created stream: that prepares the factors'
    buffers, the per-face terms and the corner index) and recording it on the same stream; the
    graph then launches on any stream with no host work per step. If a factor's work buffers are
    reallocated afterwards (a wider batch elsewhere), the next launch records the pass again.
    """

    def __init__(self, mesh: Trimesh, solver: "HeatSolver", sources: DeviceArray,
                 offsets: DeviceArray, k: int, out: DeviceArray, stream: Any, *,
                 warm: bool = True, work_set: int = 0) -> None:
        self.stream = stream
        self.k = k
        self.out = out
        self.work_set = work_set
        self._args = (mesh, solver, sources, offsets)
        self.handle = None
        self._record(warm)

    def _generations(self) -> tuple[int, int]:
        solver = self._args[1]
        return (solver.heat_factor.work_generation(self.work_set),
                solver.poisson_factor.work_generation(self.work_set))

    def _record(self, warm: bool = True) -> None:
        import ctypes  # noqa: PLC0415

        self.close()
        mesh, solver, sources, offsets = self._args
        k, out, stream = self.k, self.out, self.stream
        if warm:
            # One eager pass prepares what the recording must find ready (the factors' buffers,
            # the per-face terms, the corner index); skipped when a wider step already did.
            _lib.call("ob_device_synchronize")  # buffers allocated on other streams are ready
            _batch_columns(mesh, solver, sources, offsets, k, 0, True, stream=stream, out=out,
                           work_set=self.work_set)
            _lib.call("ob_stream_synchronize", stream)
        self._recorded = self._generations()
        with capture_guard():
            _lib.call("ob_capture_begin", stream)
            error: BaseException | None = None
            try:
                _batch_columns(mesh, solver, sources, offsets, k, 0, True, stream=stream, out=out,
                               work_set=self.work_set)
            except BaseException as exc:  # noqa: BLE001 -- the capture must be closed first
                error = exc
            handle, kernels = ctypes.c_void_p(0), ctypes.c_int(0)
            status = _lib.lib.ob_capture_end(stream, ctypes.byref(handle), ctypes.byref(kernels))
        if error is not None:
            raise error
        _lib.check(status, "ob_capture_end")
        self.handle = handle
        self.kernels = int(kernels.value)

    RECORDING_STREAM = object()

    def launch(self, stream: Any = RECORDING_STREAM) -> DeviceArray:
        """Replay the pass on ``stream`` (``None``: the legacy default stream; by default the
        recording stream); returns ``out``."""
        if self._generations() != self._recorded:
            self._record()
        _lib.call("ob_graph_launch", self.handle,
                  self.stream if stream is BatchStep.RECORDING_STREAM else stream)
        return self.out

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.lib.ob_graph_destroy(self.handle)
            self.handle.value = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


class BatchPipeline:
    """A stream of batches on one resident mesh, host arrays out, pipelined: consecutive batches
    run on the factors' two work sets, each on its own stream (``BatchStep``), so batch i + 1's
    pass overlaps batch i's pass and its copy of the distances to pinned host memory (a third
    stream; ordered by events).

    ``map(batches)`` yields, in order, each batch's ``(k, V)`` float64 distances as a view of a
    pinned host buffer, valid until the generator has advanced twice more (copy it to keep it).
    Every batch has exactly ``k`` source sets (each a list of source vertices; host-validated).
    """

    def __init__(self, mesh: Trimesh, k: int, *, method: str = "meshlab", max_sources: int = 0) -> None:
        import ctypes  # noqa: PLC0415

        if method != "meshlab":
            raise NotImplementedError("BatchPipeline serves method='meshlab' (the batched pass)")

        from ordito_b200.device import PinnedArray  # noqa: PLC0415

        solver = mesh.heat_solver(None, method=method)
        if not solver.factor():
            raise RuntimeError("BatchPipeline: the systems could not be factored (over budget)")
        n = mesh.n_vertices
        self.n, self.k = n, k
        capacity = max(max_sources, 4 * k)
        self.copy = ctypes.c_void_p(0)
        _lib.call("ob_stream_create", ctypes.byref(self.copy))
        self.capacity = capacity
        self.slots = []
        for work_set in range(2):
            compute = ctypes.c_void_p(0)
            _lib.call("ob_stream_create", ctypes.byref(compute))
            src = DeviceArray.from_host(np.zeros(capacity, dtype=np.int32))
            off = DeviceArray.from_host(np.arange(k + 1, dtype=np.int32))
            out = DeviceArray.empty((k, n), np.float64)
            step = BatchStep(mesh, solver, src, off, k, out, compute, work_set=work_set)
            events = [ctypes.c_void_p(0), ctypes.c_void_p(0)]
            for e in events:
                _lib.call("ob_event_create", ctypes.byref(e))
            self.slots.append({
                "compute": compute, "src": src, "off": off, "step": step,
                "host": PinnedArray((k, n), np.float64),
                "h_src": PinnedArray(capacity, np.int32), "h_off": PinnedArray(k + 1, np.int32),
                "computed": events[0], "copied": events[1], "busy": False,
            })

    def _enqueue(self, slot: dict, sets: Any) -> None:
        if len(sets) != self.k:
            raise ValueError(f"BatchPipeline: batches of {self.k} source sets")
        arrays = [np.ascontiguousarray(s, dtype=np.int32).reshape(-1) for s in sets]
        sizes = np.array([a.size for a in arrays], dtype=np.int32)
        total = int(sizes.sum())
        if total > self.capacity or sizes.min() < 1:
            raise ValueError(f"BatchPipeline: 1 or more sources a set, {self.capacity} in all at most")
        flat = np.concatenate(arrays)
        if flat.min() < 0 or flat.max() >= self.n:
            raise ValueError("BatchPipeline: source index out of range")
        if slot["busy"]:
            # This slot's last copy must be done before its buffers are written again.
            _lib.call("ob_event_synchronize", slot["copied"])
        slot["h_src"].array[:total] = flat
        slot["h_off"].array[0] = 0
        np.cumsum(sizes, out=slot["h_off"].array[1:])
        compute = slot["compute"]
        _lib.call("ob_memcpy", slot["src"].ptr, slot["h_src"].ptr, 4 * total, 0, compute, 0)
        _lib.call("ob_memcpy", slot["off"].ptr, slot["h_off"].ptr, 4 * (self.k + 1), 0, compute, 0)
        slot["step"].launch(compute)
        _lib.call("ob_event_record", slot["computed"], compute)
        _lib.call("ob_stream_wait_event", self.copy, slot["computed"])
        _lib.call("ob_memcpy", slot["host"].ptr, slot["step"].out.ptr, 8 * self.k * self.n, 1, self.copy, 0)
        _lib.call("ob_event_record", slot["copied"], self.copy)
        slot["busy"] = True

    def map(self, batches: Any):
        pending = None
        for i, sets in enumerate(batches):
            slot = self.slots[i % 2]
            self._enqueue(slot, sets)
            if pending is not None:
                _lib.call("ob_event_synchronize", pending["copied"])
                yield pending["host"].array
            pending = slot
        if pending is not None:
            _lib.call("ob_event_synchronize", pending["copied"])
            yield pending["host"].array

    def close(self) -> None:
        streams = [self.copy] + [slot["compute"] for slot in self.slots]
        for stream in streams:
            if stream.value:
                _lib.lib.ob_stream_synchronize(stream)
        for slot in self.slots:
            slot["step"].close()
            for e in ("computed", "copied"):
                _lib.lib.ob_event_destroy(slot[e])
        self.slots = []
        for stream in streams:
            if stream.value:
                _lib.lib.ob_stream_destroy(stream)
                stream.value = None


class _SingleQuery:
    """``heat_geodesic(trimesh, sources)`` with both factors held: the single-column pass recorded
    once (``BatchStep``, k = 1) and replayed on the default stream, after the sources are copied
    into its buffer; the distances are copied into a new array for the caller."""

    def __init__(self, mesh: Trimesh, solver: "HeatSolver", capacity: int) -> None:
        import ctypes  # noqa: PLC0415

        n = mesh.n_vertices
        self.n = n
        self.capacity = capacity
        self.sources = DeviceArray.from_host(np.zeros(capacity, dtype=np.int32))
        self.offsets = DeviceArray.from_host(np.array([0, 1], dtype=np.int32))
        self.bounds = np.zeros(2, dtype=np.int32)
        self.stream = ctypes.c_void_p(0)
        _lib.call("ob_stream_create", ctypes.byref(self.stream))
        self.step = BatchStep(mesh, solver, self.sources, self.offsets, 1,
                              DeviceArray.empty((1, n), np.float64), self.stream)

    def __call__(self, sources: DeviceArray) -> DeviceArray:
        m = sources.size
        self.bounds[1] = m
        _lib.call("ob_memcpy", self.sources.ptr, sources.ptr, 4 * m, 2, DEFAULT_STREAM, 0)
        _lib.call("ob_memcpy", self.offsets.ptr, self.bounds.ctypes.data, 8, 0, DEFAULT_STREAM, 0)
        self.step.launch(DEFAULT_STREAM)
        out = DeviceArray.empty(self.n, np.float64)
        _lib.call("ob_memcpy", out.ptr, self.step.out.ptr, 8 * self.n, 2, DEFAULT_STREAM, 0)
        return out

    def close(self) -> None:
        self.step.close()
        if self.stream.value:
            _lib.lib.ob_stream_destroy(self.stream)
            self.stream.value = None


def _transposed(array: DeviceArray, rows: int, cols: int) -> DeviceArray:
    out = DeviceArray.empty((cols, rows), np.float64)
    _lib.call("ob_transpose", rows, cols, array.ptr, out.ptr, DEFAULT_STREAM)
    return out


def heat_geodesic(
    mesh: Any = None,
    faces: Any = None,
    sources: Any = None,
    t: float | None = None,
    *,
    vertices: Any = None,
    use_robust: bool = False,
    method: str = "meshlab",
) -> DeviceArray:
    """Approximate geodesic distance to the nearest source vertex (heat method).

    ``heat_geodesic(trimesh, sources)`` keeps the operators, solver states and factorizations on
    the mesh; ``heat_geodesic(vertices, faces, sources, t=None)`` builds them for the call. Returns
    the ``(n_vertices,)`` float64 distance on the device. Raises ``ValueError`` for a source index
    outside ``[0, n_vertices)`` or an unknown ``method``.
    """
    if method not in ("meshlab", "igl", "potpourri3d"):
        raise ValueError(f"method must be 'meshlab', 'igl' or 'potpourri3d', got {method!r}")
    bound, held, src_arg = mesh_arguments("heat_geodesic", mesh, vertices, faces, sources)
    if src_arg is None:
        raise TypeError("heat_geodesic: sources are required")
    try:
        return _heat_geodesic(bound, src_arg, t, use_robust, method)
    finally:
        if not held:
            # The call's own mesh: released now rather than whenever a garbage collection finds
            # its reference cycle (its CG states go back to the pool for the next call).
            bound.dispose()


def _heat_geodesic(bound: Trimesh, src_arg: Any, t: float | None, use_robust: bool,
                   method: str) -> DeviceArray:
    n = bound.n_vertices
    host_sources = None
    if not hasattr(src_arg, "__cuda_array_interface__"):
        host_sources = np.ascontiguousarray(src_arg, dtype=np.int32).reshape(-1)
    src = _require_sources(src_arg if host_sources is None else host_sources, n)
    if n == 0 or bound.n_faces == 0 or src.size == 0:
        return DeviceArray.zeros(n, np.float64)
    _supported(method, use_robust)
    solver = bound.heat_solver(t, use_robust=use_robust, method=method)
    # The recorded single-query pass serves the default discretization (meshlab: Neumann heat,
    # the pinned Poisson system); the others run their own extra solves below.
    held_factors = (method == "meshlab" and solver.heat_factor is not None
                    and solver.poisson_factor is not None)
    # Host sources are checked on the host; device sources by one small read-back (the
    # reference's 4-byte flag, ordito/heat.py:5488).
    if host_sources is not None or held_factors:
        checked = host_sources if host_sources is not None else src.numpy()
        if checked.min() < 0 or checked.max() >= n:
            raise ValueError(
                "heat_geodesic: every entry of sources must be a vertex index in [0, n_vertices)"
            )
    if held_factors:
        # Both systems factored (a warm resident mesh): the whole query is one recorded pass.
        return solver.single_query(src)
    u0 = DeviceArray.empty(n, np.float64)
    invalid = DeviceArray.empty(1, np.int32)
    _lib.call("ob_seed", src.ptr, src.size, n, u0.ptr, invalid.ptr, DEFAULT_STREAM)
    if host_sources is None and int(invalid.numpy()[0]) != 0:
        raise ValueError(
            "heat_geodesic: every entry of sources must be a vertex index in [0, n_vertices)"
        )
    heat = DeviceArray.zeros(n, np.float64)
    solver.diffuse(u0, heat)
    if method == "igl":
        # igl::heat_geodesics' boundary rule: the mean of the Neumann heat and the heat pinned to
        # zero on the rim, when the mesh has one (ordito/heat.py:594-597).
        pinned = DeviceArray.zeros(n, np.float64)
        if solver.diffuse_pinned(u0, pinned):
            _lib.call("ob_axpby", n, 0.5, pinned.ptr, 0.5, heat.ptr, heat.ptr, DEFAULT_STREAM)
    return _distance_from_heat(bound, solver, src, heat)


# extend_scalar warns when the extension leaves the source values' range by more than this
# fraction of their scale (ordito/heat.py:166): the diffusion is a convex average only while every
# cotangent weight is non-negative.
_EXTEND_RANGE_TOLERANCE = 1e-4


def extend_scalar(
    mesh: Any = None,
    faces: Any = None,
    sources: Any = None,
    values: Any = None,
    t: float | None = None,
    *,
    vertices: Any = None,
) -> DeviceArray:
    """Extend values from a few source vertices over the whole surface by nearest-source
    interpolation (ordito/heat.py:2321; potpourri3d's ``MeshVectorHeatSolver.extend_scalar``).

    ``extend_scalar(trimesh, sources, values, t=...)`` or ``extend_scalar(vertices, faces, sources,
    values, t)``. The values and an indicator of the sources diffuse through the heat system for
    the same short time ``t`` (one two-column settled solve); their quotient is the extension.
    Returns the ``(n_vertices,)`` float64 field on the device. Raises ``ValueError`` when
    ``values`` is not as long as ``sources`` or a source is not a vertex index; warns
    (``UserWarning``) when the field leaves the source values' range (negative cotangent weights).
    """
    if isinstance(mesh, Trimesh):
        if vertices is not None or values is not None:
            raise TypeError("extend_scalar: pass (trimesh, sources, values) or (vertices, faces, sources, values)")
        bound, held, src_arg, val_arg = mesh, True, faces, sources
    else:
        verts = mesh if vertices is None else vertices
        if verts is None or faces is None:
            raise TypeError("extend_scalar: needs a Trimesh, or vertices and faces")
        bound, held, src_arg, val_arg = Trimesh(verts, faces), False, sources, values
    try:
        return _extend_scalar(bound, src_arg, val_arg, t)
    finally:
        if not held:
            bound.dispose()


def _extend_scalar(bound: Trimesh, src_arg: Any, val_arg: Any, t: float | None) -> DeviceArray:
    n = bound.n_vertices
    src = _require_sources(src_arg if hasattr(src_arg, "__cuda_array_interface__")
                           else np.ascontiguousarray(src_arg, dtype=np.int32).reshape(-1), n)
    if n == 0 or bound.n_faces == 0 or src.size == 0:
        return DeviceArray.zeros(n, np.float64)
    vals = as_device(val_arg if hasattr(val_arg, "__cuda_array_interface__")
                     else np.ascontiguousarray(val_arg, dtype=np.float64).reshape(-1), np.float64)
    if vals.size != src.size:
        raise ValueError(f"extend_scalar: values must hold one value per source ({src.size}), got {vals.size}")
    rhs = DeviceArray.empty((n, 2), np.float64)
    value_range = DeviceArray.empty(3, np.float64)
    invalid = DeviceArray.empty(1, np.int32)
    _lib.call("ob_extend_seed", src.ptr, vals.ptr, src.size, n, rhs.ptr, value_range.ptr, invalid.ptr,
              DEFAULT_STREAM)
    if int(invalid.numpy()[0]) != 0:
        raise ValueError("extend_scalar: every entry of sources must be a vertex index in [0, n_vertices)")
    solver = bound.heat_solver(t)
    diffused = DeviceArray.zeros((n, 2), np.float64)
    solver.diffuse(rhs, diffused)
    extended = DeviceArray.empty(n, np.float64)
    _lib.call("ob_extend_ratio", diffused.ptr, n, value_range.ptr, extended.ptr, DEFAULT_STREAM)
    low, high, excess = (float(x) for x in value_range.numpy())
    scale = max(high - low, abs(low), abs(high))
    if excess > _EXTEND_RANGE_TOLERANCE * scale:
        warnings.warn(
            f"extend_scalar: the extended field leaves the source values' range [{low:.6g}, {high:.6g}] "
            f"by {excess:.3g}. The cotangent weights of obtuse triangles are negative here, so the "
            "diffusion is not a convex average.",
            UserWarning,
            stacklevel=3,
        )
    return extended


# --------------------------------------------------------------------------------------------
# The vector heat method (Sharp, Soliman and Crane 2019): transport_tangent_vectors and log_map
# (ordito/heat.py:1740-3027), on the potpourri3d discretization.
# --------------------------------------------------------------------------------------------

# A transported direction is resolved where the diffused vector is longer than this fraction of
# the diffused magnitudes at the same vertex (ordito/heat.py:1726).
_RESOLVED_FRACTION = 1e-4
LOG_MAP_METHODS = ("heat_geodesic", "potpourri3d")


class VectorHeatOperators(NamedTuple):
    """What ``vector_heat_operators`` returns (ordito/heat.py:1740-1955). ``vector_system`` is
    ``M + t L_connection`` as the real ``2V x 2V`` CSR matrix (vertex v's tangent components in
    rows ``2v`` and ``2v + 1``: the reference's ``mat22d`` blocks written out), ``scalar`` the
    heat operators at the same ``t``, ``frames`` ``(basis_x, basis_y, normal)``."""

    vector_system: CsrMatrix
    scalar: HeatOperators
    frames: tuple[DeviceArray, DeviceArray, DeviceArray]
    preconditioner: twl.Preconditioner


def _vector_system(mesh: Trimesh, pattern: MeshOperatorPattern, rotations: DeviceArray, mass: DeviceArray,
                   t: float | None, edge_sums: DeviceArray | None) -> CsrMatrix:
    """``M + t L_connection`` over the expanded pattern (``ob_block_pattern``, ``ob_half_cot_f64``,
    ``ob_vector_heat_rows``); ``t`` None takes the device's ``h ** 2`` from ``edge_sums``."""
    n = mesh.n_vertices
    nnz = int(pattern.offsets.view(n, n + 1).numpy()[0]) if n else 0
    offsets = DeviceArray.empty(2 * n + 1, np.int32)
    columns = DeviceArray.empty(max(4 * nnz, 1), np.int32)
    _lib.call("ob_block_pattern", pattern.offsets.ptr, pattern.columns.ptr, n, offsets.ptr, columns.ptr,
              DEFAULT_STREAM)
    cot = DeviceArray.empty((max(mesh.n_faces, 1), 3), np.float64)
    _lib.call("ob_half_cot_f64", mesh.vertices.ptr, mesh.faces.ptr, mesh.n_faces, cot.ptr, DEFAULT_STREAM)
    values = DeviceArray.empty(max(4 * nnz, 1), np.float64)
    if t is None and edge_sums is None:
        raise ValueError("_vector_system: t None needs the edge sums")
    _lib.call(
        "ob_vector_heat_rows", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr, pattern.keys.ptr,
        pattern.n_keys, pattern.order.ptr, n, mesh.faces.ptr, cot.ptr, rotations.ptr, mass.ptr,
        1.0 if t is None else float(t), edge_sums.ptr if t is None else None, 1 if t is None else 0, values.ptr,
        DEFAULT_STREAM,
    )  # fmt: skip
    return CsrMatrix(2 * n, 2 * n, offsets, columns, values, 4 * nnz)


def vector_heat_operators(vertices: Any, faces: Any, t: float | None = None, *, scalar_operators: Any = None,
                          frames: Any = None, pattern: MeshOperatorPattern | None = None,
                          transport_angles: Any = None) -> VectorHeatOperators:
    """Everything the vector solvers need before their solves (ordito/heat.py:1740): the vector
    heat system ``M + t L_connection``, the scalar heat operators at the same ``t`` (or the
    caller's ``scalar_operators``, which must be at that ``t``), the vertex tangent frames (or the
    caller's ``frames``) and the vector system's Jacobi preconditioner. ``t`` None: the squared
    unique-edge mean. ``pattern`` and ``transport_angles`` may be passed prebuilt. Raises
    ``ValueError`` for a pattern of another operator or vertex count."""
    mesh = Trimesh(vertices, faces)
    if pattern is not None:
        if pattern.operator != "cotmatrix" or pattern.n_vertices != mesh.n_vertices:
            raise ValueError(
                f"pattern was built for operator={pattern.operator!r} over {pattern.n_vertices} vertices; the "
                f"heat operators need operator='cotmatrix' over {mesh.n_vertices}"
            )
        mesh._pattern = pattern
    operators, built = _assemble(mesh, t, "potpourri3d")
    if mesh.n_faces == 0:
        system = CsrMatrix(2 * mesh.n_vertices, 2 * mesh.n_vertices,
                           DeviceArray.zeros(2 * mesh.n_vertices + 1, np.int32), DeviceArray.empty(1, np.int32),
                           DeviceArray.empty(1, np.float64), 0)
    else:
        if transport_angles is None:
            rotations = mesh.halfedge_transport[1]
        else:
            angles = as_device(transport_angles, np.float64)
            if angles.size != 3 * mesh.n_faces:
                raise ValueError(f"transport_angles must hold one angle per halfedge ({3 * mesh.n_faces})")
            rotations = DeviceArray.empty((3 * mesh.n_faces, 2), np.float64)
            _lib.call("ob_polar_unit", angles.ptr, angles.size, rotations.ptr, DEFAULT_STREAM)
        system = _vector_system(mesh, mesh.mesh_operator_pattern, rotations, built.mass, t, built.edge_sums)
    return VectorHeatOperators(
        system,
        scalar_operators if scalar_operators is not None else operators,
        tuple(frames) if frames is not None else mesh.vertex_tangent_frames,
        twl.jacobi_preconditioner(system),
    )


def tangent_to_world(tangent: Any, basis_x: Any, basis_y: Any) -> DeviceArray:
    """A tangent field ``(V, 2)`` as world vectors ``(V, 3)``: ``a * basis_x + b * basis_y``."""
    from ordito_b200.tangent_space import tangent_to_world as _to_world  # noqa: PLC0415

    return _to_world(tangent, basis_x, basis_y)


def transport_tangent_vectors(
    mesh: Any = None,
    faces: Any = None,
    sources: Any = None,
    vectors: Any = None,
    t: float | None = None,
    *,
    vertices: Any = None,
) -> tuple[DeviceArray, DeviceArray]:
    """Parallel-transport tangent vectors from a few source vertices to every vertex
    (ordito/heat.py:2526; potpourri3d's ``MeshVectorHeatSolver.transport_tangent_vectors``).

    ``transport_tangent_vectors(trimesh, sources, vectors, t=...)`` or
    ``transport_tangent_vectors(vertices, faces, sources, vectors, t)``; ``vectors`` ``(k, 2)``, each
    in its own source's frame. The vector heat system diffuses the source vectors (their
    directions) and the heat system their indicator and magnitudes (the lengths), as two settled
    solves. Returns ``(transported float32 (V, 2), resolved bool (V,))`` on the device, each vector
    in its vertex's frame (``vertex_tangent_frames``); ``resolved`` is False where the direction
    cannot be told from round-off (nothing arrived, or copies cancel on the cut locus). Raises
    ``ValueError`` when ``vectors`` is not as long as ``sources`` or a source is not a vertex."""
    if isinstance(mesh, Trimesh):
        if vertices is not None or vectors is not None:
            raise TypeError("transport_tangent_vectors: pass (trimesh, sources, vectors) or "
                            "(vertices, faces, sources, vectors)")
        bound, held, src_arg, vec_arg = mesh, True, faces, sources
    else:
        verts = mesh if vertices is None else vertices
        if verts is None or faces is None:
            raise TypeError("transport_tangent_vectors: needs a Trimesh, or vertices and faces")
        bound, held, src_arg, vec_arg = Trimesh(verts, faces), False, sources, vectors
    try:
        return _transport_tangent_vectors(bound, src_arg, vec_arg, t)
    finally:
        if not held:
            bound.dispose()


def _transport_tangent_vectors(bound: Trimesh, src_arg: Any, vec_arg: Any,
                               t: float | None) -> tuple[DeviceArray, DeviceArray]:
    n = bound.n_vertices
    src = _require_sources(src_arg if hasattr(src_arg, "__cuda_array_interface__")
                           else np.ascontiguousarray(src_arg, dtype=np.int32).reshape(-1), n)
    if n == 0 or bound.n_faces == 0 or src.size == 0:
        return DeviceArray.zeros((n, 2), np.float32), DeviceArray.zeros(n, np.bool_)
    vec = as_device(vec_arg if hasattr(vec_arg, "__cuda_array_interface__")
                    else np.ascontiguousarray(vec_arg, dtype=np.float32).reshape(-1), np.float32)
    if vec.size != 2 * src.size:
        raise ValueError(f"transport_tangent_vectors: vectors must hold one 2D vector per source ({src.size}), "
                         f"got {vec.size // 2}")
    field_rhs = DeviceArray.empty(2 * n, np.float64)
    scalar_rhs = DeviceArray.empty((n, 2), np.float64)
    invalid = DeviceArray.empty(1, np.int32)
    _lib.call("ob_transport_seed", src.ptr, vec.ptr, src.size, n, field_rhs.ptr, scalar_rhs.ptr, invalid.ptr,
              DEFAULT_STREAM)
    if int(invalid.numpy()[0]) != 0:
        raise ValueError("transport_tangent_vectors: every entry of sources must be a vertex index in "
                         "[0, n_vertices)")
    solver = bound.heat_solver(t)
    field = DeviceArray.zeros(2 * n, np.float64)
    solver.diffuse_tangent(field_rhs, field)
    scalars = DeviceArray.zeros((n, 2), np.float64)
    solver.diffuse(scalar_rhs, scalars)
    transported = DeviceArray.empty((n, 2), np.float32)
    resolved = DeviceArray.empty(n, np.bool_)
    _lib.call("ob_transport_tail", field.ptr, scalars.ptr, n, _RESOLVED_FRACTION, transported.ptr, resolved.ptr,
              DEFAULT_STREAM)
    return transported, resolved


def log_map(
    mesh: Any = None,
    faces: Any = None,
    source: int | None = None,
    t: float | None = None,
    *,
    vertices: Any = None,
    method: str = "heat_geodesic",
) -> DeviceArray:
    """Every vertex's position in the source vertex's tangent plane (ordito/heat.py:2745): length
    the geodesic distance, direction the initial direction of the geodesic, as float32 ``(V, 2)``
    in the source's frame, ``(0, 0)`` at the source.

    ``method="heat_geodesic"`` (default): radius and radial direction from ``heat_geodesic``'s
    distance at the vector heat method's ``t``, the angle against the source's reference direction
    parallel-transported outwards. ``"potpourri3d"``: geometry-central's construction -- a second
    vector diffusion of an outward ball gives the radial direction, its divergence integrated by
    one Poisson solve the radius. Raises ``ValueError`` for a source outside ``[0, V)`` or an
    unknown ``method``."""
    if method not in LOG_MAP_METHODS:
        raise ValueError(f"log_map: method must be 'heat_geodesic' or 'potpourri3d', got {method!r}")
    if isinstance(mesh, Trimesh):
        if vertices is not None:
            raise TypeError("log_map: pass (trimesh, source) or (vertices, faces, source)")
        bound, held, src = mesh, True, faces
    else:
        verts = mesh if vertices is None else vertices
        if verts is None or faces is None:
            raise TypeError("log_map: needs a Trimesh, or vertices and faces")
        bound, held, src = Trimesh(verts, faces), False, source
    try:
        return _log_map(bound, int(src), t, method)
    finally:
        if not held:
            bound.dispose()


def _log_map(bound: Trimesh, source: int, t: float | None, method: str) -> DeviceArray:
    n = bound.n_vertices
    if n == 0 or bound.n_faces == 0:
        return DeviceArray.zeros((n, 2), np.float32)
    if not 0 <= source < n:
        raise ValueError(f"log_map: source must be a vertex index in [0, {n}), got {source}")
    solver = bound.heat_solver(t)
    if method == "potpourri3d":
        return _log_map_vector_heat(bound, solver, source)
    operators = solver.vector_operators
    invalid = DeviceArray.empty(1, np.int32)
    sources = DeviceArray.from_host(np.array([source, 2 * source], dtype=np.int32))
    field_rhs = DeviceArray.empty(2 * n, np.float64)
    _lib.call("ob_seed", sources.view(1, 2).ptr, 1, 2 * n, field_rhs.ptr, invalid.ptr, DEFAULT_STREAM)
    heat_rhs = DeviceArray.empty(n, np.float64)
    _lib.call("ob_seed", sources.ptr, 1, n, heat_rhs.ptr, invalid.ptr, DEFAULT_STREAM)
    transported = DeviceArray.zeros(2 * n, np.float64)
    solver.diffuse_tangent(field_rhs, transported)
    heat = DeviceArray.zeros(n, np.float64)
    solver.diffuse(heat_rhs, heat)
    distance = _distance_from_heat(bound, solver, sources.view(0, 1), heat)
    # The radial direction: the distance's unit face gradients, area-weighted onto the vertices.
    scalar = operators.scalar
    corner_offsets, corner_slots = bound.corner_index
    face_scratch = DeviceArray.empty((bound.n_faces, 3), np.float32)
    gradient = DeviceArray.empty((n, 3), np.float32)
    _lib.call("ob_vertex_unit_gradient", bound.vertices.ptr, bound.faces.ptr, bound.n_faces, n,
              scalar.face_normals.ptr, scalar.face_areas.ptr, distance.ptr, corner_offsets.ptr, corner_slots.ptr,
              face_scratch.ptr, gradient.ptr, DEFAULT_STREAM)
    basis_x, basis_y, _ = operators.frames
    out = DeviceArray.empty((n, 2), np.float32)
    _lib.call("ob_log_map_angles", gradient.ptr, basis_x.ptr, basis_y.ptr, transported.ptr, distance.ptr, n,
              out.ptr, DEFAULT_STREAM)
    return out


def _log_map_vector_heat(bound: Trimesh, solver: HeatSolver, source: int) -> DeviceArray:
    """``log_map(method="potpourri3d")`` (ordito/heat.py:2952): the outward ball and the reference
    direction diffused as two columns of one vector solve, the unit radial field's divergence
    integrated by the Poisson solve, the angle the radial direction's against the reference's."""
    n, n_faces = bound.n_vertices, bound.n_faces
    operators = solver.vector_operators
    ring, ring_offsets, _ = bound.vertex_one_rings
    tangent = bound.halfedge_tangent_angles
    transport = bound.halfedge_transport_angles
    rhs = DeviceArray.empty((2 * n, 2), np.float64)
    _lib.call("ob_log_map_outward_ball", bound.vertices.ptr, bound.faces.ptr, ring_offsets.ptr, ring.ptr,
              tangent.ptr, transport.ptr, source, n, rhs.ptr, DEFAULT_STREAM)
    fields = DeviceArray.zeros((2 * n, 2), np.float64)
    solver.diffuse_tangent(rhs, fields)
    corner_offsets, corner_slots = bound.corner_index
    corner_scratch = DeviceArray.empty(3 * n_faces, np.float64)
    divergence = DeviceArray.empty(n, np.float64)
    _lib.call("ob_radial_divergence", bound.vertices.ptr, bound.faces.ptr, n_faces, n, tangent.ptr, transport.ptr,
              fields.ptr, source, operators.scalar.cot_entries.ptr, corner_offsets.ptr, corner_slots.ptr,
              corner_scratch.ptr, divergence.ptr, DEFAULT_STREAM)
    distance = DeviceArray.zeros(n, np.float64)
    solver.solve_poisson(divergence, distance)
    out = DeviceArray.empty((n, 2), np.float32)
    _lib.call("ob_log_map_fields", fields.ptr, distance.ptr, source, n, out.ptr, DEFAULT_STREAM)
    return out
