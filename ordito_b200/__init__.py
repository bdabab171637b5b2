"""ordito_b200: a B200 (sm_100a) build of ordito's heat-method geodesic path.

Drop-in modules for the path: ``laplacian`` (pattern, cotangent weights, Laplacian, mass),
``heat`` (``heat_operators``, ``heat_geodesic``, ``HeatSolver``), ``linalg`` (``solve_spd``,
``solve_spd_settled``, the Jacobi, Chebyshev and multigrid preconditioners), ``cholesky``, ``mesh``
(``Trimesh``), and for the vector heat method (``heat.transport_tangent_vectors``, ``heat.log_map``)
``halfedge`` and ``tangent_space``. The compute runs in hand-written CUDA kernels behind the C ABI of
``include/ordito_b200.h`` (``libordito_b200.so``, built by ``python -m ordito_b200.build``).
"""

from ordito_b200 import config, creation  # noqa: F401  (host-only: settings, mesh generators)
from ordito_b200.config import deterministic, is_deterministic, set_deterministic  # noqa: F401

__all__ = ["array", "cholesky", "config", "creation", "device", "halfedge", "heat", "laplacian", "linalg", "mesh",
           "tangent_space", "deterministic", "is_deterministic", "set_deterministic"]
__version__ = "0.1.0"
