"""The marched settled solve (GPU): past the factorisation budget, the heat system is solved band
by band with every entry to its own relative precision (ordito/linalg.py:2765), and the distance
through it matches the float64 oracle."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import cholesky as gchol
from ordito_b200 import creation
from ordito_b200 import heat as gheat
from ordito_b200 import linalg as glinalg
from ordito_b200.device import DeviceArray
from ordito_b200.mesh import Trimesh

pytestmark = pytest.mark.gpu

ENTRY_TOL = 1e-5  # every heat entry above underflow, relative to itself
DISTANCE_TOL = 1e-5


def _heat_system(v, f):
    t, _ = hp.vertex_time(v, f, None)
    ops = hp.heat_operators(v, f, t)
    return ops, hp.csr_matrix(ops["pattern"], ops["H"])


@pytest.mark.parametrize("shape", [(128, 64), (96, 48)])
def test_march_reaches_every_entry(gpu, shape) -> None:
    v, f = creation.jittered_torus(*shape, seed=2)
    n = v.shape[0]
    ops, H = _heat_system(v, f)
    rhs = np.zeros(n)
    rhs[7] = 1.0
    exact = hp.HeatFactor(H).solve(rhs)
    gops = gheat.heat_operators(v, f.reshape(-1))
    x = DeviceArray.zeros(n, np.float64)
    rounds = glinalg.march_settled(gops.heat_system, rhs, x)
    got = x.numpy()
    assert rounds > 0
    alive = exact > 1e-280
    assert alive.sum() > 0.99 * n  # the field spans hundreds of e-folds but stays representable
    rel = np.abs(got[alive] - exact[alive]) / exact[alive]
    assert rel.max() <= ENTRY_TOL
    assert exact.max() / exact[alive].min() > 1e20  # a far field far below a normwise 1e-14 solve


def test_march_columns(gpu) -> None:
    v, f = creation.icosphere(3)
    n = v.shape[0]
    ops, H = _heat_system(v, f)
    rhs = np.zeros((n, 3))
    rhs[[0, 100, 400], [0, 1, 2]] = 1.0
    gops = gheat.heat_operators(v, f.reshape(-1))
    x = DeviceArray.zeros(n * 3, np.float64)
    glinalg.march_settled(gops.heat_system, rhs.reshape(-1), x)
    got = x.numpy().reshape(n, 3)
    factor = hp.HeatFactor(H)
    for c in range(3):
        exact = factor.solve(rhs[:, c])
        assert np.max(np.abs(got[:, c] - exact) / exact) <= ENTRY_TOL


def test_distance_past_the_budget(gpu, monkeypatch) -> None:
    # A budget below the factor's size: the heat solve marches and the Poisson solve takes the
    # multigrid preconditioner (ordito/heat.py:4118-4150), as on a mesh too large to factor.
    monkeypatch.setattr(gchol, "CHOLESKY_MEMORY_BUDGET", 1 << 10)
    v, f = creation.jittered_torus(128, 64, seed=5)
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    assert not solver.factor()
    source = np.array([11], dtype=np.int32)
    got = gheat.heat_geodesic(mesh, source, method="meshlab").numpy()
    ref = hp.heat_geodesic(v, f, source)
    assert hp.relative_linf(got, ref) <= DISTANCE_TOL
    assert solver.heat_factor is None and solver.poisson_factor is None
