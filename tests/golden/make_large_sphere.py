"""Writes tests/golden/oracle_ico9_sample.npz: the float64 oracle's distances on the large sphere.

The workload: icosphere(9) (2 621 442 vertices, 5 242 880 faces) with 1 % seeded radial noise
(seed 0), 8 single-source queries drawn by ``numpy.random.default_rng(5).choice(V, 8,
replace=False)``, the ``"meshlab"`` discretisation. The oracle solves both systems exactly
(SuperLU in a geometric nested-dissection ordering, ``oracle.heat_path.dissection_order``: the
oracle's direct solve scaled to this size; its default column ordering needs minutes and tens of
GB a factor here). A full answer is 8 x 2.6 M doubles, so the fixture keeps every 256th vertex
and each query's source, the per-query maximum distance (the scale of the relative L-inf error)
and the per-query sum over all vertices (a checksum of the whole field).

Run ``python tests/golden/make_large_sphere.py`` from the repository root (about ten minutes and
~25 GB of host memory on 8 cores).
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import heat_path as hp  # noqa: E402
from ordito_b200 import creation  # noqa: E402

STRIDE = 256


def workload() -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    vertices, faces = creation.icosphere(9)
    vertices = creation.radial_noise(vertices, 0.01, 0)
    sources = np.random.default_rng(5).choice(vertices.shape[0], 8, replace=False).astype(np.int32)
    return vertices, faces, sources


def main() -> None:
    t0 = time.time()
    vertices, faces, sources = workload()
    n = vertices.shape[0]
    t_eff, _ = hp.vertex_time(vertices, faces, None)
    ops = hp.heat_operators(vertices, faces, t_eff)
    heat = hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"]), vertices)
    print(f"heat factor {time.time() - t0:.0f} s", flush=True)
    poisson = hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"]), vertices)
    print(f"poisson factor {time.time() - t0:.0f} s", flush=True)
    sample = np.union1d(np.arange(0, n, STRIDE), sources).astype(np.int64)
    distances, scales, sums = [], [], []
    for s in sources:
        d = hp.heat_geodesic(vertices, faces, np.array([s]), operators=ops, factors=(heat, poisson))
        distances.append(d[sample])
        scales.append(float(np.max(np.abs(d))))
        sums.append(float(np.sum(d)))
        print(f"source {s}: max {scales[-1]:.6f} ({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(
        os.path.join(os.path.dirname(__file__), "oracle_ico9_sample.npz"),
        sources=sources,
        sample=sample,
        distance=np.asarray(distances),
        scale=np.asarray(scales),
        total=np.asarray(sums),
        t=np.array([ops["t"]]),
    )


if __name__ == "__main__":
    main()
