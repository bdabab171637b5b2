"""Writes tests/golden/oracle_ico3.npz: the oracle's outputs on icosphere(3), source vertex 0.

Run ``python tests/golden/make_golden.py`` from the repository root. The oracle (``oracle/``) is
itself pinned by ``known_answers.json``; these arrays freeze its outputs so a later change to the
oracle or the generator shows up as a fixture mismatch.
"""

from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import heat_path as hp  # noqa: E402
from ordito_b200 import creation  # noqa: E402


def main() -> None:
    vertices, faces = creation.icosphere(3)
    ops = hp.heat_operators(vertices, faces)
    pattern = ops["pattern"]
    distance = hp.heat_geodesic(vertices, faces, np.array([0]))
    np.savez_compressed(
        os.path.join(os.path.dirname(__file__), "oracle_ico3.npz"),
        vertices=vertices,
        faces=faces,
        offsets=pattern["offsets"],
        columns=pattern["columns"],
        run_start=pattern["run_start"],
        keys=pattern["keys"],
        cot=ops["cot"],
        L=ops["L"],
        H=ops["H"],
        mass=ops["mass"],
        t=np.array([ops["t"]]),
        distance=distance,
    )


if __name__ == "__main__":
    main()
