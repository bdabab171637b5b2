"""CPU oracle for the heat-method geodesic path: TEST INFRASTRUCTURE ONLY.

This package is a float64 (and, where the reference computes in float32, float32) restatement of
ordito's heat-method path in numpy/scipy. It exists to check the CUDA implementation in
``ordito_b200``; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import it, and only as the checker. The product path never calls into it.

Pinning: the reference (ordito 0.5.2) is Warp-DSL Python and ``warp-lang`` is not installable
here, so the reference itself cannot run. The oracle is pinned against every known-answer value
the reference's own docstrings and tests state for this path (``tests/golden/``): the unit-square
half-cotangent table (``ordito/laplacian.py:240-249``), the ``csr_from_keys`` toy example
(``ordito/array.py:1734-1745``), the lumped-mass sums on the unit cube and the 3-level icosphere
(``ordito/laplacian.py:1994-2004``), the icosphere(2) area (``ordito/creation.py``'s icosphere
docstring), ``solve_spd(M - tL, M 1) = 1`` (``ordito/linalg.py:1444-1461``) and the pole-to-pole
distance on icosphere(3) (``ordito/heat.py:519-534``). Bit-level agreement with the reference's
Warp output is therefore pinned only through those values ("parity partially pinned").
"""
