"""The packed-batch workload on the host: 256 meshes of the stated kinds and sizes, 1-16 distinct
single-source queries each, reproducible from the seed."""

from __future__ import annotations

from ordito_b200.packed import packed_workload, total_queries


def test_packed_workload() -> None:
    w = packed_workload(3, 256)
    assert len(w.meshes) == len(w.queries) == len(w.specs) == 256
    kinds = {s[0] for s in w.specs}
    assert kinds == {"icosphere", "torus"}
    for spec, (v, f), q in zip(w.specs, w.meshes, w.queries):
        if spec[0] == "icosphere":
            assert 2 <= spec[1] <= 6 and v.shape[0] == 10 * 4 ** spec[1] + 2
        else:
            assert 16 <= spec[1] <= 256 and 8 <= spec[2] <= 128 and v.shape[0] == spec[1] * spec[2]
        assert 1 <= len(q) <= 16 and len(set(q)) == len(q)
        assert all(0 <= s < v.shape[0] for s in q)
    again = packed_workload(3, 256)
    assert again.specs == w.specs and again.queries == w.queries
    assert 256 <= total_queries(w.queries) <= 16 * 256
