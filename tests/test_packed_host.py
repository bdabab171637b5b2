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


def test_mesh_bounds_match_each_mesh_alone() -> None:
    """The union's per-mesh bounding boxes (one reduceat pass) are each mesh's own float32
    extremes, empty meshes included."""
    import numpy as np

    from ordito_b200.packed import mesh_bounds

    w = packed_workload(5, 40)
    verts = [np.ascontiguousarray(v, dtype=np.float32).reshape(-1, 3) for v, _ in w.meshes]
    verts.insert(7, np.zeros((0, 3), dtype=np.float32))  # an empty mesh in between
    verts.append(np.zeros((0, 3), dtype=np.float32))     # and one at the end
    offsets = np.zeros(len(verts) + 1, dtype=np.int32)
    np.cumsum([v.shape[0] for v in verts], out=offsets[1:])
    low, high, nonempty = mesh_bounds(np.concatenate(verts), offsets)
    assert list(nonempty) == [m for m, v in enumerate(verts) if v.shape[0]]
    for m, v in enumerate(verts):
        if v.shape[0]:
            assert np.array_equal(low[m], v.min(axis=0)) and np.array_equal(high[m], v.max(axis=0))
        else:
            assert not low[m].any() and not high[m].any()
