"""Shared comparison of a GPU build (C ABI) with the oracle's build."""
import numpy as np

FIELDS = ["morton_code", "is_leaf", "origin", "width", "parent", "childs", "neighbors"]


def first_diff(a: np.ndarray, b: np.ndarray, what: str) -> str:
    if a.shape != b.shape:
        return f"{what}: shape {a.shape} vs {b.shape}"
    ab = a.view(np.uint8).reshape(a.shape[0], -1) if a.ndim == 1 else a
    bb = b.view(np.uint8).reshape(b.shape[0], -1) if b.ndim == 1 else b
    bad = np.nonzero((ab != bb).reshape(ab.shape[0], -1).any(1))[0]
    if bad.size == 0:
        return ""
    i = int(bad[0])
    msg = f"{what}: {bad.size} records differ, first at {i}"
    if a.dtype.names:
        for f in a.dtype.names:
            if not np.array_equal(a[f][i], b[f][i]):
                msg += f"\n  {f}: gpu={a[f][i]!r} oracle={b[f][i]!r}"
    else:
        msg += f": gpu={a[i]!r} oracle={b[i]!r}"
    return msg


def assert_same(gpu, orc, check_ve=True, check_keys=True):
    """gpu: svo_b200.Result, orc: oracle.Result."""
    assert gpu.depth == orc.depth, (gpu.depth, orc.depth)
    assert np.array_equal(gpu.level_counts, orc.level_counts), (gpu.level_counts, orc.level_counts)
    assert gpu.bbox.tobytes() == orc.bbox.tobytes(), (gpu.bbox, orc.bbox)
    gn = gpu.nodes()
    on = orc.nodes.view(gn.dtype)
    msg = first_diff(gn, on, "nodes")
    assert not msg, msg
    if check_keys:
        assert np.array_equal(gpu.keys(), orc.keys)
    if check_ve:
        gv, ge = gpu.vertices(), gpu.edges()
        msg = first_diff(gv, orc.vertices.view(gv.dtype), "vertices")
        assert not msg, msg
        msg = first_diff(ge, orc.edges.view(ge.dtype), "edges")
        assert not msg, msg
