"""Shared comparison of a GPU build (C ABI) with the oracle's build."""
import numpy as np

FIELDS = ["morton_code", "is_leaf", "origin", "width", "parent", "childs", "neighbors"]


def first_diff(a: np.ndarray, b: np.ndarray, what: str, chunk: int = 1 << 22) -> str:
    """'' if a and b are byte-identical, else a description of the first
    differing record.  Compares `chunk` records at a time (multi-GB arrays)."""
    if a.shape != b.shape:
        return f"{what}: shape {a.shape} vs {b.shape}"
    n = a.shape[0] if a.ndim else 1
    nbad, i = 0, -1
    for s in range(0, n, chunk):
        ab = a[s:s + chunk].view(np.uint8).reshape(-1, a.itemsize)
        bb = b[s:s + chunk].view(np.uint8).reshape(-1, b.itemsize)
        bad = np.nonzero((ab != bb).any(1))[0]
        if bad.size:
            nbad += bad.size
            if i < 0:
                i = s + int(bad[0])
    if i < 0:
        return ""
    msg = f"{what}: {nbad} records differ, first at {i}"
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
