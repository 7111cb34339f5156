"""Structural checks of the oracle's octree (the reference's create()
semantics, src/SVO.cu:341-735) on small meshes."""
import numpy as np
import pytest

from conftest import random_mesh

NONE = 0xFFFFFFFF


def _levels(r):
    off = np.concatenate([[0], np.cumsum(r.level_counts)])
    return off


def _coords(code):
    x = y = z = 0
    for i in range(21):
        x |= ((code >> (3 * i)) & 1) << i
        y |= ((code >> (3 * i + 1)) & 1) << i
        z |= ((code >> (3 * i + 2)) & 1) << i
    return x, y, z


@pytest.mark.parametrize("seed,res", [(0, 8), (1, 16), (2, 5), (3, 32)])
def test_tree_structure(oracle_mod, seed, res):
    v, f = random_mesh(seed, 40)
    r = oracle_mod.build_svo(v, f, res)
    n = r.nodes
    off = _levels(r)
    assert off[-1] == len(n) and r.level_counts[-1] == 1
    assert r.depth == len(r.level_counts)
    # groups of 8 siblings with consecutive codes
    for l in range(r.depth - 1):
        codes = n["morton_code"][off[l]:off[l + 1]].astype(np.int64)
        assert (codes.reshape(-1, 8) == (codes.reshape(-1, 8)[:, :1] // 8 * 8 + np.arange(8))).all()
    # parent/child links are mutual
    for i, node in enumerate(n):
        for k, c in enumerate(node["childs"]):
            if c != NONE:
                assert n[c]["parent"] == i
                assert n[c]["morton_code"] == node["morton_code"] * 8 + k
        if node["parent"] != NONE:
            assert i in n[node["parent"]]["childs"].tolist()
    # every non-root node has a parent; leaves have no children
    assert (n["parent"][:-1] != NONE).all() and n["parent"][-1] == NONE
    assert ((n["is_leaf"] == 1) == (n["childs"][:, 0] == NONE)).all()
    # level-1 real nodes are exactly the surface voxels
    lvl0 = set(n["morton_code"][: off[1]].tolist())
    assert set(r.keys.tolist()) <= lvl0


def test_effective_neighbors_and_owners(oracle_mod):
    v, f = random_mesh(5, 30)
    r = oracle_mod.build_svo(v, f, 16)
    nb = r.nodes["neighbors"]
    N = len(r.nodes)
    expect = np.full_like(nb, NONE)
    expect[-1, 13] = N - 1  # only the root's self entry survives (src/SVO.cu:535-542)
    assert np.array_equal(nb, expect)
    assert len(r.vertices) == 8 * N and len(r.edges) == 12 * N
    assert np.array_equal(r.vertices["owner"], np.repeat(np.arange(N, dtype=np.uint32), 8))
    assert np.array_equal(r.edges["owner"], np.repeat(np.arange(N, dtype=np.uint32), 12))
    w = np.repeat(r.nodes["width"], 8)
    bits = np.tile(np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=np.float32), (N, 1))
    assert np.array_equal(r.vertices["pos"], (w[:, None] * bits).astype(np.float32))


@pytest.mark.parametrize("seed", [0, 1])
def test_full_neighbors_brute_force(oracle_mod, seed):
    v, f = random_mesh(seed, 25)
    r = oracle_mod.build_svo(v, f, 16, flags=oracle_mod.FLAG_FULL_NEIGHBORS)
    n = r.nodes
    off = _levels(r)
    for l in range(r.depth):
        idx = {int(n["morton_code"][t]): t for t in range(off[l], off[l + 1])}
        for t in range(off[l], off[l + 1]):
            x, y, z = _coords(int(n["morton_code"][t]))
            for j in range(27):
                d = (j % 3 - 1, (j // 3) % 3 - 1, j // 9 - 1)
                q = (x + d[0], y + d[1], z + d[2])
                want = NONE
                if min(q) >= 0:
                    want = idx.get(oracle_mod.morton_encode(*q), NONE)
                if l == r.depth - 1:
                    want = t if j == 13 else NONE
                assert n["neighbors"][t, j] == want, (l, t, j)


def test_dedup_keys(oracle_mod):
    v, f = random_mesh(2, 20)
    r = oracle_mod.build_svo(v, f, 8, flags=oracle_mod.FLAG_DEDUP)
    off = _levels(r)
    verts = set()
    for l in range(r.depth):
        s = 1 << l
        for t in range(off[l], off[l + 1]):
            x, y, z = (c << l for c in _coords(int(r.nodes["morton_code"][t])))
            for i in range(8):
                verts.add(oracle_mod.morton_encode(x + s * (i & 1), y + s * ((i >> 1) & 1), z + s * ((i >> 2) & 1)))
    assert r.dedup[0].tolist() == sorted(verts)
    assert (np.diff(r.dedup[1].astype(np.float64)) > 0).all() and (np.diff(r.dedup[2].astype(np.float64)) > 0).all()


def test_error_cases(oracle_mod):
    pts = np.array([[0, 0, 0], [1, 1, 1], [0.5, 0.2, 0.1]], dtype=np.float32)
    with pytest.raises(oracle_mod.OracleError) as e:
        oracle_mod.build_svo(pts, np.zeros((0, 3), np.int32), 8)
    assert e.value.code == 4  # no surface voxels: the reference aborts
    with pytest.raises(oracle_mod.OracleError) as e:
        oracle_mod.build_svo(pts, np.array([[0, 1, 2]], np.int32), 1)
    assert e.value.code == 5  # a single voxel: undefined in the reference
    bad = pts.copy()
    bad[1, 1] = np.nan
    with pytest.raises(oracle_mod.OracleError):
        oracle_mod.build_svo(bad, np.array([[0, 1, 2]], np.int32), 8)


def test_depth_power_of_two(oracle_mod):
    v, f = random_mesh(0, 60)
    for res in (2, 4, 8, 16, 32, 64):
        r = oracle_mod.build_svo(v, f, res, flags=oracle_mod.FLAG_NO_VERT_EDGE)
        assert r.depth == int(np.log2(res)) + 1
