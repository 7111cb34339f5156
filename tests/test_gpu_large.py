"""Full-size workloads: C2 against the oracle in full, C3 (res 2048, 64-bit
Morton codes) against the oracle on a subsample and through size-independent
properties of the full build."""
import numpy as np
import pytest

from parity import assert_same, first_diff

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
NONE = 0xFFFFFFFF


def test_torus_slivers_full(gpu_ctx, oracle_mod, svo_mod):
    from svo_b200 import meshgen

    soup, _, res = meshgen.torus_slivers()
    g = gpu_ctx.build(soup, None, res)
    o = oracle_mod.build_svo(soup, np.arange(soup.shape[0], dtype=np.int32).reshape(-1, 3), res,
                             flags=oracle_mod.FLAG_NO_VERT_EDGE)
    assert_same(g, o, check_ve=False)
    # vertex / edge arrays are a pure function of the node records
    n = g.nodes()
    N = n.shape[0]
    assert g.num_vertices == 8 * N and g.num_edges == 12 * N
    v = g.vertices().reshape(N, 8)
    bits = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=np.float32)
    assert np.array_equal(v["pos"], (n["width"][:, None, None] * bits[None]).astype(np.float32))
    assert np.array_equal(v["owner"], np.repeat(np.arange(N, dtype=np.uint32), 8).reshape(N, 8))


def _heightfield_sample(stride):
    from svo_b200 import meshgen

    v, f, res = meshgen.heightfield()
    return v, f[::stride], res


def test_heightfield_subsample_res2048(gpu_ctx, oracle_mod, svo_mod):
    v, f, res = _heightfield_sample(7)
    g = gpu_ctx.build(v, f, res, svo_mod.FLAG_NO_VERT_EDGE)
    o = oracle_mod.build_svo(v, f, res, flags=oracle_mod.FLAG_NO_VERT_EDGE)
    assert o.depth == 12 and (o.keys >= 1 << 32).any()  # codes above 32 bits are exercised
    assert_same(g, o, check_ve=False)


def _assert_dedup(g, o):
    for k in range(3):
        d = g.dedup(k)
        assert d.shape == o.dedup[k].shape, (k, d.shape, o.dedup[k].shape)
        assert np.array_equal(d, o.dedup[k]), k


def test_heightfield_subsample_res2048_full_dedup(gpu_ctx, oracle_mod, svo_mod):
    """The heightfield workload's own flags -- full 27-neighbour tables and the
    vertex/edge/face dedup lists -- at resolution 2048 (64-bit Morton codes) on
    every 7th triangle: node records with all neighbours, the vertex/edge
    arrays (owner = smallest sharing node), the voxel keys and the three dedup
    lists, element for element against the oracle."""
    v, f, res = _heightfield_sample(7)
    g = gpu_ctx.build(v, f, res, svo_mod.FLAG_FULL_NEIGHBORS | svo_mod.FLAG_DEDUP)
    o = oracle_mod.build_svo(v, f, res, flags=oracle_mod.FLAG_FULL_NEIGHBORS | oracle_mod.FLAG_DEDUP)
    assert o.depth == 12 and (o.keys >= 1 << 32).any()
    # neighbour tables are really populated (not just the root's self entry):
    # every node below the root sees itself and its 7 siblings
    nb = o.nodes["neighbors"][:-1]
    assert (nb[:, 13] != NONE).all() and (nb != NONE).sum(1).min() >= 8
    assert_same(g, o)
    _assert_dedup(g, o)


@pytest.mark.parametrize("mode", ["full", "dedup"])
def test_icosphere_res1024(gpu_ctx, oracle_mod, svo_mod, mode):
    """The icosphere (config 1's mesh) at resolution 1024, the largest grid of
    32-bit Morton codes, with full neighbour tables or with dedup lists, in
    full against the oracle."""
    from svo_b200 import meshgen

    v, f, _ = meshgen.icosphere_l5()
    gf = svo_mod.FLAG_FULL_NEIGHBORS if mode == "full" else svo_mod.FLAG_DEDUP
    of = oracle_mod.FLAG_FULL_NEIGHBORS if mode == "full" else oracle_mod.FLAG_DEDUP
    g = gpu_ctx.build(v, f, 1024, gf)
    o = oracle_mod.build_svo(v, f, 1024, flags=of)
    assert o.depth == 11
    assert_same(g, o)
    if mode == "dedup":
        _assert_dedup(g, o)


def test_heightfield_full_properties(gpu_ctx, svo_mod):
    from svo_b200 import meshgen

    v, f, res = meshgen.heightfield()
    assert f.shape[0] == 4_999_122
    g = gpu_ctx.build(v, f, res)
    assert g.depth == 12
    lc = g.level_counts
    n = g.nodes()
    keys = g.keys()
    N = n.shape[0]
    assert N == lc.sum() and lc[-1] == 1
    assert np.all(np.diff(keys.astype(np.float64)) > 0) and keys[-1] < (1 << 33)
    off = np.concatenate([[0], np.cumsum(lc)])
    # siblings in groups of 8 with consecutive codes (low 32 bits at level 0)
    for l in range(g.depth - 1):
        c = n["morton_code"][off[l]:off[l + 1]].astype(np.int64).reshape(-1, 8)
        assert np.array_equal(c - c[:, :1], np.broadcast_to(np.arange(8), c.shape))
    # level-0 real nodes are the surface voxels
    real0 = np.isin(n["morton_code"][: off[1]], (keys & 0xFFFFFFFF).astype(np.uint32))
    assert real0.sum() == keys.size
    # parent/child links are mutual everywhere
    has = n["childs"][:, 0] != NONE
    idx = np.nonzero(has)[0]
    ch = n["childs"][idx].astype(np.int64)
    assert np.array_equal(ch - ch[:, :1], np.broadcast_to(np.arange(8), ch.shape))
    assert np.array_equal(n["parent"][ch[:, 0]], idx.astype(np.uint32))
    assert (n["parent"][:-1] != NONE).all() and n["parent"][-1] == NONE
    assert np.array_equal(n["is_leaf"] == 0, has)
    # widths double per level, vertex/edge counts
    w = np.array([n["width"][off[l]] for l in range(g.depth)])
    assert np.array_equal(w[1:], w[:-1] * np.float32(2.0))
    assert g.num_vertices == 8 * N and g.num_edges == 12 * N
