"""Morton-keyed unique vertex/edge/face keys (SVO_FLAG_DEDUP) against the
oracle's sort+unique lists.  The reference has no such lists (README.md:11
promises them), so these semantics are pinned by the oracle alone."""
import numpy as np
import pytest

from conftest import random_mesh

pytestmark = pytest.mark.gpu


def _check(gpu_ctx, svo_mod, oracle_mod, pts, tris, res, extra=0):
    o = oracle_mod.build_svo(pts, tris, res, oracle_mod.FLAG_DEDUP | (extra & oracle_mod.FLAG_FULL_NEIGHBORS))
    g = gpu_ctx.build(pts, tris, res, svo_mod.FLAG_DEDUP | extra)
    for k in range(3):
        d = g.dedup(k)
        assert d.shape == o.dedup[k].shape, (k, d.shape, o.dedup[k].shape)
        assert np.array_equal(d, o.dedup[k]), k
    return g


@pytest.mark.parametrize("res", [2, 4, 16, 64, 128, 256])
def test_bunny(gpu_ctx, svo_mod, oracle_mod, bunny_path, res):
    v, f = oracle_mod.load_obj(bunny_path)
    _check(gpu_ctx, svo_mod, oracle_mod, v, f, res)


@pytest.mark.parametrize("seed,n,kind,res", [(1, 40, "blob", 16), (3, 80, "grid", 8), (2, 300, "sliver", 64),
                                             (4, 60, "blob", (16, 32, 8)), (5, 3, "blob", 2), (7, 200, "grid", (64, 8, 128))])
def test_random(gpu_ctx, svo_mod, oracle_mod, seed, n, kind, res):
    v, f = random_mesh(seed, n, kind)
    _check(gpu_ctx, svo_mod, oracle_mod, v, f, res)


def test_with_full_neighbors_and_keys_off(gpu_ctx, svo_mod, oracle_mod, bunny_path):
    v, f = oracle_mod.load_obj(bunny_path)
    _check(gpu_ctx, svo_mod, oracle_mod, v, f, 64, svo_mod.FLAG_FULL_NEIGHBORS)
    g = _check(gpu_ctx, svo_mod, oracle_mod, v, f, 32, svo_mod.FLAG_NO_VERT_EDGE | svo_mod.FLAG_NO_KEYS)
    assert g.num_vertices == 0


def test_icosphere_c1(gpu_ctx, svo_mod, oracle_mod):
    from svo_b200 import meshgen

    v, f, _ = meshgen.icosphere_l5()
    _check(gpu_ctx, svo_mod, oracle_mod, v, f, 128)


def test_batch_dedup(gpu_ctx, svo_mod, oracle_mod, bunny_path):
    v, f = oracle_mod.load_obj(bunny_path)
    meshes = [(v, f, 16), (*random_mesh(1, 40), 32), (v, f, 64)]
    results, st, rc = gpu_ctx.build_batch(meshes, svo_mod.FLAG_DEDUP)
    assert rc == 0
    for (p, t, res), r in zip(meshes, results):
        o = oracle_mod.build_svo(p, t, res, oracle_mod.FLAG_DEDUP)
        for k in range(3):
            assert np.array_equal(r.dedup(k), o.dedup[k])


def test_properties_res1024(gpu_ctx, svo_mod):
    """Sorted, unique, and consistent with the node set at a size the oracle
    is slow on: every vertex key decodes to a corner of some node."""
    from svo_b200 import meshgen

    v, f, _ = meshgen.icosphere_l5()
    g = gpu_ctx.build(v, f, 1024, svo_mod.FLAG_DEDUP)
    for k in range(3):
        d = g.dedup(k)
        assert d.size > 0 and np.all(d[1:] > d[:-1])
    verts, edges, faces = g.dedup(0), g.dedup(1), g.dedup(2)
    # the low 6 bits of edge/face keys: level < depth, axis < 3
    for keys in (edges, faces):
        assert np.all((keys & 3) < 3) and np.all(((keys >> 2) & 15) < g.depth)
        # each edge/face starts at a vertex
        assert np.all(np.isin(keys >> np.uint64(6), verts))
    # the level-0 vertex count: every leaf-level node has 8 corners, shared
    assert verts.size < 8 * g.level_counts[0]
