"""Level-0 regions at resolutions >= 1024: only the 64x64x32-voxel regions
that some triangle's bbox reaches are zeroed and read, so bits left in pool
memory by earlier builds must never show up in a later octree."""
import numpy as np
import pytest

from parity import assert_same

pytestmark = pytest.mark.gpu


def _scattered(seed, n, size):
    """n small triangles at random places in the unit cube (few voxels, many
    untouched regions)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.0, 1.0, size=(n, 1, 3))
    t = c + rng.normal(size=(n, 3, 3)) * size
    t[0, 0] = 0.0  # corners pin the grid to the unit cube
    t[1, 0] = 1.0
    return t.reshape(-1, 3).astype(np.float32), np.arange(3 * n, dtype=np.int32).reshape(-1, 3)


def _dirty(gpu_ctx):
    """A dense res-2048 build whose bitmap memory goes back to the pool."""
    from svo_b200 import meshgen

    v, f, _ = meshgen.heightfield(600)
    gpu_ctx.build(v, f, 2048).close()


@pytest.mark.parametrize("res", [1024, 2048, (2048, 1024, 1536)])
def test_sparse_after_dense(gpu_ctx, oracle_mod, svo_mod, res):
    _dirty(gpu_ctx)
    v, f = _scattered(3, 120, 0.002)
    g = gpu_ctx.build(v, f, res, svo_mod.FLAG_NO_VERT_EDGE)
    o = oracle_mod.build_svo(v, f, res, flags=oracle_mod.FLAG_NO_VERT_EDGE)
    assert_same(g, o, check_ve=False)


def test_batch_mixes_region_meshes(gpu_ctx, oracle_mod, svo_mod):
    """Region-mode meshes next to small ones in one batch, after a dense build."""
    _dirty(gpu_ctx)
    meshes = [(*_scattered(4, 60, 0.003), 2048), (*_scattered(5, 40, 0.01), 64), (*_scattered(6, 200, 0.001), 1024),
              (*_scattered(7, 30, 0.02), 128)]
    results, st, rc = gpu_ctx.build_batch(meshes, svo_mod.FLAG_NO_VERT_EDGE)
    assert rc == 0 and st == [0] * len(meshes)
    for (p, t, res), r in zip(meshes, results):
        o = oracle_mod.build_svo(p, t, res, flags=oracle_mod.FLAG_NO_VERT_EDGE)
        assert_same(r, o, check_ve=False)
