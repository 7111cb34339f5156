"""Batched builds: every mesh of a batch gets exactly the octree its own
svo_build gives (bit for bit), in one pass or emitted in waves."""
import numpy as np
import pytest

from conftest import random_mesh

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.depth == b.depth and np.array_equal(a.level_counts, b.level_counts)
    assert a.nodes().tobytes() == b.nodes().tobytes()
    assert a.vertices().tobytes() == b.vertices().tobytes()
    assert a.edges().tobytes() == b.edges().tobytes()
    assert a.keys().tobytes() == b.keys().tobytes()


def _mixed_meshes(oracle_mod, bunny_path):
    import torch
    from svo_b200 import meshgen

    rng = np.random.default_rng(5)
    bunny = oracle_mod.load_obj(bunny_path)
    ico = meshgen.icosphere_l5()
    meshes = [(*random_mesh(1, 40), 16), (*bunny, 64), (ico[0], ico[1], 128), (*random_mesh(2, 300, "sliver"), 32),
              (*random_mesh(3, 80, "grid"), 8), (*random_mesh(4, 60), (16, 32, 8))]
    v, f = meshgen.jittered_icosphere(3, rng)
    meshes.append((v[f].reshape(-1, 3), None, 48))  # soup
    meshes.append((torch.from_numpy(bunny[0]).cuda(), torch.from_numpy(bunny[1]).cuda(), 32))  # device input
    meshes.append(((bunny[0] + np.float32(1e6)).astype(np.float32), bunny[1], 64))  # duplicate-removal path
    return meshes


def test_batch_equals_single_builds(gpu_ctx, oracle_mod, bunny_path):
    meshes = _mixed_meshes(oracle_mod, bunny_path)
    results, st, rc = gpu_ctx.build_batch(meshes)
    assert rc == 0 and st == [0] * len(meshes)
    for (p, t, res), r in zip(meshes, results):
        _same(r, gpu_ctx.build(p, t, res))


def test_batch_with_failing_meshes(gpu_ctx, svo_mod, bunny_path, oracle_mod):
    good = oracle_mod.load_obj(bunny_path)
    pts = np.array([[0, 0, 0], [1, 1, 1], [0.5, 0.2, 0.1]], dtype=np.float32)
    nan = pts.copy()
    nan[1, 1] = np.nan
    meshes = [(*good, 32), (pts, np.zeros((0, 3), np.int32), 8), (*good, 16), (pts, np.array([[0, 1, 2]], np.int32), 1),
              (nan, np.array([[0, 1, 2]], np.int32), 8), (pts, np.array([[0, 1, 7]], np.int32), 8), (*good, 0), (*good, 64)]
    results, st, rc = gpu_ctx.build_batch(meshes)
    assert st == [0, svo_mod.ERR_EMPTY, 0, svo_mod.ERR_DEGENERATE, svo_mod.ERR_INVALID_ARGUMENT,
                  svo_mod.ERR_INVALID_ARGUMENT, svo_mod.ERR_UNSUPPORTED, 0]
    assert rc == svo_mod.ERR_EMPTY
    for i in (0, 2, 7):
        _same(results[i], gpu_ctx.build(*meshes[i]))


def test_two_phase_waves(gpu_ctx, svo_mod, oracle_mod, bunny_path):
    meshes = _mixed_meshes(oracle_mod, bunny_path)
    b = gpu_ctx.batch(meshes)
    assert len(b) == len(meshes)
    singles = [gpu_ctx.build(p, t, res) for p, t, res in meshes]
    for i, s in enumerate(singles):
        assert b.nodes(i) == s.num_nodes
        assert b.output_bytes(i) == s.num_nodes * (168 + 128 + 336) + 8 * s.num_keys
    for first, count in ((0, 3), (3, 4), (7, len(meshes) - 7)):
        rs, st, rc = b.emit(first, count)
        assert rc == 0
        for k, r in enumerate(rs):
            _same(r, singles[first + k])
            r.close()
    _, st, rc = b.emit(0, 1)  # a mesh is emitted once
    assert st == [svo_mod.ERR_INVALID_ARGUMENT]
    b.close()


def test_mixed_flags(gpu_ctx, svo_mod, bunny_path, oracle_mod):
    v, f = oracle_mod.load_obj(bunny_path)
    flags = [0, svo_mod.FLAG_STRICT_FP, svo_mod.FLAG_FULL_NEIGHBORS, svo_mod.FLAG_NO_VERT_EDGE, 0]
    meshes = [(v, f, 32 + 8 * i, fl) for i, fl in enumerate(flags)]
    results, st, rc = gpu_ctx.build_batch(meshes)
    assert rc == 0
    for (p, t, res, fl), r in zip(meshes, results):
        s = gpu_ctx.build(p, t, res, fl)
        assert r.nodes().tobytes() == s.nodes().tobytes()
        assert r.vertices().tobytes() == s.vertices().tobytes()


def test_batch_distribution_slice(gpu_ctx, svo_mod):
    from svo_b200 import meshgen

    meshes = meshgen.batch(24, seed=3)
    results, st, rc = gpu_ctx.build_batch(meshes, svo_mod.FLAG_NO_VERT_EDGE)
    assert rc == 0
    for (p, t, res), r in zip(meshes, results):
        s = gpu_ctx.build(p, t, res, svo_mod.FLAG_NO_VERT_EDGE)
        assert r.nodes().tobytes() == s.nodes().tobytes()
        assert r.keys().tobytes() == s.keys().tobytes()


def test_autotune_keeps_results(gpu_ctx, svo_mod):
    """The autotuner only changes the voxelizer work split, never the octree."""
    from svo_b200 import meshgen

    meshes = meshgen.batch(12, seed=5)
    ref, st, rc = gpu_ctx.build_batch(meshes, svo_mod.FLAG_NO_VERT_EDGE)
    assert rc == 0
    saved = gpu_ctx.tuning
    try:
        t = gpu_ctx.autotune(meshes, svo_mod.FLAG_NO_VERT_EDGE)
        assert gpu_ctx.tuning == t and t[0] > 0 and t[1] > 0
        got, st, rc = gpu_ctx.build_batch(meshes, svo_mod.FLAG_NO_VERT_EDGE)
        assert rc == 0
        for a, b in zip(ref, got):
            assert a.nodes().tobytes() == b.nodes().tobytes()
            assert a.keys().tobytes() == b.keys().tobytes()
    finally:
        gpu_ctx.tuning = saved


def test_tuning_variants_keep_results(gpu_ctx, svo_mod):
    """Every voxelizer work split (tier thresholds, serial-tier row layout,
    queue entry size, sub-brick culling) gives the same octree."""
    from svo_b200 import meshgen

    meshes = meshgen.batch(6, seed=11)
    pts, tris, _ = meshgen.torus_slivers(20000)
    meshes.append((pts, tris, 128))
    meshes.append((pts, tris, 512))
    saved = gpu_ctx.tuning
    try:
        ref = [gpu_ctx.build(p, t, r, svo_mod.FLAG_NO_VERT_EDGE) for p, t, r in meshes]
        for tune in [(64, 256, 0, 32, 0), (64, 256, 0, 32, 1), (1, 256, 0, 32, 1), (4096, 256, 0, 32, 1),
                     (0, 7, 1, 0, 1), (256, 1024, 0, 64, 0), (256, 64, 1, 16, 1)]:
            gpu_ctx.tuning = tune
            assert gpu_ctx.tuning == tune
            for (p, t, r), a in zip(meshes, ref):
                b = gpu_ctx.build(p, t, r, svo_mod.FLAG_NO_VERT_EDGE)
                assert a.nodes().tobytes() == b.nodes().tobytes(), tune
                assert a.keys().tobytes() == b.keys().tobytes(), tune
        with pytest.raises(svo_mod.SvoError):
            gpu_ctx.tuning = (1 << 17, 256, 0, 32, 1)
        with pytest.raises(svo_mod.SvoError):
            gpu_ctx.tuning = (64, 256, 0, 32, 2)
    finally:
        gpu_ctx.tuning = saved
