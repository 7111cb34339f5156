"""GPU build (C ABI, sm_100a kernels) against the oracle, bit for bit."""
import numpy as np
import pytest

from conftest import random_mesh
from parity import assert_same

pytestmark = pytest.mark.gpu


def _both(ctx, oracle_mod, v, f, res, flags=0):
    g = ctx.build(v, f, res, flags)
    o = oracle_mod.build_svo(v, f, res, flags)
    return g, o


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("res", [2, 3, 5, 8, 16, 33, 64])
def test_random_blobs(gpu_ctx, oracle_mod, seed, res):
    v, f = random_mesh(seed, 60)
    g, o = _both(gpu_ctx, oracle_mod, v, f, res)
    assert_same(g, o)


@pytest.mark.parametrize("kind", ["grid", "sliver"])
@pytest.mark.parametrize("res", [8, 32, 128])
def test_hard_triangles(gpu_ctx, oracle_mod, kind, res):
    v, f = random_mesh(11, 200, kind)
    g, o = _both(gpu_ctx, oracle_mod, v, f, res)
    assert_same(g, o)


@pytest.mark.parametrize("res", [16, 64, 128, 256])
def test_bunny(gpu_ctx, oracle_mod, bunny_path, res):
    v, f = oracle_mod.load_obj(bunny_path)
    g, o = _both(gpu_ctx, oracle_mod, v, f, res)
    assert_same(g, o)


def test_icosphere_l5(gpu_ctx, oracle_mod):
    from svo_b200 import meshgen

    v, f, res = meshgen.icosphere_l5()
    g, o = _both(gpu_ctx, oracle_mod, v, f, res)
    assert g.num_nodes == 221177 and g.depth == 8
    assert_same(g, o)


@pytest.mark.parametrize("flags", ["strict", "full", "full_strict", "no_ve"])
def test_modes(gpu_ctx, oracle_mod, bunny_path, flags, svo_mod):
    fl = {"strict": svo_mod.FLAG_STRICT_FP, "full": svo_mod.FLAG_FULL_NEIGHBORS,
          "full_strict": svo_mod.FLAG_FULL_NEIGHBORS | svo_mod.FLAG_STRICT_FP,
          "no_ve": svo_mod.FLAG_NO_VERT_EDGE}[flags]
    v, f = oracle_mod.load_obj(bunny_path)
    g, o = _both(gpu_ctx, oracle_mod, v, f, 64, fl)
    assert_same(g, o, check_ve=flags != "no_ve")
    if flags == "no_ve":
        assert g.num_vertices == 0 and g.num_edges == 0


def test_anisotropic(gpu_ctx, oracle_mod):
    v, f = random_mesh(4, 80)
    g, o = _both(gpu_ctx, oracle_mod, v, f, (16, 32, 8))
    assert_same(g, o)


def test_soup_equals_indexed(gpu_ctx, oracle_mod):
    from svo_b200 import meshgen

    v, f = meshgen.jittered_icosphere(3, np.random.default_rng(6))
    soup = v[f].reshape(-1, 3)
    a = gpu_ctx.build(v, f, 32)
    b = gpu_ctx.build(soup, None, 32)
    o = oracle_mod.build_svo(soup, np.arange(soup.shape[0], dtype=np.int32).reshape(-1, 3), 32)
    assert_same(b, o)
    # every vertex is referenced: same bbox, so the same tree as the indexed mesh
    assert a.nodes().tobytes() == b.nodes().tobytes()


def test_device_input(gpu_ctx, oracle_mod, bunny_path):
    import torch

    v, f = oracle_mod.load_obj(bunny_path)
    dv = torch.from_numpy(v).cuda()
    df = torch.from_numpy(f).cuda()
    g = gpu_ctx.build(dv, df, 64)
    o = oracle_mod.build_svo(v, f, 64)
    assert_same(g, o)


def test_far_offset_duplicates(gpu_ctx, oracle_mod, bunny_path):
    """Far from the origin the edge corners absorb the node width: the
    consecutive-unique pass (src/SVO.cu:718-722) then really removes edges."""
    v, f = oracle_mod.load_obj(bunny_path)
    v = (v + np.float32(1.0e6)).astype(np.float32)
    g, o = _both(gpu_ctx, oracle_mod, v, f, 64)
    assert len(o.edges) < 12 * len(o.nodes) // 2
    assert_same(g, o)


def test_repeat_builds_identical(gpu_ctx, bunny_path, oracle_mod):
    v, f = oracle_mod.load_obj(bunny_path)
    a = gpu_ctx.build(v, f, 128)
    b = gpu_ctx.build(v, f, 128)
    assert a.nodes().tobytes() == b.nodes().tobytes()
    assert a.edges().tobytes() == b.edges().tobytes()


def test_errors(gpu_ctx, svo_mod):
    pts = np.array([[0, 0, 0], [1, 1, 1], [0.5, 0.2, 0.1]], dtype=np.float32)
    cases = [
        (pts, np.zeros((0, 3), np.int32), 8, svo_mod.ERR_EMPTY),
        (pts, np.array([[0, 1, 2]], np.int32), 1, svo_mod.ERR_DEGENERATE),
        (pts, np.array([[0, 1, 3]], np.int32), 8, svo_mod.ERR_INVALID_ARGUMENT),
        (pts, np.array([[0, 1, 2]], np.int32), 0, svo_mod.ERR_UNSUPPORTED),
        (pts, np.array([[0, 1, 2]], np.int32), 4096, svo_mod.ERR_UNSUPPORTED),
    ]
    bad = pts.copy()
    bad[1, 1] = np.nan
    cases.append((bad, np.array([[0, 1, 2]], np.int32), 8, svo_mod.ERR_INVALID_ARGUMENT))
    for p, f, res, code in cases:
        with pytest.raises(svo_mod.SvoError) as e:
            gpu_ctx.build(p, f, res)
        assert e.value.code == code, (res, e.value)
    # the context stays usable after errors
    r = gpu_ctx.build(pts, np.array([[0, 1, 2]], np.int32), 8)
    assert r.depth == 4


def _tiny_meshes(count: int):
    """Meshes of 1 to 8 triangles on small grids (2 to 16 per axis): random,
    lattice-aligned and zero-area triangles, and triangles clustered in one
    corner of a bounding cube stretched by an unused vertex -- tiny ones give a
    single surface voxel, larger ones a single top node in a non-zero octant,
    the two inputs the reference has no defined build for."""
    out = []
    for seed in range(count):
        rng = np.random.default_rng(1000 + seed)
        n = 1 + seed % 8
        kind = seed % 5
        tris = np.arange(n * 3, dtype=np.int32).reshape(-1, 3)
        if kind == 0:
            v = rng.normal(size=(n * 3, 3))
        elif kind == 1:
            v = rng.integers(0, 5, size=(n * 3, 3)) / 4.0
        elif kind == 2:  # repeated vertices: zero-area triangles
            v = np.repeat(rng.normal(size=(n, 3)), 3, axis=0)
        else:  # clustered near (1, 1, 1); the last vertex, at the origin, is used by no triangle
            spread = 0.3 if kind == 3 else 1e-4
            v = np.concatenate([1.0 - rng.uniform(0.0, spread, size=(n * 3, 3)), [[0.0, 0.0, 0.0]]])
        res = (2, 3, 4, 5, 8, 16, 7)[seed % 7]
        out.append((v.astype(np.float32), tris, res))
    return out


def test_tiny_meshes_exhaustive(gpu_ctx, oracle_mod, svo_mod):
    """Every tiny mesh, built in one batch, against the oracle: the same
    status, and where the build is defined, the same octree bit for bit."""
    meshes = _tiny_meshes(336)
    results, st, _ = gpu_ctx.build_batch(meshes)
    seen = set()
    for (v, f, res), r, s in zip(meshes, results, st):
        try:
            o = oracle_mod.build_svo(v, f, res)
        except oracle_mod.OracleError as e:
            assert s == e.code and r is None, (res, s, e.code)
            seen.add(e.code)
            continue
        assert s == svo_mod.OK, (res, s)
        assert_same(r, o)
        seen.add(0)
        r.close()
    assert {0, svo_mod.ERR_DEGENERATE} <= seen
