"""The allocation-free voxel-key entry point, through the C ABI.

Some callers cannot let the library allocate device memory (they own every
byte through their own arena, or an allocation's implicit synchronisation
would break their stream work).  svo_voxelize_keys_noalloc serves them with
caller-owned inputs and outputs plus a fixed scratch array inside the library.
Its keys must equal the ones svo_build produces, bit for bit, call after call
(the scratch array keeps the previous call's contents, which must not leak).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fn(svo_mod):
    f = svo_mod.lib().svo_voxelize_keys_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_uint32,
                  C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.c_void_p]
    return f


def _noalloc_keys(svo_mod, v, f, res):
    import torch

    fn = _fn(svo_mod)
    dv = torch.from_numpy(v).cuda()
    df = torch.from_numpy(f).cuda() if f is not None else None
    cap = 1 << 22
    out = torch.full((cap,), -1, dtype=torch.int64, device="cuda")
    n = C.c_int64()
    rc = fn(dv.data_ptr(), v.shape[0], df.data_ptr() if df is not None else None, 0 if f is None else f.shape[0],
            res, res, res, 0, out.data_ptr(), cap, C.byref(n), None)
    if rc != 0:
        raise svo_mod.SvoError(rc, svo_mod.lib().svo_last_error().decode())
    return out[: n.value].cpu().numpy().view(np.uint64)


def test_noalloc_matches_build_two_calls(gpu_ctx, svo_mod, oracle_mod, bunny_path):
    from svo_b200 import meshgen

    bunny = oracle_mod.load_obj(bunny_path)
    ico = meshgen.icosphere_l5()[:2]
    # two different meshes back to back, then the first again
    for (v, f), res in ((bunny, 64), (ico, 128), (bunny, 64)):
        want = gpu_ctx.build(v, f, res, svo_mod.FLAG_NO_VERT_EDGE).keys()
        got = _noalloc_keys(svo_mod, v, f, res)
        assert got.shape == want.shape and np.array_equal(got, want)


def _axis_mesh():
    """Large axis-aligned triangles across the unit cube (planes normal to each
    axis) plus a triangle from corner to corner that fixes the bounding cube."""
    t = [[(0, 0, .5), (1, 0, .5), (0, 1, .5)], [(1, 1, .25), (0, 1, .25), (1, 0, .25)],
         [(.3, 0, 0), (.3, 1, 0), (.3, 0, 1)], [(0, .7, 0), (0, .7, 1), (1, .7, 1)],
         [(0, 0, 0), (1, 1, 1), (1, 0, 1)]]
    v = np.array(t, dtype=np.float32).reshape(-1, 3)
    return v, np.arange(v.shape[0], dtype=np.int32).reshape(-1, 3)


@pytest.mark.parametrize("res", [128, 256])
@pytest.mark.parametrize("kind", ["blob", "sliver", "axis"])
def test_noalloc_large_triangles(gpu_ctx, svo_mod, oracle_mod, kind, res):
    """Triangles whose grid boxes span many 4x4x4 bricks.  This entry point
    has no queue for them (it allocates none), so the warp that set a
    triangle up walks all of its bricks; the keys must still equal the
    oracle's voxelization and svo_build's, at the largest resolution (256)
    too, on two calls in a row."""
    from conftest import random_mesh

    v, f = _axis_mesh() if kind == "axis" else random_mesh(11, 40 if kind == "blob" else 300, kind)
    want = oracle_mod.voxelize(v, f, res)
    assert want.size > 0
    for _ in range(2):
        got = _noalloc_keys(svo_mod, v, f, res)
        assert got.shape == want.shape and np.array_equal(got, want)
    assert np.array_equal(gpu_ctx.build(v, f, res, svo_mod.FLAG_NO_VERT_EDGE).keys(), want)


def test_noalloc_rejects_large_resolution_and_host_memory(gpu_ctx, svo_mod):
    import torch

    fn = _fn(svo_mod)
    v = np.random.default_rng(0).normal(size=(30, 3)).astype(np.float32)
    f = np.arange(30, dtype=np.int32).reshape(-1, 3)
    out = torch.empty(1024, dtype=torch.int64, device="cuda")
    n = C.c_int64()
    dv, df = torch.from_numpy(v).cuda(), torch.from_numpy(f).cuda()
    assert fn(dv.data_ptr(), 30, df.data_ptr(), 10, 512, 512, 512, 0, out.data_ptr(), 1024, C.byref(n), None) == \
        svo_mod.ERR_UNSUPPORTED
    assert fn(v.ctypes.data, 30, f.ctypes.data, 10, 64, 64, 64, 0, out.data_ptr(), 1024, C.byref(n), None) == \
        svo_mod.ERR_INVALID_ARGUMENT
