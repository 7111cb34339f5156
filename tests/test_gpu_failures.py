"""Failure detection, tested without faulting the GPU.

The reference ends the process on any CUDA error (CUDA_CHECK and
getLastCudaError call exit(), src/CUDAUtil.h:21-48).  This library returns a
status and keeps the context usable.  Each test provokes one failure a build
can meet -- a device-side wait that runs out (the scan's bounded look-back,
given a predecessor that never publishes), a device allocation that fails
(injected on the host at every allocation a build makes), a served request
withdrawn before it runs -- then checks the status, that no device memory is
left behind, and that the same context builds the mesh again exactly as the
oracle does.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import random_mesh
from parity import assert_same

pytestmark = pytest.mark.gpu


def _idle_memory(ctx):
    torch.cuda.synchronize()
    return ctx.memory()


def test_scan_wait_runs_out(gpu_ctx, svo_mod, oracle_mod, bunny_path):
    v, f = oracle_mod.load_obj(bunny_path)
    before = _idle_memory(gpu_ctx)
    for _ in range(2):
        assert gpu_ctx.selftest_scan_timeout() == svo_mod.ERR_DEVICE_TIMEOUT
    assert _idle_memory(gpu_ctx) == before
    g = gpu_ctx.build(v, f, 64)
    assert_same(g, oracle_mod.build_svo(v, f, 64))


def test_alloc_failure_at_every_allocation(gpu_ctx, svo_mod, oracle_mod, bunny_path):
    """A failed device allocation at any point of a build (full neighbour
    tables and dedup included) returns SVO_ERR_OUT_OF_MEMORY, frees what the
    build held, and the next build succeeds."""
    v, f = oracle_mod.load_obj(bunny_path)
    flags = svo_mod.FLAG_FULL_NEIGHBORS | svo_mod.FLAG_DEDUP
    gpu_ctx.build(v, f, 64, flags).close()
    base = _idle_memory(gpu_ctx)
    failed = 0
    try:
        for k in range(1, 200):
            svo_mod.debug_fail_alloc(k)
            try:
                g = gpu_ctx.build(v, f, 64, flags)
            except svo_mod.SvoError as e:
                assert e.code == svo_mod.ERR_OUT_OF_MEMORY, (k, str(e))
                assert svo_mod.debug_fail_alloc(0) == 0, k  # the injected failure was the one reported
                failed += 1
                assert _idle_memory(gpu_ctx) == base, k
                continue
            # the build made fewer than k allocations: the injection is still armed
            assert svo_mod.debug_fail_alloc(0) > 0, k
            g.close()
            break
        else:
            pytest.fail("a build made 200 allocations or more")
    finally:
        svo_mod.debug_fail_alloc(0)
    assert failed >= 5
    assert _idle_memory(gpu_ctx) == base
    o = oracle_mod.build_svo(v, f, 64, flags=oracle_mod.FLAG_FULL_NEIGHBORS | oracle_mod.FLAG_DEDUP)
    g = gpu_ctx.build(v, f, 64, flags)
    assert_same(g, o)
    for k in range(3):
        assert np.array_equal(g.dedup(k), o.dedup[k])


def test_batch_alloc_failures_report_every_mesh(gpu_ctx, svo_mod, oracle_mod, bunny_path):
    """In a batch, an allocation failure anywhere leaves every mesh with either
    a result and SVO_OK or no result and a failure status, never a result-less
    SVO_OK; the meshes that did build are correct."""
    from svo_b200 import _descs

    v, f = oracle_mod.load_obj(bunny_path)
    meshes = [(v, f, 16), (*random_mesh(1, 40), 32), (v, f, 64)]
    flags = svo_mod.FLAG_DEDUP
    want = [oracle_mod.build_svo(p, t, r, flags=oracle_mod.FLAG_DEDUP) for p, t, r in meshes]
    L = svo_mod.lib()
    for r in gpu_ctx.build_batch(meshes, flags)[0]:
        r.close()
    base = _idle_memory(gpu_ctx)
    seen_fail = 0
    try:
        for k in range(1, 300):
            descs, keep = _descs(meshes, flags)
            outs = (C.c_void_p * len(meshes))()
            st = (C.c_int * len(meshes))(*([-1] * len(meshes)))
            svo_mod.debug_fail_alloc(k)
            rc = L.svo_build_batch(gpu_ctx.handle, descs, len(meshes), None, outs, st)
            left = svo_mod.debug_fail_alloc(0)
            for i in range(len(meshes)):
                assert (st[i] == svo_mod.OK) == (outs[i] is not None), (k, i, st[i])
                if st[i] != svo_mod.OK:
                    assert st[i] == svo_mod.ERR_OUT_OF_MEMORY, (k, i, st[i])
            if rc != svo_mod.OK:
                assert left == 0 and any(s != svo_mod.OK for s in st), k
                seen_fail += 1
            for i in range(len(meshes)):
                if outs[i] is not None:
                    r = svo_mod.Result(C.c_void_p(outs[i]))
                    assert_same(r, want[i])
                    for d in range(3):
                        assert np.array_equal(r.dedup(d), want[i].dedup[d])
                    r.close()
            assert _idle_memory(gpu_ctx) == base, k
            if rc == svo_mod.OK:
                assert left > 0, k  # no injected failure was swallowed
                break
        else:
            pytest.fail("a batch made 300 allocations or more")
    finally:
        svo_mod.debug_fail_alloc(0)
    assert seen_fail >= 5
