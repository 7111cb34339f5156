"""Checks the oracle's floating-point machinery against nvcc.

The reference's arithmetic is Eigen 3.4 compiled by nvcc with its default
--fmad=true; which products nvcc fuses into FMAs is not visible in the source
and depends on context (loop-invariant products are hoisted before fusion).
The pattern itself is pinned by the reference's own build
(tests/test_ref_pins.py).  Here tests/fp_probe.cu restates the triangle setup
and voxel loop in plain float code with Eigen's evaluation order; built with
default contraction it must agree bit for bit with the oracle's contraction
model, and built with --fmad=false with the oracle's strict model -- on small
shapes, on the setup values and on the complete voxel test, including
lattice-aligned triangles where many tests are decided by the last bit.  In
the probe's restated loop nvcc fuses the third ZX edge test's z product
(a*p.z) where the reference's own loop fuses its x product; the voxel test is
compared under the probe's pattern (PROBE_SITES), everything else under the
reference's.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

# the oracle's contraction sites as nvcc fuses them in the probe's loop: the
# reference's pattern with the third ZX test fusing its first product
PROBE_SITES = [0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 0]
REFERENCE_SITES = [0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1]


@pytest.fixture(scope="module")
def probes(tmp_path_factory):
    out = {}
    d = tmp_path_factory.mktemp("fp_probe")
    src = os.path.join(ROOT, "tests", "fp_probe.cu")
    for name, extra in (("fmad", []), ("nofmad", ["--fmad=false"])):
        so = str(d / f"probe_{name}.so")
        subprocess.run(["nvcc", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler",
                        "-fPIC", *extra, "-o", so, src], check=True)
        lib = C.CDLL(so)
        lib.fp_probe_run.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        out[name] = lib
    return out


def _run(lib, op, x, k_in, k_out):
    x = np.ascontiguousarray(x, dtype=np.float32)
    n = x.size // k_in
    y = np.zeros(n * k_out, dtype=np.float32)
    assert lib.fp_probe_run(op, x.ctypes.data, n, k_in, k_out, y.ctypes.data) == 0
    return y.reshape(n, k_out)


def _operands(rng, n, k):
    mant = rng.uniform(-1, 1, size=(n, k))
    exp = rng.integers(-6, 7, size=(n, k))
    return (mant * 2.0 ** exp).astype(np.float32)


@pytest.mark.parametrize("op", [0, 1, 2, 3, 4])
def test_small_shapes(probes, oracle_mod, op):
    rng = np.random.default_rng(op)
    k_in, k_out = oracle_mod.FP_ARITY[op]
    x = _operands(rng, 200_000, k_in)
    fused = _run(probes["fmad"], op, x, k_in, k_out)
    plain = _run(probes["nofmad"], op, x, k_in, k_out)
    ref = oracle_mod.fp_eval(op, False, x)
    strict = oracle_mod.fp_eval(op, True, x)
    assert np.array_equal(fused.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(plain.view(np.uint32), strict.view(np.uint32))
    if op != 4:  # the shapes really differ between the two models
        assert (ref.view(np.uint32) != strict.view(np.uint32)).mean() > 0.05


def _voxel_cases(rng, n, aligned):
    u = np.float32(1.0 / 60.0)
    if aligned:  # vertices on a quarter-voxel lattice: many exactly borderline tests
        tri = rng.integers(16, 224, size=(n, 1, 3))[:, :, :] + rng.integers(-12, 13, size=(n, 3, 3))
        tri = (tri.astype(np.float32) * (u / np.float32(4.0))).astype(np.float32)
    else:
        base = rng.uniform(4, 56, size=(n, 1, 3))
        tri = base + rng.normal(scale=rng.choice([0.3, 2.0, 8.0], size=(n, 1, 1)), size=(n, 3, 3))
        tri = (np.clip(tri, 0.0, 59.9) * u).astype(np.float32)
    vox = np.floor(tri.astype(np.float64).mean(1) / u + rng.integers(-2, 3, size=(n, 3))).clip(0, 59)
    return np.concatenate([tri.reshape(n, 9), vox, np.full((n, 1), u), np.full((n, 1), 60.0)], 1).astype(np.float32)


@pytest.mark.parametrize("aligned,seed", [(False, 11), (True, 11), (True, 12), (True, 13)])
def test_voxel_predicate(probes, oracle_mod, aligned, seed):
    x = _voxel_cases(np.random.default_rng(seed), 300_000, aligned)
    fused = _run(probes["fmad"], 5, x, 14, 1)
    plain = _run(probes["nofmad"], 5, x, 14, 1)
    oracle_mod.set_fp_sites(PROBE_SITES)
    try:
        ref = oracle_mod.fp_eval(5, False, x)
    finally:
        oracle_mod.set_fp_sites(REFERENCE_SITES)
    strict = oracle_mod.fp_eval(5, True, x)
    assert 0.05 < ref.mean() < 0.95
    assert np.array_equal(fused, ref), int((fused != ref).sum())
    # the setup values (normal, plane and edge constants) too
    s_fused = _run(probes["fmad"], 6, x, 14, 14)
    s_plain = _run(probes["nofmad"], 6, x, 14, 14)
    assert np.array_equal(s_fused.view(np.uint32), oracle_mod.fp_eval(6, False, x).view(np.uint32))
    assert np.array_equal(s_plain.view(np.uint32), oracle_mod.fp_eval(6, True, x).view(np.uint32))
    assert np.array_equal(plain, strict), int((plain != strict).sum())
    if aligned:  # borderline cases where the two models disagree do occur
        assert (ref != strict).sum() > 0
