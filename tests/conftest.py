import gzip
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "gpu-svo_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def bunny_path(tmp_path_factory):
    """The reference's sample mesh (bunny.obj), unpacked from the fixture."""
    p = tmp_path_factory.mktemp("mesh") / "bunny.obj"
    with gzip.open(os.path.join(GOLDEN, "bunny.obj.gz"), "rb") as f:
        p.write_bytes(f.read())
    return str(p)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def svo_mod():
    import svo_b200

    svo_b200.lib()
    return svo_b200


@pytest.fixture(scope="session")
def gpu_ctx(svo_mod):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = svo_mod.Context(0)
    yield ctx
    ctx.close()


def random_mesh(seed: int, n_tris: int, kind: str = "blob"):
    """Small seeded meshes for parity tests."""
    rng = np.random.default_rng(seed)
    if kind == "blob":
        v = rng.normal(size=(max(3, n_tris), 3)).astype(np.float32)
        f = rng.integers(0, v.shape[0], size=(n_tris, 3)).astype(np.int32)
        return v, f
    if kind == "grid":  # axis-aligned triangles on grid-like coordinates
        v = (rng.integers(0, 9, size=(max(3, n_tris), 3)) / 8.0).astype(np.float32)
        f = rng.integers(0, v.shape[0], size=(n_tris, 3)).astype(np.int32)
        return v, f
    if kind == "sliver":
        c = rng.uniform(0, 1, size=(n_tris, 1, 3))
        d = rng.normal(size=(n_tris, 1, 3))
        t = np.concatenate([c - d * 0.3, c + d * 0.3, c + rng.normal(size=(n_tris, 1, 3)) * 0.002], 1)
        return t.reshape(-1, 3).astype(np.float32), np.arange(3 * n_tris, dtype=np.int32).reshape(-1, 3)
    raise ValueError(kind)
