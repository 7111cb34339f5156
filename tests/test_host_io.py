"""Host-side pieces of the product against the oracle: bounding cube and the
byte-exact tree writer (src/IO.h:8-90, src/SVO.cu:737-753)."""
import hashlib

import numpy as np
import pytest

from conftest import random_mesh


@pytest.mark.parametrize("seed", range(6))
def test_bbox_cube_matches_oracle(oracle_mod, svo_mod, seed):
    rng = np.random.default_rng(seed)
    pts = (rng.normal(size=(1000, 3)) * rng.uniform(0.01, 100, size=3) + rng.normal(size=3) * 50).astype(np.float32)
    assert oracle_mod.bbox_cube(pts).tobytes() == svo_mod.bbox_cube(pts).tobytes()


def test_bbox_cube_rejects_nonfinite(svo_mod):
    pts = np.array([[0, 0, 0], [1, np.inf, 0]], dtype=np.float32)
    with pytest.raises(svo_mod.SvoError):
        svo_mod.bbox_cube(pts)


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


@pytest.mark.parametrize("res", [8, 32])
def test_writer_bytes_bunny(tmp_path, bunny_path, oracle_mod, svo_mod, res):
    pts, tri = oracle_mod.load_obj(bunny_path)
    r = oracle_mod.build_svo(pts, tri, res)
    a, b = str(tmp_path / "a.obj"), str(tmp_path / "b.obj")
    r.write_tree(a)
    svo_mod.write_tree_nodes(r.nodes.view(svo_mod.NODE_DTYPE), b)
    assert _sha(a) == _sha(b)


def test_writer_bytes_special_values(tmp_path, oracle_mod, svo_mod):
    """Odd floats through both writers: signed zeros, subnormals, huge, ties."""
    v, f = random_mesh(3, 50)
    r = oracle_mod.build_svo(v, f, 4)
    nodes = r.nodes.copy()
    rng = np.random.default_rng(7)
    specials = np.array([0.0, -0.0, 1e-45, -3e-39, 3.4e38, -1.17549435e-38, 0.0009765625, 123456.5,
                         999999.5, 1e6, 9.999995e5, 0.1, 2.5e-5, 1.0000005, 65504.0], dtype=np.float32)
    vals = np.concatenate([specials, rng.normal(size=4000).astype(np.float32) * 10.0 ** rng.integers(-12, 12, 4000)])
    reps = int(np.ceil(vals.size / (nodes.shape[0] * 4)))
    vals = np.tile(vals, reps)[: nodes.shape[0] * 4].astype(np.float32)
    nodes["origin"] = vals[: nodes.shape[0] * 3].reshape(-1, 3)
    nodes["width"] = vals[nodes.shape[0] * 3:]
    a, b = str(tmp_path / "a.obj"), str(tmp_path / "b.obj")
    # write through the oracle (std::ofstream) from the same node array
    import ctypes as C
    oracle_mod.lib().oracle_write_tree  # loaded
    h = r._handle
    base = oracle_mod.lib().oracle_result_nodes(h)
    C.memmove(base, nodes.ctypes.data, nodes.nbytes)
    r.write_tree(a)
    svo_mod.write_tree_nodes(nodes.view(svo_mod.NODE_DTYPE), b)
    assert _sha(a) == _sha(b)
