"""The oracle against the reference's own build.

tests/golden/ref_pins.json holds what GPU-SVO itself computed (its unmodified
src/SVO.cu and src/BaseModel.cpp, built by oracle/ref/build_ref.sh and run on a
B200 by tests/golden/make_ref_fixtures.py) for the inputs of tests/refcases.py:
depth, level sizes, bounding cube, SHA-256 of the node / vertex / edge arrays,
of the surface-voxel codes and of the tree .obj.  The oracle must reproduce
every one of them with the reference's default semantics.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import refcases

PINS = os.path.join(refcases.GOLDEN, "ref_pins.json")
VOXELS = os.path.join(refcases.GOLDEN, "ref_voxels.npz")


def load_pins():
    if not os.path.exists(PINS):
        return {}
    return {k: v for k, v in json.load(open(PINS)).items() if "sha256" in v}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8)).hexdigest()


def file_sha(path: str) -> str:
    with open(path, "rb") as fh:
        return hashlib.sha256(fh.read()).hexdigest()


def check_result(pin: dict, depth, level_counts, bbox, nodes, vertices, edges, voxels_u32, name: str):
    """Compares one build's outputs with the reference's recorded ones."""
    assert depth == pin["depth"], name
    # depthNumNodes holds every level but the single-node top (src/SVO.cu:436-437)
    assert list(level_counts[:-1]) == pin["depth_num_nodes"] and level_counts[-1] == 1, name
    assert np.array_equal(np.asarray(bbox, np.float32), np.asarray(pin["bbox"], np.float32)), name
    assert (nodes.shape[0], vertices.shape[0], edges.shape[0], voxels_u32.shape[0]) == \
        (pin["num_nodes"], pin["num_vertices"], pin["num_edges"], pin["num_voxels"]), name
    if os.path.exists(VOXELS):
        ref_vox = np.load(VOXELS)
        if name in ref_vox.files:
            assert np.array_equal(voxels_u32, ref_vox[name]), name
    assert sha(voxels_u32) == pin["sha256"]["voxels"], name
    assert sha(nodes) == pin["sha256"]["nodes"], name
    assert sha(vertices) == pin["sha256"]["vertices"], name
    assert sha(edges) == pin["sha256"]["edges"], name


PIN_CASES = [n for n in refcases.CASES if refcases.CASES[n][3]]


@pytest.mark.parametrize("name", PIN_CASES)
def test_oracle_matches_reference(oracle_mod, tmp_path_factory, name):
    pins = load_pins()
    if name not in pins:
        pytest.skip("no recording of the reference for this case")
    pin = pins[name]
    d = tmp_path_factory.mktemp("ref")
    pts, tris = oracle_mod.load_obj(refcases.write_case_obj(name, str(d)))
    assert tris.shape[0] == pin["triangles"]
    o = oracle_mod.build_svo(pts, tris, pin["res"])
    check_result(pin, o.depth, o.level_counts, o.bbox, o.nodes, o.vertices, o.edges,
                 o.keys.astype(np.uint32), name)
    if "tree_obj" in pin["sha256"]:
        path = str(d / f"{name}_tree.obj")
        o.write_tree(path)
        assert file_sha(path) == pin["sha256"]["tree_obj"], name
    o.close()


def test_pins_cover_the_cases():
    """Every case was recorded (none skipped as undefined in the reference),
    and the reference CLI wrote the same tree file as the harness."""
    if not os.path.exists(PINS):
        pytest.skip("no recording of the reference")
    raw = json.load(open(PINS))
    assert set(raw) == set(refcases.CASES)
    assert all("sha256" in v for v in raw.values())
    cli = raw["bunny_res64"]["cli"]
    assert cli["sha256"] == raw["bunny_res64"]["sha256"]["tree_obj"]
    assert cli["file"] == f"bunny_{raw['bunny_res64']['depth']}_tree.obj"


def test_oracle_voxel_file_matches_reference(oracle_mod, tmp_path):
    """writeVoxel (src/SVO.cu:755-777): the reference built with NDEBUG writes
    bunny_1_voxel.obj from create(); the oracle writes the same bytes."""
    pins = load_pins()
    if "voxel_obj" not in pins.get("bunny_res64", {}):
        pytest.skip("no recording of the reference's voxel file")
    o = oracle_mod.build_svo(*oracle_mod.load_obj(refcases.write_case_obj("bunny_res64", str(tmp_path))), 64)
    o.write_voxels(str(tmp_path / "voxels.obj"))
    assert file_sha(str(tmp_path / "voxels.obj")) == pins["bunny_res64"]["voxel_obj"]["sha256"]
