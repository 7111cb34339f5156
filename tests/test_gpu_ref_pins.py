"""The product against the reference's own build, on the GPU.

Every input of tests/refcases.py -- config 1, config 2 in full, a heightfield
sample at resolution 1024 (the reference's largest), the reference's bunny at
four resolutions, random, lattice-aligned and sliver meshes -- is built through
the C ABI with default flags; its node / vertex / edge arrays, surface-voxel
codes and tree .obj must hash to what GPU-SVO itself produced
(tests/golden/ref_pins.json), and the CLI must print what the reference's CLI
printed and write the same file.
"""
import os
import subprocess

import numpy as np
import pytest

import refcases
from test_ref_pins import check_result, file_sha, load_pins

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(refcases.CASES))
def test_product_matches_reference(gpu_ctx, svo_mod, tmp_path_factory, name):
    pins = load_pins()
    if name not in pins:
        pytest.skip("no recording of the reference for this case")
    pin = pins[name]
    d = tmp_path_factory.mktemp("refgpu")
    pts, tris = svo_mod.load_obj(refcases.write_case_obj(name, str(d)))
    g = gpu_ctx.build(pts, tris, pin["res"])
    keys = g.keys()
    assert keys.size == 0 or int(keys.max()) < (1 << 31)
    check_result(pin, g.depth, g.level_counts, g.bbox, g.nodes(), g.vertices(), g.edges(),
                 keys.astype(np.uint32), name)
    if "tree_obj" in pin["sha256"]:
        path = str(d / f"{name}_tree.obj")
        g.write_tree(path)
        assert file_sha(path) == pin["sha256"]["tree_obj"], name
    g.close()


def test_cli_matches_reference_cli(svo_mod, tmp_path):
    """svo_main <mesh.obj> <res> against the reference's main.cpp on its
    default mesh and resolution: same stdout, same file name, same bytes."""
    pins = load_pins()
    if "bunny_res64" not in pins or "cli" not in pins["bunny_res64"]:
        pytest.skip("no recording of the reference CLI")
    cli = pins["bunny_res64"]["cli"]
    obj = refcases.write_case_obj("bunny_res64", str(tmp_path))
    r = subprocess.run([svo_mod.CLI_PATH, obj, "64"], cwd=tmp_path, capture_output=True, text=True, check=True)
    assert r.stdout == cli["stdout"]
    assert file_sha(str(tmp_path / cli["file"])) == cli["sha256"]


def test_voxel_file_matches_reference(gpu_ctx, svo_mod, tmp_path):
    """svo_write_voxels against the file the reference's create() writes in
    its NDEBUG build (writeVoxel, src/SVO.cu:411-419, 755-777)."""
    pins = load_pins()
    if "voxel_obj" not in pins.get("bunny_res64", {}):
        pytest.skip("no recording of the reference's voxel file")
    pts, tris = svo_mod.load_obj(refcases.write_case_obj("bunny_res64", str(tmp_path)))
    g = gpu_ctx.build(pts, tris, 64)
    g.write_voxels(str(tmp_path / "voxels.obj"))
    assert file_sha(str(tmp_path / "voxels.obj")) == pins["bunny_res64"]["voxel_obj"]["sha256"]
