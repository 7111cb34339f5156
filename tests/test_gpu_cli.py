"""The CLI (main.cpp:7-17 of the reference): same arguments, stdout and a
byte-identical <stem>_<depth>_tree.obj."""
import hashlib
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(svo_mod, cwd, *args):
    env = dict(os.environ)
    return subprocess.run([svo_mod.CLI_PATH, *args], cwd=cwd, capture_output=True, text=True, env=env, timeout=300)


def _sha(p):
    return hashlib.sha256(open(p, "rb").read()).hexdigest()


@pytest.mark.parametrize("res", [32, 64, 128])
def test_cli_bunny(tmp_path, bunny_path, svo_mod, oracle_mod, gpu_ctx, res):
    shutil.copy(bunny_path, tmp_path / "bunny.obj")
    p = _run(svo_mod, tmp_path, "bunny.obj", str(res))
    assert p.returncode == 0, p.stderr
    o = oracle_mod.build_svo(*oracle_mod.load_obj(bunny_path), res)
    name = f"bunny_{o.depth}_tree.obj"
    assert p.stdout == (f"Sparse Voxel Octree depth: {o.depth}\n"
                        f"[I/O] Writing octree data in obj format to file {name} \n")
    o.write_tree(str(tmp_path / "oracle.obj"))
    assert _sha(tmp_path / name) == _sha(tmp_path / "oracle.obj")


def test_cli_defaults(tmp_path, bunny_path, svo_mod, gpu_ctx):
    shutil.copy(bunny_path, tmp_path / "bunny.obj")
    p = _run(svo_mod, tmp_path)
    assert p.returncode == 0, p.stderr
    assert (tmp_path / "bunny_7_tree.obj").exists()  # res 64 -> depth 7


def test_cli_icosphere(tmp_path, svo_mod, oracle_mod, gpu_ctx):
    from svo_b200 import meshgen

    v, f, res = meshgen.icosphere_l5()
    path = tmp_path / "ico.obj"
    meshgen.write_obj(str(path), v, f)
    p = _run(svo_mod, tmp_path, "ico.obj", str(res))
    assert p.returncode == 0, p.stderr
    o = oracle_mod.build_svo(*oracle_mod.load_obj(str(path)), res)
    o.write_tree(str(tmp_path / "oracle.obj"))
    assert _sha(tmp_path / f"ico_{o.depth}_tree.obj") == _sha(tmp_path / "oracle.obj")


def test_cli_missing_file(tmp_path, svo_mod):
    p = _run(svo_mod, tmp_path, "nope.obj", "64")
    assert p.returncode == 1
    assert "ERROR: loading obj:(nope.obj) file is not good" in p.stderr
