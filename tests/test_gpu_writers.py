"""The OBJ writers on GPU builds against the oracle's std::ofstream writers:
writeTree (src/SVO.cu:737-753) and writeVoxel (src/SVO.cu:755-777, one cube per
surface voxel at modelBBox.min + width * (x, y, z)), byte for byte."""
import hashlib

import pytest

from conftest import random_mesh

pytestmark = pytest.mark.gpu


def _sha(p):
    with open(p, "rb") as fh:
        return hashlib.sha256(fh.read()).hexdigest()


@pytest.mark.parametrize("case", ["bunny64", "bunny128", "icosphere128", "blob64", "grid32", "sliver256"])
def test_writers_match_oracle(gpu_ctx, svo_mod, oracle_mod, bunny_path, tmp_path, case):
    from svo_b200 import meshgen

    if case.startswith("bunny"):
        v, f = oracle_mod.load_obj(bunny_path)
    elif case.startswith("icosphere"):
        v, f, _ = meshgen.icosphere_l5()
    else:
        kind = case.rstrip("0123456789")
        v, f = random_mesh(21, 200, kind)
    res = int(case[len(case.rstrip("0123456789")):])
    g = gpu_ctx.build(v, f, res)
    o = oracle_mod.build_svo(v, f, res)
    for name, a, b in (("voxels", g.write_voxels, o.write_voxels), ("tree", g.write_tree, o.write_tree)):
        a(str(tmp_path / f"g_{name}.obj"))
        b(str(tmp_path / f"o_{name}.obj"))
        assert _sha(tmp_path / f"g_{name}.obj") == _sha(tmp_path / f"o_{name}.obj"), name
