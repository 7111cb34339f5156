"""Inputs on which the reference's own build (GPU-SVO's src/SVO.cu, run by
oracle/_ref/ref_dump) was recorded in tests/golden/ref_pins.json.

Each case is a mesh written as an OBJ file (both the reference and this
project parse that file, src/BaseModel.cpp:3-25) and a cubic resolution up to
1024, the largest the reference's 32-bit Morton codes handle.  `tree` marks
the cases whose tree .obj (src/SVO.cu:737-753) was hashed too, `cpu` the cases
small enough for the CPU oracle in the CPU test suite.
"""
from __future__ import annotations

import gzip
import os
import sys

TESTS = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(TESTS, "golden")
sys.path.insert(0, os.path.join(os.path.dirname(TESTS), "gpu-svo_b200"))

# name: (mesh, resolution, tree, cpu)
CASES = {
    "bunny_res16": ("bunny", 16, True, True),
    "bunny_res64": ("bunny", 64, True, True),  # the reference CLI's defaults
    "bunny_res128": ("bunny", 128, True, True),
    "bunny_res256": ("bunny", 256, True, True),
    "icosphere_l5_res128": ("icosphere_l5", 128, True, True),  # config 1
    "blob300_res64": ("blob300", 64, True, True),
    "grid200_res64": ("grid200", 64, True, True),
    "grid200_res128": ("grid200", 128, True, True),
    "sliver300_res128": ("sliver300", 128, True, True),
    "torus_slivers_every16_res512": ("torus_slivers_every16", 512, False, True),  # config 2, sampled
    "heightfield_every64_res1024": ("heightfield_every64", 1024, False, False),
    "torus_slivers_res512": ("torus_slivers", 512, False, False),  # config 2 in full
}


def mesh(kind: str):
    """(points float32[n,3], tris int32[m,3] or None for a soup)."""
    from svo_b200 import meshgen

    if kind == "bunny":
        return None, None
    if kind == "icosphere_l5":
        v, f, _ = meshgen.icosphere_l5()
        return v, f
    if kind.startswith("torus_slivers"):
        soup, _, _ = meshgen.torus_slivers()
        if kind.endswith("every16"):
            soup = soup.reshape(-1, 3, 3)[::16].reshape(-1, 3)
        return soup, None
    if kind == "heightfield_every64":
        v, f, _ = meshgen.heightfield()
        return v, f[::64]
    from conftest import random_mesh

    for prefix, seed in (("blob", 1), ("grid", 3), ("sliver", 2)):
        if kind.startswith(prefix):
            return random_mesh(seed, int(kind[len(prefix):]), prefix)
    raise ValueError(kind)


def write_case_obj(name: str, directory: str) -> str:
    """Writes the case's mesh as an OBJ file in `directory`; returns its path."""
    from svo_b200 import meshgen

    kind = CASES[name][0]
    path = os.path.join(directory, f"{kind}.obj")
    if os.path.exists(path):
        return path
    if kind == "bunny":
        with gzip.open(os.path.join(GOLDEN, "bunny.obj.gz"), "rb") as src, open(path, "wb") as dst:
            dst.write(src.read())
        return path
    v, f = mesh(kind)
    meshgen.write_obj(path, v, f)
    return path
