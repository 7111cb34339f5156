"""The public headers as a user compiles them: include/svo_b200.h as strict
C99 (every declared entry point referenced and linked against the library)
and the C++ facade (include/svo/SVO.h) in the usage the integration notes
show.  Compile and link only: running needs a GPU."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT
from test_capi_exports import _declared

INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "gpu-svo_b200", "lib")


def _build(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_header_strict_c99(tmp_path, svo_mod):
    names = sorted(_declared())
    src = ["#include <svo_b200.h>", "#include <stdio.h>", "typedef void (*fn)(void);", "static const fn all[] = {"]
    src += [f"    (fn){n}," for n in names]
    src += ["};", "int main(void) {", "    svo_tuning t = {64, 256, 0, 32, 0};",
            "    svo_mesh_desc d;", "    (void)d;", "    printf(\"%u %d\\n\", t.serial_max, (int)(sizeof all / sizeof all[0]));",
            "    return 0;", "}"]
    c = tmp_path / "all.c"
    c.write_text("\n".join(src) + "\n")
    _build(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", INC, str(c), "-L", LIBDIR,
            "-lsvo_b200", "-o", str(tmp_path / "all")])


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_facade(tmp_path, svo_mod):
    c = tmp_path / "app.cpp"
    c.write_text("""
#include <svo/SVO.h>
#include <cstdio>
int main(int argc, char **argv) {
    SparseVoxelOctree svo(argc > 1 ? argv[1] : "bunny.obj", 128, 128, 128);
    svo.setBuildFlags(SVO_FLAG_FULL_NEIGHBORS);
    svo.create();
    svo.writeTree("bunny");
    const std::vector<SVONode> &nodes = svo.nodes();
    std::printf("%zu %u\\n", nodes.size(), nodes.empty() ? 0u : nodes[0].mortonCode);
    return 0;
}
""")
    _build(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", INC, str(c), "-L", LIBDIR, "-lsvo_b200",
            "-o", str(tmp_path / "app")])
