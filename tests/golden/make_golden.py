#!/usr/bin/env python3
"""Regenerates the golden fixtures in this directory from the reference tree.

Run in a container that has the GPU-SVO reference checked out (default
/root/reference, or $GPU_SVO_REF); the fixtures it writes are committed, so
nothing at test time reads the reference.

  morton_ref.npz  Morton encode/decode results of the reference's own
                  src/MortonLUT.h (host LUT paths, src/MortonLUT.h:482-529),
                  produced by oracle/_ref/pin_morton (oracle/ref/build_ref.sh).
  luts_ref.json   The reference's lookup tables, read as text:
                  neighbor_LUTparent / neighbor_LUTchild (src/MortonLUT.h:531-596),
                  d_vertSharedLUT (src/SVO.cu:567-584), d_edgeSharedLUT (src/SVO.cu:611-627).
  bunny.obj.gz    The reference's sample input mesh (bunny.obj, the CLI default
                  of main.cpp:8), gzip-compressed, used as a test input.
"""
import gzip
import json
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("GPU_SVO_REF", "/root/reference")


def c_array(text: str, name: str) -> list:
    m = re.search(re.escape(name) + r"\s*(\[[^=]*\])\s*=\s*\{", text)
    if not m:
        raise SystemExit(f"table {name} not found")
    i = m.end()
    depth = 1
    j = i
    while depth:
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
        j += 1
    body = re.sub(r"//[^\n]*", "", text[i : j - 1])
    return [int(v) for v in re.findall(r"-?\d+", body)]


def main() -> None:
    subprocess.run([os.path.join(REPO, "oracle", "ref", "build_ref.sh")], check=True,
                   env=dict(os.environ, GPU_SVO_REF=REF))
    out = subprocess.run([os.path.join(REPO, "oracle", "_ref", "pin_morton")], check=True,
                         capture_output=True, text=True).stdout
    enc, dec = [], []
    for line in out.splitlines():
        f = line.split()
        if f[0] == "E":
            enc.append([int(v) for v in f[1:]])
        elif f[0] == "D":
            dec.append([int(v) for v in f[1:]])
    np.savez_compressed(os.path.join(HERE, "morton_ref.npz"),
                        encode=np.array(enc, dtype=np.uint32), decode=np.array(dec, dtype=np.uint32))

    lut_h = open(os.path.join(REF, "src", "MortonLUT.h")).read()
    svo_cu = open(os.path.join(REF, "src", "SVO.cu"), encoding="utf-8-sig").read()
    luts = {
        "neighbor_LUTparent": c_array(lut_h, "neighbor_LUTparent"),
        "neighbor_LUTchild": c_array(lut_h, "neighbor_LUTchild"),
        "d_vertSharedLUT": c_array(svo_cu, "d_vertSharedLUT"),
        "d_edgeSharedLUT": c_array(svo_cu, "d_edgeSharedLUT"),
    }
    assert len(luts["neighbor_LUTparent"]) == 216 and len(luts["neighbor_LUTchild"]) == 216
    assert len(luts["d_vertSharedLUT"]) == 64 and len(luts["d_edgeSharedLUT"]) == 48
    with open(os.path.join(HERE, "luts_ref.json"), "w") as f:
        json.dump(luts, f)

    with open(os.path.join(REF, "bunny.obj"), "rb") as f:
        data = f.read()
    with gzip.GzipFile(os.path.join(HERE, "bunny.obj.gz"), "wb", compresslevel=9, mtime=0) as f:
        f.write(data)
    print("wrote morton_ref.npz, luts_ref.json, bunny.obj.gz", file=sys.stderr)


if __name__ == "__main__":
    main()
