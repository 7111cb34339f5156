#!/usr/bin/env python3
"""Records the reference's own build outputs as golden fixtures.

Runs oracle/_ref/ref_dump -- GPU-SVO's unmodified src/SVO.cu and
src/BaseModel.cpp compiled by oracle/ref/build_ref.sh -- on every case of
tests/refcases.py (needs a CUDA GPU) and writes
  <out>/ref_pins.json   per case: depth, counts, depthNumNodes, bounding cube,
                        SHA-256 of the node / vertex / edge / voxel arrays and
                        of the tree .obj, and the reference's own timings
  <out>/ref_voxels.npz  the voxel code lists of the cases of at most 2^17 voxels
and checks the reference's CLI (oracle/_ref/ref_main, main.cpp) on the bunny at
its default resolution against the harness's tree file; its NDEBUG build
(oracle/_ref/ref_main_ndebug) records the surface-voxel file writeVoxel writes.

Every input first goes through the CPU oracle: inputs it rejects as undefined
in the reference (a single surface voxel, or a single top-level node in a
non-zero octant, where the reference writes past its node array) are never
handed to the reference.

  python tests/golden/make_ref_fixtures.py --out gpurun_out/refpins [--cases a,b]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gpu-svo_b200"))
REF_DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "ref_main")
REF_MAIN_NDEBUG = os.path.join(ROOT, "oracle", "_ref", "ref_main_ndebug")
SEGMENTS = (("nodes", 168), ("vertices", 16), ("edges", 28), ("voxels", 4))


def run_ref(obj: str, res: int, work: str, stem: str, tree: bool):
    """Runs ref_dump; returns (meta, {segment: sha256}, voxels u32 array)."""
    cmd = [REF_DUMP, obj, str(res), work, stem] + (["tree"] if tree else [])
    p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE)
    head = p.stdout.read(40)
    if len(head) != 40 or head[:8] != b"SVOREF1\0":
        err = p.stderr.read().decode(errors="replace")
        p.wait()
        raise RuntimeError(f"ref_dump failed ({p.returncode}): {err[-2000:]}")
    counts = np.frombuffer(head[8:], dtype=np.uint64)
    digests, voxels = {}, None
    for (name, size), n in zip(SEGMENTS, counts):
        h, left = hashlib.sha256(), int(n) * size
        keep = [] if name == "voxels" else None
        while left:
            b = p.stdout.read(min(left, 64 << 20))
            if not b:
                raise RuntimeError(f"ref_dump stream ended early in {name}")
            h.update(b)
            if keep is not None:
                keep.append(b)
            left -= len(b)
        digests[name] = h.hexdigest()
        if keep is not None:
            voxels = np.frombuffer(b"".join(keep), dtype=np.uint32)
    err = p.stderr.read().decode(errors="replace")
    if p.wait() != 0:
        raise RuntimeError(f"ref_dump exited {p.returncode}: {err[-2000:]}")
    meta = json.load(open(os.path.join(work, "meta.json")))
    meta["stderr"] = [l for l in err.splitlines() if l.strip()][-4:]
    return meta, digests, voxels


def main():
    import oracle
    import refcases

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--cases", default="")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    names = [c for c in args.cases.split(",") if c] or list(refcases.CASES)
    work = tempfile.mkdtemp(prefix="svoref_")
    pins, vox = {}, {}
    try:
        for name in names:
            kind, res, tree, _ = refcases.CASES[name]
            obj = refcases.write_case_obj(name, work)
            pts, tris = oracle.load_obj(obj)
            try:  # the oracle refuses the inputs the reference has no defined build for
                oracle.build_svo(pts, tris, res, flags=oracle.FLAG_NO_VERT_EDGE).close()
            except oracle.OracleError as e:
                pins[name] = {"skipped": str(e)}
                print(f"{name}: skipped ({e})", flush=True)
                continue
            case_dir = os.path.join(work, name)
            os.makedirs(case_dir, exist_ok=True)
            t = time.time()
            meta, dig, voxels = run_ref(obj, res, case_dir, kind, tree)
            entry = {"mesh": kind, "res": res, "triangles": int(tris.shape[0]), "sha256": dig, **meta,
                     "wall_s": time.time() - t}
            if tree:
                path = os.path.join(case_dir, f"{kind}_{meta['depth']}_tree.obj")
                with open(path, "rb") as fh:
                    entry["sha256"]["tree_obj"] = hashlib.sha256(fh.read()).hexdigest()
                entry["tree_obj_bytes"] = os.path.getsize(path)
            if voxels.size <= (1 << 17):
                vox[name] = voxels
            pins[name] = entry
            print(f"{name}: depth {meta['depth']}, {meta['num_nodes']} nodes, {meta['num_voxels']} voxels, "
                  f"create {meta['create_ms']:.1f} ms", flush=True)
            shutil.rmtree(case_dir)
        # the reference's CLI on its defaults (main.cpp:7-17): same file as the harness wrote
        if "bunny_res64" in pins and "sha256" in pins["bunny_res64"]:
            cli = os.path.join(work, "cli")
            os.makedirs(cli, exist_ok=True)
            obj = refcases.write_case_obj("bunny_res64", work)
            r = subprocess.run([REF_MAIN, obj, "64"], cwd=cli, capture_output=True, text=True, check=True)
            fname = f"bunny_{pins['bunny_res64']['depth']}_tree.obj"
            out = os.path.join(cli, fname)
            with open(out, "rb") as fh:
                sha = hashlib.sha256(fh.read()).hexdigest()
            pins["bunny_res64"]["cli"] = {"argv": ["main", "bunny.obj", "64"], "stdout": r.stdout,
                                          "file": fname, "sha256": sha}
            if sha != pins["bunny_res64"]["sha256"]["tree_obj"]:
                raise RuntimeError("the reference CLI's tree file differs from the harness's")
            # the NDEBUG build: create() also writes the surface voxels (writeVoxel, src/SVO.cu:411-419)
            nd = os.path.join(work, "ndebug")
            os.makedirs(nd, exist_ok=True)
            r = subprocess.run([REF_MAIN_NDEBUG, obj, "64"], cwd=nd, capture_output=True, text=True, check=True)
            with open(os.path.join(nd, "bunny_1_voxel.obj"), "rb") as fh:
                vsha = hashlib.sha256(fh.read()).hexdigest()
            with open(os.path.join(nd, fname), "rb") as fh:
                if hashlib.sha256(fh.read()).hexdigest() != sha:
                    raise RuntimeError("the NDEBUG build's tree file differs")
            pins["bunny_res64"]["voxel_obj"] = {"file": "bunny_1_voxel.obj", "sha256": vsha, "stdout": r.stdout}
    finally:
        shutil.rmtree(work, ignore_errors=True)
        with open(os.path.join(args.out, "ref_pins.json"), "w") as fh:
            json.dump(pins, fh, indent=1, sort_keys=True)
        np.savez_compressed(os.path.join(args.out, "ref_voxels.npz"), **vox)


if __name__ == "__main__":
    main()
