"""The multi-process path of bench.py on CPU: two gloo ranks (replicas only --
the only collective is the max over ranks of the timer)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, os, sys, io, contextlib
sys.path.insert(0, os.environ["SVO_ROOT"])
import bench
rank, world = bench.dist_setup(2)
assert world == 2 and rank == int(os.environ["RANK"])
m = bench.dist_max(float(10 * (rank + 1)))
bench.dist_barrier()
sys.argv = ["bench.py", "--impl", "reference", "--workload", "icosphere_l5", "--steps", "1", "--warmup", "0",
            "--gpus", "2"]
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    bench.run_reference(bench.parse_args(), rank)
bench.dist_barrier()
bench.dist_done()
print(json.dumps({"rank": rank, "max": m, "ref_lines": [l for l in buf.getvalue().splitlines() if l.startswith("{")]}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(300)
def test_two_gloo_ranks(oracle_mod):
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                   LOCAL_RANK=str(rank), SVO_ROOT=ROOT, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=280)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    by_rank = {o["rank"]: o for o in outs}
    assert by_rank[0]["max"] == 20.0 and by_rank[1]["max"] == 20.0
    # the reference arm runs on rank 0 only and prints one line there
    assert len(by_rank[0]["ref_lines"]) == 1 and by_rank[1]["ref_lines"] == []
    line = json.loads(by_rank[0]["ref_lines"][0])
    assert line["impl"] == "reference" and line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
