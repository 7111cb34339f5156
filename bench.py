#!/usr/bin/env python3
"""Benchmark of the octree build path: one step = one full SVO build
(voxelize -> octree levels -> node records + vertex/edge arrays, bit-exact
with the reference's semantics) of a seeded synthetic mesh.

Default workload: the 4,999,122-triangle heightfield at resolution 2048
(depth 11) with full neighbour tables and vertex/edge/face dedup
(svo_b200.meshgen.heightfield).  `value` is whole-job triangles/s with the
mesh already resident in HBM; `e2e` is the same metric through the C ABI with
pinned host buffers (host->device copy of the mesh and device->host copy of
the whole octree -- nodes, vertices, edges, keys, dedup lists -- inside the
timed region).  `--workload torus_slivers` is the 1M-triangle soup at
resolution 512.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Multi-GPU (torchrun): replicas only -- every rank builds the same workload
independently (one build does not shard), no collective on the data path;
value = triangles of all ranks / max over ranks of the device time.

--impl reference times the CPU restatement of the reference's build
(oracle/, all host threads) on a bounded sample of the same workload.

On one GPU the default line also carries `batch256` and `serve`: short runs of
the 256-mesh batch (against one plain build per mesh) and of the served
Poisson stream (p50/p99 latency against the plain per-request path), measured
after the headline's timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-svo_b200"))

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 256 << 20
# Algorithmic bytes of one node in the emission kernel: node record 168 B,
# 8 vertices x 16 B, 12 edges x 28 B written; one 8-byte group code read per
# 8 sibling nodes.
EMIT_BYTES_PER_NODE = 168 + 8 * 16 + 12 * 28 + 1
EMIT_BYTES_PER_NODE_NODES_ONLY = 168 + 1  # SVO_FLAG_NO_VERT_EDGE: the node records alone
# Every stride-th triangle of a single-mesh workload is the bounded sample the
# CPU legs (the oracle) build, with the workload's own flags.
CPU_STRIDE = {"torus_slivers": 16, "heightfield": 128, "icosphere_l5": 1}
TUNING_KEYS = ("serial_max", "warp_max", "split", "inplace_max", "serial_packed")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["heightfield", "torus_slivers", "icosphere_l5", "batch256", "serve"],
                    default="heightfield")
    ap.add_argument("--rates", default="200,500,1000,2000,5000", help="serve: Poisson arrival rates (req/s)")
    ap.add_argument("--window", type=float, default=1.0, help="serve: seconds of arrivals per rate")
    ap.add_argument("--flags", type=int, default=-1, help="override the workload's build flags (SVO_FLAG_*)")
    ap.add_argument("--wave-gb", type=float, default=48.0, help="batch256: device bytes of results per emit wave")
    ap.add_argument("--res", type=int, default=0, help="override the workload's resolution")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="heightfield: skip the short batched and served runs reported beside the headline")
    ap.add_argument("--tune", type=int, default=1, help="single-mesh workloads: autotune the voxelizer split first")
    ap.add_argument("--tuning", default="", help="single-mesh workloads: use this split instead "
                    "(serial_max,warp_max,split,inplace_max,serial_packed)")
    return ap.parse_args()


def workload(name: str):
    """(points, tris, res, name, build flags) of a single-mesh workload."""
    import svo_b200 as S
    from svo_b200 import meshgen

    if name == "torus_slivers":
        pts, tris, res = meshgen.torus_slivers()
        return pts, tris, res, "torus_slivers_1M_res512", 0
    if name == "heightfield":
        # 5M triangles at resolution 2048 with full neighbour tables and vertex/edge/face dedup
        pts, tris, res = meshgen.heightfield()
        return pts, tris, res, "heightfield_5M_res2048_full_dedup", S.FLAG_FULL_NEIGHBORS | S.FLAG_DEDUP
    pts, tris, res = meshgen.icosphere_l5()
    return pts, tris, res, "icosphere_l5_res128", 0


def n_triangles(pts, tris) -> int:
    return pts.shape[0] // 3 if tris is None else tris.shape[0]


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------
def dist_setup(n_gpus: int):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and not dist.is_initialized():
        import datetime

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    rank = dist.get_rank() if dist.is_initialized() else 0
    return rank, world


def dist_max(x: float) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_initialized():
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier() -> None:
    import torch.distributed as dist

    if dist.is_initialized():
        dist.barrier()


def dist_done() -> None:
    import torch.distributed as dist

    if dist.is_initialized():
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and clock-event reasons sampled while the timed steps run:
    NVML every 5 ms in a thread (read-only queries), else `nvidia-smi -lms 100`.
    Entering waits for the first sample, so even a short timed region is
    covered."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list[str] = []
        self.times: list[float] = []
        self.t_start = 0.0
        self._stop = threading.Event()
        self._t = None

    def _nvml_handle(self):
        import pynvml as N

        N.nvmlInit()
        try:
            import torch

            p = torch.cuda.get_device_properties(self.dev)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return N, N.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return N, N.nvmlDeviceGetHandleByIndex(self.dev)

    def _poll_nvml(self, N, h):
        R = {"hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
             "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
             "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
             "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap}
        smax = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        while True:
            sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
            bits = N.nvmlDeviceGetCurrentClocksEventReasons(h)
            act = ["Active" if bits & R[k] else "Not Active" for k in
                   ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")]
            self.lines.append(", ".join([str(self.dev), str(sm), str(smax), "", hex(bits)] + act))
            self.times.append(time.time())
            if self._stop.wait(0.005):
                break

    def __enter__(self):
        try:
            N, h = self._nvml_handle()
            self._t = threading.Thread(target=self._poll_nvml, args=(N, h), daemon=True)
            self._t.start()
        except Exception:
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                     "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self._t = threading.Thread(target=self._read, daemon=True)
                self._t.start()
            except (FileNotFoundError, OSError):
                self.proc = None
        t0 = time.time()
        while self._t is not None and not self.lines and time.time() - t0 < 5.0 and self._t.is_alive():
            time.sleep(0.001)
        self.t_start = time.time()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        elif self._t is not None:
            self._t.join(timeout=5)

    def summary(self) -> dict:
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines
        if self.times:  # NVML samples: those taken while the timed steps ran, if any
            inside = [l for l, t in zip(self.lines, self.times) if t >= self.t_start]
            lines = inside or self.lines[-1:]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU legs (the oracle: CPU restatement of the reference's build)
# ---------------------------------------------------------------------------
def cpu_sample(pts, tris, stride: int):
    """Every stride-th triangle of the workload (a bounded sample)."""
    if tris is None:
        soup = pts.reshape(-1, 3, 3)[::stride].reshape(-1, 3)
        return soup, np.arange(soup.shape[0], dtype=np.int32).reshape(-1, 3)
    return pts, tris[::stride]


def time_cpu_build(pts, tris, res, threads: int, flags: int = 0) -> float:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    t = time.perf_counter()
    r = oracle.build_svo(pts, tris, res, flags=flags & (oracle.FLAG_FULL_NEIGHBORS | oracle.FLAG_DEDUP),
                         threads=threads)
    dt = time.perf_counter() - t
    r.close()
    return dt


def cpu_sample_text(stride: int, wname: str, nt: int, res: int, flags: int) -> str:
    import svo_b200 as S

    extra = [n for b, n in ((S.FLAG_FULL_NEIGHBORS, "full neighbour tables"), (S.FLAG_DEDUP, "dedup lists"))
             if flags & b]
    return (f"every {stride}th triangle of {wname} ({nt} triangles), res {res}, full build (voxels, levels, "
            f"nodes, vertex/edge arrays{''.join(', ' + e for e in extra)})")


def batch_cpu_sample(meshes, stride: int = 32):
    """Every stride-th mesh of the batch, resolutions capped at 256 (a bounded sample)."""
    return [(p, t, min(r, 256)) for p, t, r in meshes[::stride]]


def workload_config(wname: str, triangles: int, res: int, flags: int, gpus: int) -> dict:
    """The workload as both arms name it: the same dict in our line and in the
    reference arm's (which times a sample of it, stated in its cpu_baseline)."""
    return {"workload": wname, "triangles": triangles, "resolution": res, "flags": flags,
            "parallelism": f"replicas{gpus}",
            "l2_flush": "GPU arm: 256 MiB device write before every step, outside the timed span"}


def run_reference(args, rank: int):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.workload in ("batch256", "serve"):
        from svo_b200 import meshgen

        sample_meshes = batch_cpu_sample(meshgen.batch(256, seed=3))
        nt = sum(t.shape[0] for _, t, _ in sample_meshes)
        wname, res = "batch256_seed3", [r for _, _, r in sample_meshes]

        def one():
            return sum(time_cpu_build(p, t, r, threads) for p, t, r in sample_meshes)

        sample = (f"every 32nd mesh of the 256-mesh batch ({len(sample_meshes)} meshes, {nt} triangles), "
                  f"resolution capped at 256, full builds")
        config = {"workload": wname, "sample_triangles": nt, "resolution": res}
    else:
        pts, tris, res, wname, wflags = workload(args.workload)
        flags = wflags if args.flags < 0 else args.flags
        if args.res:
            res, wname = args.res, f"{wname.rsplit('_res', 1)[0]}_res{args.res}"
        stride = CPU_STRIDE[args.workload]
        spts, stris = cpu_sample(pts, tris, stride)
        nt = stris.shape[0]
        config = workload_config(wname, n_triangles(pts, tris), res, flags, args.gpus)

        def one():
            return time_cpu_build(spts, stris, res, threads, flags)

        sample = cpu_sample_text(stride, wname, nt, res, flags)
    for _ in range(args.warmup):
        one()
    times = [one() for _ in range(args.steps)]
    total = sum(times)
    value = nt * len(times) / total
    line = {
        "impl": "reference", "metric": "tris/s", "value": value, "unit": "tris/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config, "sample_triangles": nt,
        "cpu_baseline": {"value": value, "unit": "tris/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "tris/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU build path (its build is CUDA); this times the CPU restatement "
                "of its algorithm (oracle/) on the host cores",
        "reference_cuda": reference_cuda_build(),
    }
    print(json.dumps(line), flush=True)


# The input on which the reference's own CUDA build is timed beside ours: every
# 16th triangle of the torus + sliver soup at resolution 512 (within the
# reference's 32-bit Morton codes), as an OBJ file both programs read.
REF_CUDA_INPUT = ("torus_slivers_every16_res512", 16, 512)


def write_ref_cuda_input(directory: str) -> str:
    from svo_b200 import meshgen

    soup, _, _ = meshgen.torus_slivers()
    path = os.path.join(directory, "torus_slivers_every16.obj")
    meshgen.write_obj(path, soup.reshape(-1, 3, 3)[:: REF_CUDA_INPUT[1]].reshape(-1, 3), None)
    return path


def reference_cuda_build():
    """GPU-SVO's own CUDA build (its unmodified src/SVO.cu, compiled for
    sm_100a into oracle/_ref/ref_dump where the reference tree was present) on
    REF_CUDA_INPUT, on this GPU: the wall time of SparseVoxelOctree::create()
    -- host triangle gather, device build, copies of the octree back to the
    host -- best of 2.  None when the binary is absent."""
    import tempfile

    exe = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
    if not os.path.exists(exe):
        return None
    with tempfile.TemporaryDirectory() as td:
        obj = write_ref_cuda_input(td)
        runs = []
        for _ in range(2):
            r = subprocess.run([exe, obj, str(REF_CUDA_INPUT[2]), td, "ref"], stdout=subprocess.DEVNULL,
                               stderr=subprocess.PIPE, text=True)
            if r.returncode != 0:
                return {"error": r.stderr[-300:]}
            runs.append(json.load(open(os.path.join(td, "meta.json"))))
    best = min(runs, key=lambda m: m["create_ms"])
    return {"workload": REF_CUDA_INPUT[0], "create_ms": best["create_ms"], "load_ms": best["load_ms"],
            "voxelize_ms": best["voxelize_ms"], "nodes": best["num_nodes"],
            "what": "SparseVoxelOctree::create() wall time of the reference's own build on this GPU"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank: int, world: int):
    import torch

    import svo_b200 as S

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    sid = stream.cuda_stream
    pts, tris, res, wname, wflags = workload(args.workload)
    bflags = wflags if args.flags < 0 else args.flags
    if args.res:
        res, wname = args.res, f"{wname.rsplit('_res', 1)[0]}_res{args.res}"
    nt = n_triangles(pts, tris)
    ctx = S.Context(dev)
    d_pts = torch.from_numpy(pts).cuda()
    d_tris = torch.from_numpy(tris).cuda() if tris is not None else None
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")
    # voxelizer work split for this mesh (svo_ctx_autotune, before any timing;
    # results do not depend on it)
    if args.tuning:
        ctx.tuning = tuple(int(x) for x in args.tuning.split(","))
        tuning = ctx.tuning
    else:
        tuning = ctx.autotune([(d_pts, d_tris, res)], bflags, sid) if args.tune else ctx.tuning

    def step(flags=0):
        flush.fill_(1)  # L2 flush before each step, outside the timed span
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = ctx.build(d_pts, d_tris, res, flags | bflags, sid)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        return ms, r

    for _ in range(args.warmup):
        _, r = step()
        r.close()
    dist_barrier()
    torch.cuda.synchronize()
    launches0 = S.kernel_launches()
    step_ms = []
    info = {}
    with ClockSampler(dev) as clocks:
        for _ in range(args.steps):
            ms, r = step()
            step_ms.append(ms)
            info = {"nodes": r.num_nodes, "vertices": r.num_vertices, "edges": r.num_edges, "keys": r.num_keys,
                    "depth": r.depth, "flags": bflags}
            if bflags & S.FLAG_DEDUP:
                info["dedup_keys"] = [int(S.lib().svo_result_num_dedup(r.handle, k)) for k in range(3)]
            r.close()
    torch.cuda.synchronize()
    launches = S.kernel_launches() - launches0
    dist_barrier()
    total_ms = dist_max(sum(step_ms))
    value = world * nt * args.steps / (total_ms / 1e3)
    nodes_per_s = world * info["nodes"] * args.steps / (total_ms / 1e3)

    # per-stage device times (separate steps, with events inside the library)
    stage = {}
    for _ in range(3):
        _, r = step(S.FLAG_TIMINGS)
        for k, v in r.timings().items():
            stage.setdefault(k, []).append(v)
        r.close()
    stage = {k: statistics.median(v) for k, v in stage.items()}
    emit_ms = stage.get("emit", 0.0)
    peaks = json.load(open(PEAKS_PATH)) if os.path.exists(PEAKS_PATH) else {}
    peak = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))
    emit_bytes = (EMIT_BYTES_PER_NODE_NODES_ONLY if bflags & S.FLAG_NO_VERT_EDGE else EMIT_BYTES_PER_NODE) * info["nodes"]
    achieved = emit_bytes / (emit_ms / 1e3) / 1e9 if emit_ms > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "emit_traffic_per_node.json")
    tsrc = None
    if os.path.exists(tpath) and not bflags & S.FLAG_NO_VERT_EDGE:
        # DRAM bytes per node of the k_emit variant this build runs, from an
        # ncu capture of a smaller case, scaled by this build's node count
        ent = json.load(open(tpath)).get("full_neighbors" if bflags & S.FLAG_FULL_NEIGHBORS else "default")
        if ent:
            traffic = ent["dram_bytes_per_node"] * info["nodes"]
            tsrc = f"ncu: {ent['dram_bytes_per_node']} DRAM B/node of k_emit on {ent['case']}, x this build's nodes"
    # whole-build algorithmic bytes: soup read 36 B per triangle, 8 B per
    # surface-voxel key, the node records and vertex/edge arrays as written,
    # 8 B per dedup key
    build_bytes = (36 * nt + 8 * info["keys"] + 168 * info["nodes"] + 16 * info["vertices"]
                   + 28 * info["edges"] + 8 * sum(info.get("dedup_keys", [])))
    build_ms = dist_max(sum(step_ms)) / args.steps
    build_gbs = build_bytes / (build_ms / 1e3) / 1e9
    roofline = {
        "kernel": "k_emit (node records + vertex/edge arrays)",
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": (achieved / peak) if achieved else None, "traffic": traffic, "traffic_source": tsrc,
        "peak_source": "measured" if peaks else "fallback",
        "algorithmic_bytes": emit_bytes, "launch_ms": emit_ms,
        "stage_ms": stage,
        "build_bytes_alg": build_bytes, "build_gbs": build_gbs, "build_frac": build_gbs / peak,
        "build_note": "whole build: algorithmic bytes (36 B/triangle + 8 B/key + 168 B/node + 16 B/vertex + "
                      "28 B/edge + 8 B/dedup key) / ms_per_step, of measured copy bandwidth",
    }

    # end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        h_pts = torch.from_numpy(pts).pin_memory()
        h_tris = torch.from_numpy(tris).pin_memory() if tris is not None else None
        nb = [info["nodes"] * 168, info["vertices"] * 16, info["edges"] * 28, info["keys"] * 8]
        nd = info.get("dedup_keys", [])
        nb += [8 * n for n in nd]
        out = [torch.empty(max(b, 1), dtype=torch.uint8).pin_memory() for b in nb]
        lib = S.lib()

        def e2e_step():
            flush.fill_(1)
            torch.cuda.synchronize()
            t = time.perf_counter()
            r = ctx.build(h_pts.numpy(), None if h_tris is None else h_tris.numpy(), res, bflags, sid)
            for fn, buf, n in ((lib.svo_result_copy_nodes, out[0], info["nodes"]),
                               (lib.svo_result_copy_vertices, out[1], info["vertices"]),
                               (lib.svo_result_copy_edges, out[2], info["edges"]),
                               (lib.svo_result_copy_keys, out[3], info["keys"])):
                S._check(fn(r.handle, buf.data_ptr(), n))
            for k, n in enumerate(nd):
                S._check(lib.svo_result_copy_dedup(r.handle, k, out[4 + k].data_ptr(), n))
            dt = time.perf_counter() - t
            r.close()
            return dt

        e2e_step()
        dist_barrier()
        ts = [e2e_step() for _ in range(max(2, min(args.steps, 5)))]
        tmax = dist_max(sum(ts))
        e2e = {"value": world * nt * len(ts) / tmax, "unit": "tris/s",
               "h2d_bytes_per_step": int(h_pts.numel() * 4 + (0 if h_tris is None else h_tris.numel() * 4)),
               "d2h_bytes_per_step": int(sum(nb)), "ms_per_step": 1e3 * tmax / len(ts),
               "timer": "host wall clock around svo_build + svo_result_copy_* (synchronous calls)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        stride = CPU_STRIDE[args.workload]
        spts, stris = cpu_sample(pts, tris, stride)
        threads = os.cpu_count() or 1
        dt = min(time_cpu_build(spts, stris, res, threads, bflags) for _ in range(2))
        cpu = {"value": stris.shape[0] / dt, "unit": "tris/s", "cores": threads, "kind": "port",
               "sample": cpu_sample_text(stride, wname, stris.shape[0], res, bflags) + "; best of 2 oracle builds"}

    same_input = None
    if rank == 0 and world == 1 and not args.no_extras:
        same_input = ours_on_ref_cuda_input(ctx, sid)

    writer = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import tempfile

        r = ctx.build(d_pts, d_tris, res, bflags, sid)
        nodes = r.nodes()[: 1 << 18]
        r.close()
        with tempfile.TemporaryDirectory() as td:
            writer = time_writers(nodes, td)

    if rank == 0:
        line = {
            "metric": "tris/s", "value": value, "unit": "tris/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dist_max(sum(step_ms)) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(wname, nt, res, bflags, world),
            "octree": {k: v for k, v in info.items() if k != "flags"},
            "tuning": dict(zip(TUNING_KEYS, tuning)),
            "nodes_per_s": nodes_per_s,
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary(),
            "gpu_launches": launches, "writer": writer, "ref_cuda_input": same_input,
        }
    ctx.close()
    return line if rank == 0 else None


def ours_on_ref_cuda_input(ctx, sid: int) -> dict:
    """This library on the input the reference arm times the reference's own
    CUDA build on: from the host arrays of the loaded OBJ to the octree (nodes,
    vertex/edge arrays) back in host memory, like create(); best of 5 after a
    warm-up, host wall clock."""
    import tempfile

    import torch

    import svo_b200 as S

    with tempfile.TemporaryDirectory() as td:
        pts, tris = S.load_obj(write_ref_cuda_input(td))
    res = REF_CUDA_INPUT[2]
    lib = S.lib()

    def once():
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = ctx.build(pts, tris, res, 0, sid)
        bufs = (np.empty(r.num_nodes, S.NODE_DTYPE), np.empty(r.num_vertices, S.VERTEX_DTYPE),
                np.empty(r.num_edges, S.EDGE_DTYPE))
        for fn, b in zip((lib.svo_result_copy_nodes, lib.svo_result_copy_vertices, lib.svo_result_copy_edges), bufs):
            S._check(fn(r.handle, b.ctypes.data, b.shape[0]))
        dt = time.perf_counter() - t
        n = r.num_nodes
        r.close()
        return dt, n

    once()
    best = min(once() for _ in range(5))
    return {"workload": REF_CUDA_INPUT[0], "e2e_ms": 1e3 * best[0], "nodes": best[1],
            "what": "svo_build from host arrays + node/vertex/edge copies to host, wall time"}


def result_digest(r) -> str:
    """SHA-256 over a result's node, vertex, edge and key arrays (host copies)."""
    import hashlib

    h = hashlib.sha256()
    for a in (r.nodes(), r.vertices(), r.edges(), r.keys()):
        h.update(np.ascontiguousarray(a).view(np.uint8))
    return h.hexdigest()


def batch_equals_plain(ctx, pctx, d_meshes, flags: int, sid: int, stride: int = 32) -> dict:
    """Every stride-th mesh of one (untimed) batch against its own plain build,
    byte for byte over all output arrays; raises on a difference."""
    idx = list(range(0, len(d_meshes), stride))
    results, st, rc = ctx.build_batch([d_meshes[i] for i in idx], flags, sid)
    if rc != 0:
        raise RuntimeError(f"batch build failed: {st}")
    for i, r in zip(idx, results):
        p = pctx.build(*d_meshes[i], flags, sid)
        if result_digest(r) != result_digest(p):
            raise RuntimeError(f"mesh {i}: the batched result differs from its plain build")
        p.close()
        r.close()
    return {"meshes": len(idx), "arrays": "nodes, vertices, edges, keys", "identical": True}


def time_writers(nodes: np.ndarray, tmpdir: str) -> dict:
    """The tree .obj writer (writeTree, src/SVO.cu:737-753) on the same nodes:
    this library's multithreaded formatter against the oracle's std::ofstream
    writer; both files must be byte-identical."""
    import hashlib

    import svo_b200 as S

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    a, b = os.path.join(tmpdir, "ours.obj"), os.path.join(tmpdir, "oracle.obj")
    t = time.perf_counter()
    S.write_tree_nodes(nodes, a)
    ours = time.perf_counter() - t
    t = time.perf_counter()
    oracle.write_tree_nodes(nodes, b)
    theirs = time.perf_counter() - t
    digests = []
    for path in (a, b):
        with open(path, "rb") as fh:
            digests.append(hashlib.sha256(fh.read()).hexdigest())
    size = os.path.getsize(a)
    os.remove(a)
    os.remove(b)
    if digests[0] != digests[1]:
        raise RuntimeError("the tree writers disagree")
    lines = 20 * nodes.shape[0]
    return {"nodes": int(nodes.shape[0]), "lines": lines, "bytes": size, "threads": os.cpu_count() or 1,
            "ours_s": ours, "ours_lines_per_s": lines / ours, "ours_mb_per_s": size / ours / 1e6,
            "oracle_s": theirs, "oracle_lines_per_s": lines / theirs, "identical": True}


def run_batch(args, rank: int, world: int):
    """256 meshes (seed 3, icosphere/torus, 320-80k triangles, resolutions
    64-512) built as one batch -- counting phase for all meshes, then emission
    in waves of at most --wave-gb of results -- next to the plain path (one
    svo_build per mesh) on the same resident meshes; both with the work split
    the autotuner picks for this batch.  Device time between two
    events on the build stream, host work between launches included."""
    import torch

    import svo_b200 as S
    from svo_b200 import meshgen

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    sid = stream.cuda_stream
    meshes = meshgen.batch(256, seed=3)
    flags = 0 if args.flags < 0 else args.flags
    d_meshes = [(torch.from_numpy(p).cuda(), torch.from_numpy(t).cuda(), r) for p, t, r in meshes]
    nt = sum(t.shape[0] for _, t, _ in meshes)
    ctx = S.Context(dev)
    # the voxelizer work split for this mix of meshes, chosen by the library's autotuner (untimed
    # setup); the plain path keeps the default split (made for single builds) in a context of its own
    tuning = ctx.autotune(d_meshes, flags, sid)
    pctx = S.Context(dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")
    budget = int(args.wave_gb * 1e9)

    def waves(b):
        out, first, acc = [], 0, 0
        for i in range(len(b)):
            ob = max(0, b.output_bytes(i))
            if i > first and acc + ob > budget:
                out.append((first, i - first))
                first, acc = i, 0
            acc += ob
        out.append((first, len(b) - first))
        return out

    def timed(fn):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        extra = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), extra

    def mark():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    def batch_once(extra_flags=0, phases=None):
        # phases (a list, with FLAG_TIMINGS): the CUDA-event ms of the counting phase and of each wave
        e = [mark()] if phases is not None else None
        b = ctx.batch(d_meshes, flags | extra_flags, sid)
        if e:
            e.append(mark())
        nodes, emit_ms, w = 0, 0.0, waves(b)
        for first, count in w:
            rs, st, rc = b.emit(first, count)
            if rc != 0:
                raise RuntimeError(f"batch emit failed: {st}")
            if e:
                e.append(mark())
            if extra_flags & S.FLAG_TIMINGS:
                emit_ms += rs[0].timings().get("emit", 0.0)
            for r in rs:
                nodes += r.num_nodes
                r.close()
        b.close()
        if e:
            e[-1].synchronize()
            phases[:] = [e[i].elapsed_time(e[i + 1]) for i in range(len(e) - 1)]
        return nodes, emit_ms, len(w)

    def plain_once():
        nodes = 0
        for p, t, r in d_meshes:
            res = pctx.build(p, t, r, flags, sid)
            nodes += res.num_nodes
            res.close()
        return nodes

    for _ in range(args.warmup):
        timed(batch_once)
        timed(plain_once)
    dist_barrier()
    torch.cuda.synchronize()
    launches0 = S.kernel_launches()
    batch_ms, plain_ms = [], []
    with ClockSampler(dev) as clocks:
        for _ in range(args.steps):
            ms, (nodes, _, nwaves) = timed(batch_once)
            batch_ms.append(ms)
    launches = S.kernel_launches() - launches0
    for _ in range(args.steps):
        ms, pnodes = timed(plain_once)
        plain_ms.append(ms)
    assert pnodes == nodes
    same = batch_equals_plain(ctx, pctx, d_meshes, flags, sid)
    dist_barrier()
    t_batch = dist_max(sum(batch_ms))
    t_plain = dist_max(sum(plain_ms))
    value = world * nt * args.steps / (t_batch / 1e3)
    plain_value = world * nt * args.steps / (t_plain / 1e3)
    emit_ms = statistics.median([batch_once(S.FLAG_TIMINGS)[1] for _ in range(3)])
    ph = []
    flush.fill_(1)
    batch_once(0, ph)
    phases = {"count_ms": ph[0], "wave_ms": ph[1:],
              "what": "one untimed batch after the timed steps: CUDA events on the build stream around "
                      "svo_batch_create (counting phase of all meshes) and each svo_batch_emit wave"}
    peaks = json.load(open(PEAKS_PATH)) if os.path.exists(PEAKS_PATH) else {}
    peak = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))
    emit_bytes = EMIT_BYTES_PER_NODE * nodes
    achieved = emit_bytes / (emit_ms / 1e3) / 1e9 if emit_ms > 0 else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sample_meshes = batch_cpu_sample(meshes)
        threads = os.cpu_count() or 1
        dt = sum(time_cpu_build(p, t, r, threads) for p, t, r in sample_meshes)
        st = sum(t.shape[0] for _, t, _ in sample_meshes)
        cpu = {"value": st / dt, "unit": "tris/s", "cores": threads, "kind": "port",
               "sample": f"every 32nd mesh ({len(sample_meshes)} meshes, {st} triangles), resolution capped at "
                         f"256, full oracle builds"}
    if rank == 0:
        line = {
            "metric": "tris/s", "value": value, "unit": "tris/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_batch / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch256_seed3", "meshes": len(meshes), "triangles": nt,
                       "resolutions": "64/128/256/512", "nodes": nodes, "flags": flags,
                       "emit_waves": nwaves, "wave_bytes": budget, "parallelism": f"replicas{world}",
                       "tuning": dict(zip(TUNING_KEYS, tuning)),
                       "plain_tuning": dict(zip(TUNING_KEYS, pctx.tuning)),
                       "l2_flush": "256 MiB device write before every step, outside the timed span"},
            "nodes_per_s": world * nodes * args.steps / (t_batch / 1e3),
            "plain": {"value": plain_value, "unit": "tris/s", "ms_per_step": t_plain / args.steps,
                      "path": "one svo_build per mesh, same stream, same flags, default work split"},
            "batch_over_plain": value / plain_value, "phases": phases,
            "batch_equals_plain": same,
            "e2e": None,
            "roofline": {"kernel": "k_emit (all waves)", "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "traffic": None,
                         "peak_source": "measured" if peaks else "fallback", "algorithmic_bytes": emit_bytes,
                         "launch_ms": emit_ms},
            "cpu_baseline": cpu, "clocks": clocks.summary(), "gpu_launches": launches,
        }
    ctx.close()
    return line if rank == 0 else None


def run_serve(args, rank: int, world: int):
    """Poisson request stream: meshes of the batch distribution (64 resident
    meshes, seed 4), resolutions drawn from {64, 128, 256, 512, 1024} (seed 5),
    arrivals at each rate for --window seconds.  Served: svo_server with 3
    workers, batches of up to 64, 40 GB admission budget.  Plain: the same
    requests one svo_build at a time in arrival order (one worker, batches of
    one).  Latency = build finished - submitted, from the server's clock."""
    import torch

    import svo_b200 as S
    from svo_b200 import meshgen

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(4)
    pool = [meshgen.batch_mesh(rng) for _ in range(64)]
    dpool = [(torch.from_numpy(p).cuda(), torch.from_numpy(t).cuda(), t.shape[0]) for p, t in pool]
    ctx = S.Context(dev)
    flags = 0 if args.flags < 0 else args.flags
    budget = 40 * 10**9
    rates = [float(x) for x in args.rates.split(",") if x]

    def run(rate, workers, max_batch, reqs, arrivals):
        srv = S.Server(ctx, budget, workers=workers, max_batch=max_batch, flags=flags)
        tickets = [None] * len(reqs)
        t0 = time.perf_counter()

        def client():
            for i, ((mi, res), at) in enumerate(zip(reqs, arrivals)):
                d = at - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                p, t, _ = dpool[mi]
                tickets[i] = srv.submit(p, t, res)

        th = threading.Thread(target=client)
        th.start()
        lat = []
        for _ in range(len(reqs)):  # completion order: each result released as soon as it is built
            got = srv.next(timeout_us=300_000_000)
            if got is None:
                raise RuntimeError("a served request was not built within 300 s")
            t, r, st, l = got
            if st != 0:
                raise RuntimeError(f"request {t} failed: {st}")
            lat.append(l)
            srv.release(t)
        th.join()
        span = time.perf_counter() - t0
        batches = srv.stats()["batches"]
        srv.close()
        lat = np.array(lat) * 1e3
        tris = sum(dpool[mi][2] for mi, _ in reqs)
        return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "req_per_s": len(reqs) / span, "tris_per_s": tris / span, "batches": int(batches),
                "span_s": span}

    # warm-up: every resolution once, both paths
    warm = [(i % 64, r) for i, r in enumerate((64, 128, 256, 512, 1024) * 2)]
    run(1000.0, 3, 64, warm, [0.0] * len(warm))
    run(1000.0, 1, 1, warm, [0.0] * len(warm))
    launches0 = S.kernel_launches()
    out = []
    with ClockSampler(dev) as clocks:
        for k, rate in enumerate(rates):
            rr = np.random.default_rng(5 + k)
            n = max(50, min(1500, int(rate * args.window)))
            arrivals = np.cumsum(rr.exponential(1.0 / rate, size=n)).tolist()
            reqs = [(int(rr.integers(0, 64)), int(rr.choice([64, 128, 256, 512, 1024]))) for _ in range(n)]
            served = run(rate, 3, 64, reqs, arrivals)
            plain = run(rate, 1, 1, reqs, arrivals)
            out.append({"rate": rate, "requests": n, "served": served, "plain": plain})
    launches = S.kernel_launches() - launches0
    ctx.close()
    if rank == 0:
        top = out[-1]
        line = {
            "metric": "tris/s served (p50/p99 latency per rate)", "value": top["served"]["tris_per_s"],
            "unit": "tris/s", "n_gpus": world, "steps": len(out), "warmup": 2, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "serve_poisson", "mesh_pool": "64 meshes of the batch distribution (seed 4)",
                       "resolutions": "64/128/256/512/1024", "budget_bytes": budget, "served_workers": 3,
                       "served_max_batch": 64, "flags": flags, "window_s": args.window,
                       "parallelism": f"replicas{world}"},
            "rates": out, "e2e": None, "roofline": None, "cpu_baseline": None, "clocks": clocks.summary(),
            "gpu_launches": launches,
        }
        return line
    return None


def extras(args, rank: int, world: int) -> dict:
    """Short runs of the batched (256 meshes) and served (Poisson stream)
    workloads beside the headline build, outside its timed region: each with
    its own warm-up, CUDA-event or server-clock timing and clock samples."""
    import copy

    b = copy.copy(args)
    b.steps, b.warmup, b.no_cpu, b.flags = 3, 2, True, -1
    batch = run_batch(b, rank, world)
    sv = copy.copy(args)
    sv.rates, sv.window, sv.flags = "500,2000", 0.5, -1
    serve = run_serve(sv, rank, world)
    keep_b = ("value", "unit", "ms_per_step", "plain", "batch_over_plain", "batch_equals_plain", "phases", "config",
              "clocks")
    return {"batch256": {k: batch[k] for k in keep_b} if batch else None,
            "serve": {k: serve[k] for k in ("rates", "config", "clocks")} if serve else None}


def main():
    args = parse_args()
    rank, world = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rank)
            return
        if args.workload == "batch256":
            line = run_batch(args, rank, world)
        elif args.workload == "serve":
            line = run_serve(args, rank, world)
        else:
            line = run_ours(args, rank, world)
            if line is not None and world == 1 and args.workload == "heightfield" and not args.no_extras:
                line.update(extras(args, rank, world))
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        dist_done()


if __name__ == "__main__":
    main()
