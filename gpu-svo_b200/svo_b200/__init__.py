"""Python binding (ctypes) of the B200 SVO library, libsvo_b200.so.

The library is the product: CUDA kernels for sm_100a behind the C ABI in
include/svo_b200.h.  This module only marshals arguments; it fails loudly when
the shared library is missing (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libsvo_b200.so")
CLI_PATH = os.path.join(PKG_ROOT, "bin", "svo_main")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_OUT_OF_MEMORY = 3
ERR_EMPTY = 4
ERR_DEGENERATE = 5
ERR_IO = 6
ERR_PARSE = 7
ERR_UNSUPPORTED = 8
ERR_DEVICE_TIMEOUT = 9
ERR_TIMEOUT = 10
ERR_CANCELLED = 11

FLAG_FULL_NEIGHBORS = 0x1
FLAG_DEDUP = 0x2
FLAG_STRICT_FP = 0x4
FLAG_NO_VERT_EDGE = 0x8
FLAG_NO_KEYS = 0x10
FLAG_TIMINGS = 0x20
TIMING_STAGES = ("total", "bbox", "voxelize", "pyramid", "scan", "compact", "emit", "unique", "dedup")

NODE_DTYPE = np.dtype(
    [
        ("morton_code", "<u4"),
        ("is_leaf", "u1"),
        ("pad_", "u1", (3,)),
        ("origin", "<f4", (3,)),
        ("width", "<f4"),
        ("parent", "<u4"),
        ("childs", "<u4", (8,)),
        ("neighbors", "<u4", (27,)),
    ]
)
VERTEX_DTYPE = np.dtype([("pos", "<f4", (3,)), ("owner", "<u4")])
EDGE_DTYPE = np.dtype([("p0", "<f4", (3,)), ("p1", "<f4", (3,)), ("owner", "<u4")])
assert NODE_DTYPE.itemsize == 168 and VERTEX_DTYPE.itemsize == 16 and EDGE_DTYPE.itemsize == 28


class SvoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"svo error {code}: {msg}")
        self.code = code


class _Aabb(C.Structure):
    _fields_ = [("min", C.c_float * 3), ("max", C.c_float * 3), ("width", C.c_float * 3)]


class Tuning(C.Structure):
    _fields_ = [("serial_max", C.c_uint32), ("warp_max", C.c_uint32), ("split", C.c_uint32),
                ("inplace_max", C.c_uint32), ("serial_packed", C.c_uint32)]


class MeshDesc(C.Structure):
    _fields_ = [
        ("points", C.c_void_p),
        ("n_points", C.c_int64),
        ("tris", C.c_void_p),
        ("n_tris", C.c_int64),
        ("res", C.c_int * 3),
        ("flags", C.c_uint32),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("mem_budget", C.c_uint64), ("workers", C.c_int), ("max_batch", C.c_int), ("flags", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("queued", C.c_int64), ("busy_workers", C.c_int), ("reserved_bytes", C.c_uint64),
                ("batches", C.c_uint64), ("built", C.c_uint64), ("build_seconds", C.c_double),
                ("queue_seconds", C.c_double), ("peak_reserved_bytes", C.c_uint64), ("requeued", C.c_uint64),
                ("admitted_batches", C.c_uint64), ("decided_batches", C.c_uint64)]


_lib = None


def lib() -> C.CDLL:
    """Loads libsvo_b200.so (build it with `make -C gpu-svo_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `make -C gpu-svo_b200`")
        L = C.CDLL(LIB_PATH)
        vp, i64, i64p = C.c_void_p, C.c_int64, C.POINTER(C.c_int64)
        L.svo_last_error.restype = C.c_char_p
        L.svo_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
        L.svo_ctx_destroy.argtypes = [vp]
        L.svo_ctx_destroy.restype = None
        L.svo_ctx_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.svo_ctx_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.svo_ctx_autotune.argtypes = [vp, C.POINTER(MeshDesc), C.c_int, C.c_uint32, vp, C.POINTER(Tuning)]
        L.svo_load_obj.argtypes = [C.c_char_p, C.POINTER(vp), i64p, C.POINTER(vp), i64p]
        L.svo_free_host.argtypes = [vp]
        L.svo_free_host.restype = None
        L.svo_bbox_cube.argtypes = [vp, i64, C.POINTER(_Aabb)]
        L.svo_build.argtypes = [vp, vp, i64, vp, i64, C.c_int, C.c_int, C.c_int, C.c_uint32, vp, C.POINTER(vp)]
        L.svo_build_batch.argtypes = [vp, C.POINTER(MeshDesc), C.c_int, vp, C.POINTER(vp), C.POINTER(C.c_int)]
        L.svo_result_free.argtypes = [vp]
        L.svo_result_free.restype = None
        L.svo_result_depth.argtypes = [vp]
        for name in ("num_nodes", "num_vertices", "num_edges", "num_keys"):
            f = getattr(L, f"svo_result_{name}")
            f.argtypes = [vp]
            f.restype = i64
        L.svo_result_level_counts.argtypes = [vp, vp, C.c_int]
        L.svo_result_bbox.argtypes = [vp, C.POINTER(_Aabb)]
        for name in ("nodes", "vertices", "edges", "keys"):
            f = getattr(L, f"svo_result_{name}_device")
            f.argtypes = [vp]
            f.restype = vp
            g = getattr(L, f"svo_result_copy_{name}")
            g.argtypes = [vp, vp, i64]
        L.svo_result_timings.argtypes = [vp, vp, C.c_int]
        L.svo_batch_create.argtypes = [vp, C.POINTER(MeshDesc), C.c_int, C.c_uint32, vp, C.POINTER(vp)]
        L.svo_batch_size.argtypes = [vp]
        L.svo_batch_mesh_status.argtypes = [vp, C.c_int]
        L.svo_batch_mesh_nodes.argtypes = [vp, C.c_int]
        L.svo_batch_mesh_nodes.restype = i64
        L.svo_batch_mesh_output_bytes.argtypes = [vp, C.c_int]
        L.svo_batch_mesh_output_bytes.restype = i64
        L.svo_batch_emit.argtypes = [vp, C.c_int, C.c_int, C.POINTER(vp), C.POINTER(C.c_int)]
        L.svo_batch_free.argtypes = [vp]
        L.svo_batch_free.restype = None
        L.svo_estimate_bytes.argtypes = [i64, i64, C.c_int, C.c_int, C.c_int, C.c_uint32]
        L.svo_estimate_bytes.restype = C.c_uint64
        L.svo_server_create.argtypes = [vp, C.POINTER(ServerConfig), C.POINTER(vp)]
        L.svo_server_submit.argtypes = [vp, C.POINTER(MeshDesc), C.POINTER(C.c_uint64)]
        L.svo_server_wait.argtypes = [vp, C.c_uint64, i64, C.POINTER(vp), C.POINTER(C.c_int),
                                      C.POINTER(C.c_double)]
        L.svo_server_release.argtypes = [vp, C.c_uint64]
        L.svo_server_next.argtypes = [vp, i64, C.POINTER(C.c_uint64), C.POINTER(vp), C.POINTER(C.c_int),
                                      C.POINTER(C.c_double)]
        L.svo_server_stats.argtypes = [vp, C.POINTER(ServerStats)]
        L.svo_server_cancel.argtypes = [vp, C.c_uint64]
        L.svo_ctx_memory.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.svo_selftest_scan_timeout.argtypes = [vp, vp]
        L.svo_debug_fail_alloc.argtypes = [i64]
        L.svo_debug_fail_alloc.restype = i64
        L.svo_server_destroy.argtypes = [vp]
        L.svo_server_destroy.restype = None
        L.svo_fleet_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(ServerConfig), C.POINTER(vp)]
        L.svo_fleet_submit.argtypes = L.svo_server_submit.argtypes
        L.svo_fleet_wait.argtypes = L.svo_server_wait.argtypes
        L.svo_fleet_next.argtypes = L.svo_server_next.argtypes
        L.svo_fleet_release.argtypes = L.svo_server_release.argtypes
        L.svo_fleet_cancel.argtypes = L.svo_server_cancel.argtypes
        L.svo_fleet_member.argtypes = [vp, C.c_uint64]
        L.svo_fleet_stats.argtypes = [vp, C.c_int, C.POINTER(ServerStats)]
        L.svo_fleet_destroy.argtypes = [vp]
        L.svo_fleet_destroy.restype = None
        L.svo_ctx_device.argtypes = [vp, C.POINTER(C.c_int)]
        L.svo_kernel_launches.restype = i64
        L.svo_result_num_dedup.argtypes = [vp, C.c_int]
        L.svo_result_num_dedup.restype = i64
        L.svo_result_copy_dedup.argtypes = [vp, C.c_int, vp, i64]
        L.svo_write_tree.argtypes = [vp, C.c_char_p]
        L.svo_write_tree_nodes.argtypes = [vp, i64, C.c_char_p]
        L.svo_write_voxels.argtypes = [vp, C.c_char_p]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != OK:
        raise SvoError(rc, lib().svo_last_error().decode(errors="replace"))


def load_obj(path: str):
    """BaseModel::loadOBJ -> (points float32[n,3], tris int32[m,3])."""
    L = lib()
    pp, tp = C.c_void_p(), C.c_void_p()
    npnt, ntri = C.c_int64(), C.c_int64()
    _check(L.svo_load_obj(os.fsencode(path), C.byref(pp), C.byref(npnt), C.byref(tp), C.byref(ntri)))
    try:
        pts = np.ctypeslib.as_array(C.cast(pp, C.POINTER(C.c_float)), (max(1, npnt.value * 3),))[: npnt.value * 3]
        tri = np.ctypeslib.as_array(C.cast(tp, C.POINTER(C.c_int32)), (max(1, ntri.value * 3),))[: ntri.value * 3]
        return pts.reshape(-1, 3).copy(), tri.reshape(-1, 3).copy()
    finally:
        L.svo_free_host(pp)
        L.svo_free_host(tp)


def bbox_cube(points: np.ndarray) -> np.ndarray:
    pts = np.ascontiguousarray(points, dtype=np.float32)
    box = _Aabb()
    _check(lib().svo_bbox_cube(pts.ctypes.data, pts.shape[0], C.byref(box)))
    return np.array(list(box.min) + list(box.max) + list(box.width), dtype=np.float32)


def kernel_launches() -> int:
    """Kernels launched by the library in this process so far."""
    return int(lib().svo_kernel_launches())


def write_tree_nodes(nodes: np.ndarray, path: str) -> None:
    n = np.ascontiguousarray(nodes, dtype=NODE_DTYPE)
    _check(lib().svo_write_tree_nodes(n.ctypes.data, n.shape[0], os.fsencode(path)))


def _res3(res):
    if isinstance(res, (int, np.integer)):
        return (int(res),) * 3
    return tuple(int(r) for r in res)


def _ptr(a) -> int:
    """Address of a numpy array, or of a torch tensor (host or CUDA)."""
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


class Context:
    """svo_ctx: per-device state (memory pool, tuning)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().svo_ctx_create(device, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            lib().svo_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def memory(self) -> tuple:
        """(scratch bytes, result bytes) allocated from the context's pools now."""
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().svo_ctx_memory(self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    def selftest_scan_timeout(self, stream: int = 0) -> int:
        """Status of the scan self-test (ERR_DEVICE_TIMEOUT when the bounded wait works)."""
        return int(lib().svo_selftest_scan_timeout(self.handle, stream or None))

    @property
    def tuning(self) -> tuple:
        """(serial_max, warp_max, split, inplace_max, serial_packed) of the voxelizer work split."""
        t = Tuning()
        _check(lib().svo_ctx_get_tuning(self._h, C.byref(t)))
        return (t.serial_max, t.warp_max, t.split, t.inplace_max, t.serial_packed)

    @tuning.setter
    def tuning(self, value) -> None:
        cur = self.tuning
        v = tuple(int(x) for x in value) + cur[len(value):]
        _check(lib().svo_ctx_set_tuning(self._h, C.byref(Tuning(*v))))

    def autotune(self, meshes, flags: int = 0, stream: int = 0) -> tuple:
        """svo_ctx_autotune over sample meshes [(points, tris, res), ...]: installs
        and returns the fastest (serial_max, warp_max, split, inplace_max, serial_packed)."""
        descs, keep = _descs(meshes, flags)
        t = Tuning()
        _check(lib().svo_ctx_autotune(self._h, descs, len(meshes), flags, stream or None, C.byref(t)))
        return (t.serial_max, t.warp_max, t.split, t.inplace_max, t.serial_packed)

    def build(self, points, tris, res, flags: int = 0, stream: int = 0) -> "Result":
        """svo_build.  points float32[n,3] and tris int32[m,3] (tris=None: soup),
        numpy (host) or torch CUDA tensors (device)."""
        if isinstance(points, np.ndarray):
            points = np.ascontiguousarray(points, dtype=np.float32)
        if isinstance(tris, np.ndarray):
            tris = np.ascontiguousarray(tris, dtype=np.int32)
        n_points = points.shape[0]
        n_tris = 0 if tris is None else tris.shape[0]
        rx, ry, rz = _res3(res)
        h = C.c_void_p()
        _check(lib().svo_build(self._h, _ptr(points), n_points, _ptr(tris), n_tris, rx, ry, rz, flags,
                               stream or None, C.byref(h)))
        return Result(h)

    def batch(self, meshes, flags: int = 0, stream: int = 0) -> "Batch":
        """svo_batch_create over [(points, tris, res), ...] (counting phase)."""
        descs, keep = _descs(meshes, flags)
        h = C.c_void_p()
        _check(lib().svo_batch_create(self._h, descs, len(meshes), flags, stream or None, C.byref(h)))
        return Batch(h, keep)

    def build_batch(self, meshes, flags: int = 0, stream: int = 0):
        """svo_build_batch over [(points, tris, res), ...] or [(points, tris, res, flags), ...];
        returns (results, statuses, rc)."""
        descs, keep = _descs(meshes, flags)
        outs = (C.c_void_p * len(meshes))()
        st = (C.c_int * len(meshes))()
        rc = lib().svo_build_batch(self._h, descs, len(meshes), stream or None, outs, st)
        results = [Result(C.c_void_p(outs[i])) if st[i] == OK else None for i in range(len(meshes))]
        return results, list(st), rc


def debug_fail_alloc(n: int) -> int:
    """svo_debug_fail_alloc: the n-th device allocation of a build from now on
    fails (0 disarms); returns the countdown it replaces (> 0: not fired)."""
    return int(lib().svo_debug_fail_alloc(int(n)))


def estimate_bytes(n_points: int, n_tris: int, res, flags: int = 0) -> int:
    """svo_estimate_bytes: the server's admission estimate for one mesh."""
    return int(lib().svo_estimate_bytes(n_points, n_tris, *_res3(res), flags))


class Server:
    """svo_server: continuous batching of build requests under a device-memory
    budget.  Mesh arrays must stay alive until their request is released."""

    _api = "svo_server_"

    def __init__(self, ctx: "Context", mem_budget: int, workers: int = 2, max_batch: int = 64, flags: int = 0):
        cfg = ServerConfig(int(mem_budget), int(workers), int(max_batch), int(flags))
        h = C.c_void_p()
        _check(lib().svo_server_create(ctx.handle, C.byref(cfg), C.byref(h)))
        self._h = h
        self._flags = flags
        self._keep = {}

    def _fn(self, name):
        return getattr(lib(), self._api + name)

    def submit(self, points, tris, res) -> int:
        descs, keep = _descs([(points, tris, res)], self._flags)
        t = C.c_uint64()
        _check(self._fn("submit")(self._h, descs, C.byref(t)))
        self._keep[t.value] = (descs, keep)
        return t.value

    def wait(self, ticket: int, timeout_us: int = -1):
        """(Result borrowed until release, status, latency seconds); None on timeout."""
        r = C.c_void_p()
        st = C.c_int()
        lat = C.c_double()
        rc = self._fn("wait")(self._h, ticket, timeout_us, C.byref(r), C.byref(st), C.byref(lat))
        if rc == ERR_TIMEOUT:
            return None
        _check(rc)
        return (Result(r, owned=False) if st.value == OK else None), st.value, lat.value

    def next(self, timeout_us: int = -1):
        """(ticket, Result borrowed until release, status, latency s) of the next
        finished request in completion order; None on timeout."""
        t = C.c_uint64()
        r = C.c_void_p()
        st = C.c_int()
        lat = C.c_double()
        rc = self._fn("next")(self._h, timeout_us, C.byref(t), C.byref(r), C.byref(st), C.byref(lat))
        if rc == ERR_TIMEOUT:
            return None
        _check(rc)
        return t.value, (Result(r, owned=False) if st.value == OK else None), st.value, lat.value

    def release(self, ticket: int) -> None:
        _check(self._fn("release")(self._h, ticket))
        self._keep.pop(ticket, None)

    def cancel(self, ticket: int) -> None:
        """Withdraws a queued request (it finishes with ERR_CANCELLED)."""
        _check(self._fn("cancel")(self._h, ticket))

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib().svo_server_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            self._fn("destroy")(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Fleet(Server):
    """svo_fleet: one server per context (one context per GPU) behind one
    ticket space; each request is built whole on the member holding the fewest
    estimated bytes.  The contexts must outlive the fleet."""

    _api = "svo_fleet_"

    def __init__(self, ctxs, mem_budget: int, workers: int = 2, max_batch: int = 64, flags: int = 0):
        cfg = ServerConfig(int(mem_budget), int(workers), int(max_batch), int(flags))
        hs = (C.c_void_p * len(ctxs))(*[c.handle for c in ctxs])
        h = C.c_void_p()
        _check(lib().svo_fleet_create(hs, len(ctxs), C.byref(cfg), C.byref(h)))
        self._h = h
        self._flags = flags
        self._keep = {}
        self._n = len(ctxs)

    def member(self, ticket: int) -> int:
        """Index of the context that builds `ticket` (-1: not held)."""
        return lib().svo_fleet_member(self._h, ticket)

    def stats(self, member: int = None):
        """One member's server statistics, or a list of all of them."""
        if member is None:
            return [self.stats(i) for i in range(self._n)]
        s = ServerStats()
        _check(lib().svo_fleet_stats(self._h, member, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}


def _descs(meshes, flags):
    keep = []
    descs = (MeshDesc * len(meshes))()
    for i, item in enumerate(meshes):
        pts, tri, res = item[:3]
        f = item[3] if len(item) > 3 else flags
        if isinstance(pts, np.ndarray):
            pts = np.ascontiguousarray(pts, dtype=np.float32)
        if isinstance(tri, np.ndarray):
            tri = np.ascontiguousarray(tri, dtype=np.int32)
        keep.append((pts, tri))
        d = descs[i]
        d.points = _ptr(pts)
        d.n_points = pts.shape[0]
        d.tris = _ptr(tri) if tri is not None else None
        d.n_tris = 0 if tri is None else tri.shape[0]
        d.res[:] = _res3(res)
        d.flags = f
    return descs, keep


class Batch:
    """svo_batch: counting phase done for every mesh; emit() writes octrees."""

    def __init__(self, h, keep):
        self._h = h
        self._keep = keep

    def __len__(self) -> int:
        return lib().svo_batch_size(self._h)

    def status(self, i: int) -> int:
        return lib().svo_batch_mesh_status(self._h, i)

    def nodes(self, i: int) -> int:
        return lib().svo_batch_mesh_nodes(self._h, i)

    def output_bytes(self, i: int) -> int:
        return lib().svo_batch_mesh_output_bytes(self._h, i)

    def emit(self, first: int, count: int):
        outs = (C.c_void_p * count)()
        st = (C.c_int * count)()
        rc = lib().svo_batch_emit(self._h, first, count, outs, st)
        return [Result(C.c_void_p(outs[i])) if st[i] == OK else None for i in range(count)], list(st), rc

    def close(self) -> None:
        if self._h:
            lib().svo_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Result:
    """svo_result: device-resident octree of one build (owned: freed by
    close(); borrowed: a server's result, valid until its ticket is released)."""

    def __init__(self, h: C.c_void_p, owned: bool = True):
        self._h = h
        self._owned = owned

    def close(self) -> None:
        if self._h and self._owned:
            lib().svo_result_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def depth(self) -> int:
        return lib().svo_result_depth(self._h)

    @property
    def num_nodes(self) -> int:
        return lib().svo_result_num_nodes(self._h)

    @property
    def num_vertices(self) -> int:
        return lib().svo_result_num_vertices(self._h)

    @property
    def num_edges(self) -> int:
        return lib().svo_result_num_edges(self._h)

    @property
    def num_keys(self) -> int:
        return lib().svo_result_num_keys(self._h)

    @property
    def level_counts(self) -> np.ndarray:
        out = np.zeros(64, dtype=np.int64)
        n = lib().svo_result_level_counts(self._h, out.ctypes.data, 64)
        return out[:n].copy()

    @property
    def bbox(self) -> np.ndarray:
        box = _Aabb()
        _check(lib().svo_result_bbox(self._h, C.byref(box)))
        return np.array(list(box.min) + list(box.max) + list(box.width), dtype=np.float32)

    def _copy(self, name: str, n: int, dtype) -> np.ndarray:
        out = np.zeros(n, dtype=dtype)
        _check(getattr(lib(), f"svo_result_copy_{name}")(self._h, out.ctypes.data, n))
        return out

    def nodes(self) -> np.ndarray:
        return self._copy("nodes", self.num_nodes, NODE_DTYPE)

    def vertices(self) -> np.ndarray:
        return self._copy("vertices", self.num_vertices, VERTEX_DTYPE)

    def edges(self) -> np.ndarray:
        return self._copy("edges", self.num_edges, EDGE_DTYPE)

    def keys(self) -> np.ndarray:
        return self._copy("keys", self.num_keys, np.uint64)

    def timings(self) -> dict:
        """Per-stage device ms of a build made with FLAG_TIMINGS."""
        ms = np.zeros(16, dtype=np.float32)
        n = lib().svo_result_timings(self._h, ms.ctypes.data, 16)
        return {TIMING_STAGES[i]: float(ms[i]) for i in range(n)}

    def dedup(self, kind: int) -> np.ndarray:
        n = lib().svo_result_num_dedup(self._h, kind)
        out = np.zeros(max(n, 0), dtype=np.uint64)
        _check(lib().svo_result_copy_dedup(self._h, kind, out.ctypes.data, out.shape[0]))
        return out

    def device_ptr(self, name: str) -> int:
        return getattr(lib(), f"svo_result_{name}_device")(self._h) or 0

    def write_tree(self, path: str) -> None:
        _check(lib().svo_write_tree(self._h, os.fsencode(path)))

    def write_voxels(self, path: str) -> None:
        _check(lib().svo_write_voxels(self._h, os.fsencode(path)))
