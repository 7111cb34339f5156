"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, as the checker or the timed CPU baseline.  The product
(gpu-svo_b200/) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

FLAG_FULL_NEIGHBORS = 0x1
FLAG_DEDUP = 0x2
FLAG_STRICT_FP = 0x4
FLAG_NO_VERT_EDGE = 0x8

# SVONode (src/SVO.h:20-35), 168 bytes
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


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        i64p = C.POINTER(C.c_int64)
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_load_obj.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), i64p, C.POINTER(C.c_void_p), i64p]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_bbox_cube.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        L.oracle_morton_encode.argtypes = [C.c_uint32] * 3
        L.oracle_morton_encode.restype = C.c_uint64
        L.oracle_morton_decode.argtypes = [C.c_uint64] + [C.POINTER(C.c_uint32)] * 3
        L.oracle_build.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int,
                                   C.c_uint32, C.c_int, C.POINTER(C.c_void_p)]
        L.oracle_voxelize.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int,
                                      C.c_uint32, C.c_int, C.POINTER(C.c_void_p), i64p]
        for name in ("num_nodes", "num_vertices", "num_edges", "num_keys"):
            f = getattr(L, f"oracle_result_{name}")
            f.argtypes = [C.c_void_p]
            f.restype = C.c_int64
        L.oracle_result_depth.argtypes = [C.c_void_p]
        L.oracle_result_level_counts.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        for name in ("nodes", "vertices", "edges", "keys", "bbox"):
            f = getattr(L, f"oracle_result_{name}")
            f.argtypes = [C.c_void_p]
            f.restype = C.c_void_p
        L.oracle_result_num_dedup.argtypes = [C.c_void_p, C.c_int]
        L.oracle_result_num_dedup.restype = C.c_int64
        L.oracle_result_dedup.argtypes = [C.c_void_p, C.c_int]
        L.oracle_result_dedup.restype = C.c_void_p
        L.oracle_tables.argtypes = [C.c_void_p] * 4
        L.oracle_fp_eval.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p]
        L.oracle_set_fp_sites.argtypes = [C.c_void_p, C.c_int]
        L.oracle_result_free.argtypes = [C.c_void_p]
        L.oracle_write_tree.argtypes = [C.c_void_p, C.c_char_p]
        L.oracle_write_voxels.argtypes = [C.c_void_p, C.c_char_p]
        L.oracle_write_tree_nodes.argtypes = [C.c_void_p, C.c_int64, C.c_char_p]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise OracleError(rc, lib().oracle_last_error().decode())


def _copy(ptr: int, n: int, dtype) -> np.ndarray:
    out = np.empty(n, dtype=dtype)
    if n:
        C.memmove(out.ctypes.data, ptr, out.nbytes)
    return out


def load_obj(path: str):
    """BaseModel::loadOBJ -> (points float32[n,3], tris int32[m,3])."""
    L = lib()
    pp, tp = C.c_void_p(), C.c_void_p()
    npnt, ntri = C.c_int64(), C.c_int64()
    _check(L.oracle_load_obj(path.encode(), C.byref(pp), C.byref(npnt), C.byref(tp), C.byref(ntri)))
    pts = _copy(pp.value, npnt.value * 3, np.float32).reshape(-1, 3)
    tri = _copy(tp.value, ntri.value * 3, np.int32).reshape(-1, 3)
    L.oracle_free(pp)
    L.oracle_free(tp)
    return pts, tri


def bbox_cube(points: np.ndarray) -> np.ndarray:
    pts = np.ascontiguousarray(points, dtype=np.float32)
    out = np.zeros(9, dtype=np.float32)
    _check(lib().oracle_bbox_cube(pts.ctypes.data, pts.shape[0], out.ctypes.data))
    return out


def morton_encode(x: int, y: int, z: int) -> int:
    return int(lib().oracle_morton_encode(x, y, z))


def tables() -> dict:
    out = {"neighbor_LUTparent": np.zeros(216, np.int16), "neighbor_LUTchild": np.zeros(216, np.int16),
           "d_vertSharedLUT": np.zeros(64, np.int16), "d_edgeSharedLUT": np.zeros(48, np.int16)}
    lib().oracle_tables(*(a.ctypes.data for a in out.values()))
    return out


FP_ARITY = {0: (4, 1), 1: (6, 1), 2: (4, 1), 3: (3, 1), 4: (3, 3), 5: (14, 1), 6: (14, 14)}
FP_SITES = ("cross", "sq_inner", "sq_outer", "d12_inner", "d12_outer", "d_edge", "plane_inner", "plane_outer",
            "loop_xy0", "loop_xy1", "loop_xy2", "loop_yz0", "loop_yz1", "loop_yz2", "loop_zx0", "loop_zx1", "loop_zx2")


def set_fp_sites(choice) -> None:
    """Contraction choice per site (0 first product, 1 second, 2 none)."""
    arr = (C.c_int * len(choice))(*choice)
    lib().oracle_set_fp_sites(arr, len(choice))


def fp_eval(op: int, strict: bool, operands: np.ndarray) -> np.ndarray:
    """The oracle's float model for one expression shape (see oracle_fp_eval)."""
    k_in, k_out = FP_ARITY[op]
    a = np.ascontiguousarray(operands, dtype=np.float32).reshape(-1, k_in)
    out = np.zeros((a.shape[0], k_out), dtype=np.float32)
    _check(lib().oracle_fp_eval(op, int(strict), a.ctypes.data, a.shape[0], out.ctypes.data))
    return out


def morton_decode(code: int):
    x, y, z = C.c_uint32(), C.c_uint32(), C.c_uint32()
    lib().oracle_morton_decode(code, C.byref(x), C.byref(y), C.byref(z))
    return x.value, y.value, z.value


def _res3(res):
    if isinstance(res, int):
        return (res, res, res)
    return tuple(int(r) for r in res)


def voxelize(points, tris, res, flags: int = 0, threads: int = 0) -> np.ndarray:
    pts = np.ascontiguousarray(points, dtype=np.float32)
    tri = np.ascontiguousarray(tris, dtype=np.int32)
    rx, ry, rz = _res3(res)
    cp, n = C.c_void_p(), C.c_int64()
    L = lib()
    _check(L.oracle_voxelize(pts.ctypes.data, pts.shape[0], tri.ctypes.data, tri.shape[0], rx, ry, rz,
                             flags, threads, C.byref(cp), C.byref(n)))
    out = _copy(cp.value, n.value, np.uint64)
    L.oracle_free(cp)
    return out


class Result:
    """Outputs of the oracle's create(); each array is copied into numpy on
    first access (the handle keeps the oracle's own copy until close())."""

    def __init__(self, handle):
        L = lib()
        self.depth = L.oracle_result_depth(handle)
        lc = np.zeros(64, dtype=np.int64)
        n = L.oracle_result_level_counts(handle, lc.ctypes.data, 64)
        self.level_counts = lc[:n].copy()
        self.bbox = _copy(L.oracle_result_bbox(handle), 9, np.float32)
        self._handle = handle
        self._cache = {}

    def _get(self, name, fetch):
        if name not in self._cache:
            if not self._handle:
                raise OracleError(-1, "result already closed")
            self._cache[name] = fetch(lib(), self._handle)
        return self._cache[name]

    @property
    def nodes(self) -> np.ndarray:
        return self._get("nodes", lambda L, h: _copy(L.oracle_result_nodes(h), L.oracle_result_num_nodes(h),
                                                      NODE_DTYPE))

    @property
    def vertices(self) -> np.ndarray:
        return self._get("vertices", lambda L, h: _copy(L.oracle_result_vertices(h),
                                                         L.oracle_result_num_vertices(h), VERTEX_DTYPE))

    @property
    def edges(self) -> np.ndarray:
        return self._get("edges", lambda L, h: _copy(L.oracle_result_edges(h), L.oracle_result_num_edges(h),
                                                      EDGE_DTYPE))

    @property
    def keys(self) -> np.ndarray:
        return self._get("keys", lambda L, h: _copy(L.oracle_result_keys(h), L.oracle_result_num_keys(h),
                                                     np.uint64))

    @property
    def dedup(self) -> list:
        return self._get("dedup", lambda L, h: [
            _copy(L.oracle_result_dedup(h, k), max(0, L.oracle_result_num_dedup(h, k)), np.uint64)
            for k in range(3)])

    def write_tree(self, path: str) -> None:
        _check(lib().oracle_write_tree(self._handle, path.encode()))

    def write_voxels(self, path: str) -> None:
        """writeVoxel as create() calls it: one cube per surface voxel."""
        _check(lib().oracle_write_voxels(self._handle, path.encode()))

    def close(self) -> None:
        if self._handle:
            lib().oracle_result_free(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_tree_nodes(nodes: np.ndarray, path: str) -> None:
    """writeTree's std::ofstream writer over a node array (168-byte records)."""
    n = np.ascontiguousarray(nodes)
    assert n.dtype.itemsize == NODE_DTYPE.itemsize
    _check(lib().oracle_write_tree_nodes(n.ctypes.data, n.shape[0], path.encode()))


def build_svo(points, tris, res, flags: int = 0, threads: int = 0) -> Result:
    pts = np.ascontiguousarray(points, dtype=np.float32)
    tri = np.ascontiguousarray(tris, dtype=np.int32)
    rx, ry, rz = _res3(res)
    h = C.c_void_p()
    _check(lib().oracle_build(pts.ctypes.data, pts.shape[0], tri.ctypes.data, tri.shape[0], rx, ry, rz,
                              flags, threads, C.byref(h)))
    return Result(h.value)
