"""The C-ABI library loads and exports every entry point its headers declare."""
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(svo_\w+)\s*\(", text))
    return names


def test_exports(svo_mod):
    names = _declared()
    assert len(names) >= 25
    L = svo_mod.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_cli_built(svo_mod):
    assert os.access(svo_mod.CLI_PATH, os.X_OK)


def test_estimate_bytes_host_only(svo_mod):
    """The admission estimate is host arithmetic: grows with resolution and triangles, drops without vertex/edge arrays."""
    e64 = svo_mod.estimate_bytes(1000, 2000, 64)
    e128 = svo_mod.estimate_bytes(1000, 2000, 128)
    assert 0 < e64 < e128
    assert svo_mod.estimate_bytes(1000, 4000, 64) > e64
    assert svo_mod.estimate_bytes(1000, 2000, 1024, svo_mod.FLAG_NO_VERT_EDGE) < svo_mod.estimate_bytes(1000, 2000, 1024)
    # 16 res^2 nodes of 632 bytes dominate at res 1024
    assert 16 * 1024 ** 2 * 632 < svo_mod.estimate_bytes(0, 0, 1024) < 12e9
    # the dedup's candidate bitmap (res^3 bits) comes on top of its 32 key bytes per node
    plain, dedup = svo_mod.estimate_bytes(0, 0, 1024), svo_mod.estimate_bytes(0, 0, 1024, svo_mod.FLAG_DEDUP)
    assert dedup - plain == 1024 ** 3 // 8 + 16 * 1024 ** 2 * 32


def test_fleet_argument_checks_host_only(svo_mod):
    """The multi-GPU fleet rejects bad arguments before touching a device."""
    import ctypes as C

    L = svo_mod.lib()
    h = C.c_void_p()
    cfg = svo_mod.ServerConfig(1 << 30, 1, 1, 0)
    assert L.svo_fleet_create(None, 1, C.byref(cfg), C.byref(h)) == svo_mod.ERR_INVALID_ARGUMENT
    none = (C.c_void_p * 1)(None)
    assert L.svo_fleet_create(none, 1, C.byref(cfg), C.byref(h)) == svo_mod.ERR_INVALID_ARGUMENT
    assert L.svo_fleet_create(none, 0, C.byref(cfg), C.byref(h)) == svo_mod.ERR_INVALID_ARGUMENT
    assert not h.value
    assert L.svo_fleet_member(None, 5) == -1
    assert L.svo_fleet_stats(None, 0, None) == svo_mod.ERR_INVALID_ARGUMENT
    assert L.svo_fleet_release(None, 1) == svo_mod.ERR_INVALID_ARGUMENT
    L.svo_fleet_destroy(None)
