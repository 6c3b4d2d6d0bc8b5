"""The C ABI library loads, exports every symbol the headers under include/
declare, fails loudly when it is missing (there is no CPU fallback), and
behaves on a machine without a GPU (no compute call is made here)."""
import glob
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import spatial_query_b200 as sq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(headers=None):
    names = set()
    for h in headers or sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(sq_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_query_surface():
    syms = declared_symbols()
    for name in ["sq_ctx_create", "sq_bvh_upload", "sq_bvh_refit", "sq_raycast_nearest", "sq_raycast_all",
                 "sq_raycast_crossings", "sq_shapecast_nearest", "sq_shapecast_all", "sq_overlap", "sq_tree_build"]:
        assert name in syms


def test_library_exports_every_declared_symbol():
    lib = sq.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) <= set(sq.SIGNATURES)


def test_every_header_is_covered():
    heads = sorted(os.path.basename(h) for h in glob.glob(os.path.join(ROOT, "include", "*.h")))
    assert heads == ["sq.h", "sq_guide.h"]
    assert "sq_guide_create" in declared_symbols() and "sq_raycast_nearest_guided_d" in declared_symbols()


def test_missing_library_raises():
    code = ("import spatial_query_b200 as sq\n"
            "sq.LIB_PATH = '/nonexistent/libsqcuda.so'\n"
            "sq._lib = None\n"
            "try:\n"
            "    sq.lib()\n"
            "except ImportError as e:\n"
            "    print('raised', 'missing' in str(e))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.stdout.strip() == "raised True", out.stdout + out.stderr


_NULL_PROBE = """
import ctypes as C, sys
import spatial_query_b200 as sq
L = sq.lib()
P = C.c_void_p
v = int(sys.argv[1])
bad = []
calls = 0
for name, (res, args) in sorted(sq.SIGNATURES.items()):
    if res is not C.c_int32 or not args or args[0] is not P:
        continue
    vals = [float(v) if a in (C.c_float, C.c_double) else
            v if a in (C.c_int32, C.c_uint32, C.c_int64, C.c_uint64, C.c_size_t) else None for a in args]
    rc = getattr(L, name)(*vals)
    calls += 1
    if rc not in range(0, 8):
        bad.append((name, rc))
print(calls, bad)
"""


@pytest.mark.parametrize("size", [0, 1, 3])
def test_null_handles_return_a_status(size):
    """Every entry point that takes a handle, called with null handles and
    pointers and small sizes, returns a status code instead of faulting
    (a separate process, so that a crash names itself)."""
    out = subprocess.run([sys.executable, "-c", _NULL_PROBE, str(size)], cwd=ROOT, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    calls, bad = out.stdout.strip().split(" ", 1)
    assert int(calls) >= 60 and bad == "[]", out.stdout


def test_version():
    assert sq.lib().sq_version() == 1


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_headless_returns_none_without_a_device():
    """GpuRaycaster::headless returns None with no adapter (gpu/mod.rs:308-324)."""
    g = sq.Geometry("balls", 3, np.array([[0, 0, 0, 1]], np.float32))
    assert sq.GpuRaycaster.headless(sq.HostBvh.build(g), g) is None


def test_prim_aabbs_match_provider_bounds():
    tri = np.array([[0, 0, 0, 1, 2, -1, -3, 0.5, 4]], np.float32)
    a = sq.Geometry("tris", 3, tri).world_aabbs()
    assert np.array_equal(a, np.array([[-3, 0, -1, 1, 2, 4]], np.float32))
    b = sq.Geometry("balls", 2, np.array([[1, 2, 0.5]], np.float32)).world_aabbs()
    assert np.array_equal(b, np.array([[0.5, 1.5, 1.5, 2.5]], np.float32))


def test_tree_build_rejects_small_capacity():
    lib = sq.lib()
    import ctypes as C
    a = np.zeros((10, 6), np.float32)
    nn = C.c_uint32(0)
    out = np.empty((4, 6), np.float32)
    small = np.empty(4, np.uint32)
    rc = lib.sq_tree_build(3, 10, a.ctypes.data, 1, 4, C.byref(nn), out.ctypes.data, small.ctypes.data,
                           small.ctypes.data, small.ctypes.data, np.empty(10, np.uint32).ctypes.data)
    assert rc == sq.SQ_ERR_CAPACITY
