"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle (liboracle.so).

The oracle restates the spatial-query crate's CPU query path
(crates/spatial-query/src/{maths,accel,query}) in C++ (sq_oracle.hpp). Only
the test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use it, always as the checker or the timed CPU reference, never
as part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
NO_HIT = 0xFFFFFFFF

KIND = {"boxes": 0, "balls": 1, "balls_near": 2, "tris": 3}
INST_KIND = {"mesh": 0, "box": 1, "ball": 2}

_lib = None

P = C.c_void_p
F32P = C.POINTER(C.c_float)


def build() -> str:
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u32, i32, i64, u64, f32 = C.c_uint32, C.c_int, C.c_int64, C.c_uint64, C.c_float
        L.orc_scene_new.restype = P
        L.orc_scene_new.argtypes = [i32, i32, i32, u32, P, P, P]
        L.orc_scene_free.argtypes = [P]
        L.orc_scene_refit.argtypes = [P, P]
        L.orc_scene_node_count.restype = u32
        L.orc_scene_node_count.argtypes = [P]
        L.orc_scene_tree.argtypes = [P, P, P, P, P, P]
        L.orc_scene_stats.argtypes = [P, P, P]
        L.orc_nearest.argtypes = [P, i32, u32, P, P, f32, u64, i64, i32, P, P, P, P, P, P, P]
        L.orc_all.argtypes = [P, i32, i32, u32, P, P, f32, u64, i64, i32, u32, P, P, P, P, P, P, P]
        L.orc_shapecast_nearest.argtypes = [P, i32, u32, P, P, f32, u64, i64, i32, P, P, P, P, P, P]
        L.orc_shapecast_all.argtypes = [P, i32, u32, P, P, f32, u64, i64, i32, u32, P, P, P, P, P, P]
        L.orc_overlap.argtypes = [P, i32, u32, P, u64, i64, i32, P, P, P]
        L.orc_ray_intersect.argtypes = [i32, P, P, f32, P, P]
        L.orc_normalize.argtypes = [i32, u32, P]
        L.orc_blas_set_new.restype = P
        L.orc_blas_set_new.argtypes = [i32, u32, P, P]
        L.orc_blas_set_free.argtypes = [P]
        L.orc_tlas_new.restype = P
        L.orc_tlas_new.argtypes = [i32, i32, i32, u32, P, P, P, P, P, P, P]
        L.orc_tlas_free.argtypes = [P]
        L.orc_tlas_refit.argtypes = [P, P, P, P]
        L.orc_tlas_rebuild.argtypes = [P]
        L.orc_tlas_needs_rebuild.argtypes = [P, f32]
        L.orc_tlas_node_count.restype = u32
        L.orc_tlas_node_count.argtypes = [P]
        L.orc_tlas_tree.argtypes = [P, P, P, P, P, P, P]
        L.orc_tlas_nearest.argtypes = [P, i32, u32, P, P, f32, u64, i64, i32, P, P, P, P, P, P, P]
        L.orc_tlas_all.argtypes = [P, i32, u32, P, P, f32, u64, i64, i32, u32, P, P, P, P, P]
        L.orc_tlas_shapecast_nearest.argtypes = [P, u32, P, P, f32, u64, i64, i32, P, P, P, P, P]
        L.orc_tlas_shapecast_all.argtypes = [P, u32, P, P, f32, u64, i64, i32, u32, P, P, P, P, P]
        L.orc_tlas_overlap.argtypes = [P, u32, P, u64, i64, i32, P, P, P]
        L.orc_iso_apply.argtypes = [i32, P, P, i32, P, P]
        L.orc_iso_transform_aabb.argtypes = [i32, P, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def default_threads() -> int:
    return os.cpu_count() or 1


class Hits:
    """Nearest-hit results: leaf (NO_HIT = none), toi, normal, point, sub."""

    def __init__(self, n, dim, f64=False):
        self.leaf = np.empty(n, np.uint32)
        self.toi = np.empty(n, np.float64 if f64 else np.float32)
        self.normal = np.empty((n, dim), np.float32)
        self.point = np.empty((n, dim), np.float32)
        self.sub = np.empty(n, np.uint32)
        self.stats = None


class HitLists:
    """All-hits results: count (full), and the first k entries per query."""

    def __init__(self, n, k, dim, f64=False):
        self.count = np.empty(n, np.uint32)
        self.leaf = np.empty((n, k), np.uint32)
        self.toi = np.empty((n, k), np.float64 if f64 else np.float32)
        self.normal = np.empty((n, k, dim), np.float32)
        self.sub = np.empty((n, k), np.uint32)
        self.stats = None


class Scene:
    """A provider plus its Bvh, built by the oracle's tree::build restatement."""

    def __init__(self, kind: str, dim: int, prims, layers=None, sub=None, prec: int = 32):
        self.kind, self.dim, self.prec = kind, dim, prec
        self.prims = _f32(prims)
        self.n = 0 if self.prims is None else self.prims.shape[0]
        data = self.prims if self.n else np.zeros(1, np.float32)
        self._layers = None if layers is None else np.ascontiguousarray(layers, dtype=np.uint64)
        self._sub = None if sub is None else np.ascontiguousarray(sub, dtype=np.uint32)
        self.h = lib().orc_scene_new(dim, prec, KIND[kind], self.n, _p(data), _p(self._layers), _p(self._sub))
        if not self.h:
            raise ValueError("oracle: unsupported scene")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_scene_free(self.h)
            self.h = None

    def refit(self, prims):
        self.prims = _f32(prims)
        lib().orc_scene_refit(self.h, _p(self.prims))

    def tree(self):
        nn = lib().orc_scene_node_count(self.h)
        b = np.empty((nn, 2 * self.dim), np.float32)
        ca = np.empty(nn, np.uint32)
        cb = np.empty(nn, np.uint32)
        pc = np.empty(nn, np.uint32)
        pi = np.empty(self.n, np.uint32)
        lib().orc_scene_tree(self.h, _p(b), _p(ca), _p(cb), _p(pc), _p(pi))
        return dict(bounds=b, child_a=ca, child_b=cb, prim_count=pc, prim_indices=pi)

    def stats(self):
        out = np.zeros(4, np.uint64)
        q = C.c_double(0)
        lib().orc_scene_stats(self.h, _p(out), C.byref(q))
        return dict(node_count=int(out[0]), leaf_count=int(out[1]), prim_count=int(out[2]),
                    max_depth=int(out[3]), quality=q.value)

    def nearest(self, rays, max_toi, mask=~0 & 0xFFFFFFFFFFFFFFFF, exclude=-1, naive=False, threads=None,
                stats=False) -> Hits:
        rays = _f32(rays).reshape(-1, 2 * self.dim)
        n = rays.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        f64 = self.prec == 64
        h = Hits(n, self.dim, f64)
        st = np.empty((n, 4), np.uint64) if stats else None
        lib().orc_nearest(self.h, 1 if naive else 0, n, _p(rays), _p(mt), 0.0 if per else float(max_toi), mask,
                          exclude, threads or default_threads(), _p(h.leaf), None if f64 else _p(h.toi),
                          _p(h.toi) if f64 else None, _p(h.normal), _p(h.point), _p(h.sub), _p(st))
        h.stats = st
        return h

    def all(self, rays, max_toi, k=16, crossings=False, mask=0xFFFFFFFFFFFFFFFF, exclude=-1, naive=False,
            threads=None, stats=False) -> HitLists:
        rays = _f32(rays).reshape(-1, 2 * self.dim)
        n = rays.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        f64 = self.prec == 64
        h = HitLists(n, k, self.dim, f64)
        st = np.empty((n, 4), np.uint64) if stats else None
        lib().orc_all(self.h, 1 if naive else 0, 1 if crossings else 0, n, _p(rays), _p(mt),
                      0.0 if per else float(max_toi), mask, exclude, threads or default_threads(), k, _p(h.count),
                      _p(h.leaf), None if f64 else _p(h.toi), _p(h.toi) if f64 else None, _p(h.normal), _p(h.sub),
                      _p(st))
        h.stats = st
        return h

    def shapecast_nearest(self, casts, max_toi, mask=0xFFFFFFFFFFFFFFFF, exclude=-1, naive=False,
                          threads=None) -> Hits:
        casts = _f32(casts).reshape(-1, 4 * self.dim)
        n = casts.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        f64 = self.prec == 64
        h = Hits(n, self.dim, f64)
        lib().orc_shapecast_nearest(self.h, 1 if naive else 0, n, _p(casts), _p(mt), 0.0 if per else float(max_toi),
                                    mask, exclude, threads or default_threads(), _p(h.leaf),
                                    None if f64 else _p(h.toi), _p(h.toi) if f64 else None, _p(h.normal),
                                    _p(h.point), _p(h.sub))
        return h

    def shapecast_all(self, casts, max_toi, k=16, mask=0xFFFFFFFFFFFFFFFF, exclude=-1, naive=False,
                      threads=None) -> HitLists:
        casts = _f32(casts).reshape(-1, 4 * self.dim)
        n = casts.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        f64 = self.prec == 64
        h = HitLists(n, k, self.dim, f64)
        lib().orc_shapecast_all(self.h, 1 if naive else 0, n, _p(casts), _p(mt), 0.0 if per else float(max_toi),
                                mask, exclude, threads or default_threads(), k, _p(h.count), _p(h.leaf),
                                None if f64 else _p(h.toi), _p(h.toi) if f64 else None, _p(h.normal), _p(h.sub))
        return h

    def overlap(self, regions, mask=0xFFFFFFFFFFFFFFFF, exclude=-1, naive=False, threads=None):
        """CSR result: (offsets[n+1] u64, leaves u32), leaves ascending per query."""
        regions = _f32(regions).reshape(-1, 2 * self.dim)
        n = regions.shape[0]
        t = threads or default_threads()
        counts = np.empty(n, np.uint32)
        lib().orc_overlap(self.h, 1 if naive else 0, n, _p(regions), mask, exclude, t, _p(counts), None, None)
        offsets = np.zeros(n + 1, np.uint64)
        offsets[1:] = np.cumsum(counts, dtype=np.uint64)
        leaves = np.empty(max(int(offsets[-1]), 1), np.uint32)
        lib().orc_overlap(self.h, 1 if naive else 0, n, _p(regions), mask, exclude, t, None, _p(offsets),
                          _p(leaves))
        return offsets, leaves[: int(offsets[-1])]


class BlasSet:
    """Triangle meshes, each with its own Bvh (the lower level of a Tlas)."""

    def __init__(self, offsets, tris, prec=32):
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.tris = _f32(tris)
        self.h = lib().orc_blas_set_new(prec, len(self.offsets) - 1, _p(self.offsets), _p(self.tris))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_blas_set_free(self.h)
            self.h = None


class TlasScene:
    """Instances (mesh / box / ball kinds) under a Tlas (accel/tlas.rs)."""

    def __init__(self, kind: str, dim: int, rot, trans, param, blas_id=None, blas: BlasSet | None = None,
                 layers=None, sub=None, prec: int = 32):
        self.kind, self.dim, self.prec = kind, dim, prec
        self.rot = _f32(rot)
        self.trans = _f32(trans)
        self.param = _f32(param)
        self.n = self.trans.shape[0] if self.trans is not None else 0
        self.blas_id = None if blas_id is None else np.ascontiguousarray(blas_id, dtype=np.uint32)
        self.blas = blas
        self._layers = None if layers is None else np.ascontiguousarray(layers, dtype=np.uint64)
        self._sub = None if sub is None else np.ascontiguousarray(sub, dtype=np.uint32)
        z = np.zeros(1, np.float32)
        self.h = lib().orc_tlas_new(dim, prec, INST_KIND[kind], self.n, _p(self.rot if self.n else z),
                                    _p(self.trans if self.n else z), _p(self.param if self.n else z),
                                    _p(self.blas_id), blas.h if blas else None, _p(self._layers), _p(self._sub))
        if not self.h:
            raise ValueError("oracle: unsupported tlas")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_tlas_free(self.h)
            self.h = None

    def refit(self, trans, rot=None, param=None):
        self.trans = _f32(trans)
        if rot is not None:
            self.rot = _f32(rot)
        if param is not None:
            self.param = _f32(param)
        lib().orc_tlas_refit(self.h, _p(None if rot is None else self.rot), _p(self.trans),
                             _p(None if param is None else self.param))

    def rebuild(self):
        lib().orc_tlas_rebuild(self.h)

    def needs_rebuild(self, factor):
        return bool(lib().orc_tlas_needs_rebuild(self.h, factor))

    def tree(self):
        nn = lib().orc_tlas_node_count(self.h)
        b = np.empty((nn, 2 * self.dim), np.float32)
        ca = np.empty(nn, np.uint32)
        cb = np.empty(nn, np.uint32)
        pc = np.empty(nn, np.uint32)
        ii = np.empty(self.n, np.uint32)
        wa = np.empty((self.n, 2 * self.dim), np.float32)
        lib().orc_tlas_tree(self.h, _p(b), _p(ca), _p(cb), _p(pc), _p(ii), _p(wa))
        return dict(bounds=b, child_a=ca, child_b=cb, prim_count=pc, prim_indices=ii, world_aabbs=wa)

    def nearest(self, rays, max_toi, mask=0xFFFFFFFFFFFFFFFF, exclude=-1, naive=False, threads=None,
                stats=False) -> Hits:
        rays = _f32(rays).reshape(-1, 2 * self.dim)
        n = rays.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        f64 = self.prec == 64
        h = Hits(n, self.dim, f64)
        st = np.empty((n, 4), np.uint64) if stats else None
        lib().orc_tlas_nearest(self.h, 1 if naive else 0, n, _p(rays), _p(mt), 0.0 if per else float(max_toi), mask,
                               exclude, threads or default_threads(), _p(h.leaf), None if f64 else _p(h.toi),
                               _p(h.toi) if f64 else None, _p(h.normal), _p(h.point), _p(h.sub), _p(st))
        h.stats = st
        return h

    def all(self, rays, max_toi, k=16, crossings=False, mask=0xFFFFFFFFFFFFFFFF, exclude=-1,
            threads=None) -> HitLists:
        rays = _f32(rays).reshape(-1, 2 * self.dim)
        n = rays.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        h = HitLists(n, k, self.dim)
        lib().orc_tlas_all(self.h, 1 if crossings else 0, n, _p(rays), _p(mt), 0.0 if per else float(max_toi),
                           mask, exclude, threads or default_threads(), k, _p(h.count), _p(h.leaf), _p(h.toi),
                           _p(h.normal), _p(h.sub))
        return h

    def shapecast_nearest(self, casts, max_toi, mask=0xFFFFFFFFFFFFFFFF, exclude=-1, threads=None) -> Hits:
        casts = _f32(casts).reshape(-1, 4 * self.dim)
        n = casts.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        h = Hits(n, self.dim)
        lib().orc_tlas_shapecast_nearest(self.h, n, _p(casts), _p(mt), 0.0 if per else float(max_toi), mask,
                                         exclude, threads or default_threads(), _p(h.leaf), _p(h.toi),
                                         _p(h.normal), _p(h.point), _p(h.sub))
        return h

    def shapecast_all(self, casts, max_toi, k=16, mask=0xFFFFFFFFFFFFFFFF, exclude=-1, threads=None) -> HitLists:
        casts = _f32(casts).reshape(-1, 4 * self.dim)
        n = casts.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        h = HitLists(n, k, self.dim)
        lib().orc_tlas_shapecast_all(self.h, n, _p(casts), _p(mt), 0.0 if per else float(max_toi), mask, exclude,
                                     threads or default_threads(), k, _p(h.count), _p(h.leaf), _p(h.toi),
                                     _p(h.normal), _p(h.sub))
        return h

    def overlap(self, regions, mask=0xFFFFFFFFFFFFFFFF, exclude=-1, threads=None):
        regions = _f32(regions).reshape(-1, 2 * self.dim)
        n = regions.shape[0]
        t = threads or default_threads()
        counts = np.empty(n, np.uint32)
        lib().orc_tlas_overlap(self.h, n, _p(regions), mask, exclude, t, _p(counts), None, None)
        offsets = np.zeros(n + 1, np.uint64)
        offsets[1:] = np.cumsum(counts, dtype=np.uint64)
        leaves = np.empty(max(int(offsets[-1]), 1), np.uint32)
        lib().orc_tlas_overlap(self.h, n, _p(regions), mask, exclude, t, None, _p(offsets), _p(leaves))
        return offsets, leaves[: int(offsets[-1])]


def ray_intersect(box, ray, max_toi):
    dim = len(box) // 2
    b = _f32(box)
    r = _f32(ray)
    te = C.c_float(0)
    tx = C.c_float(0)
    ok = lib().orc_ray_intersect(dim, _p(b), _p(r), max_toi, C.byref(te), C.byref(tx))
    return (te.value, tx.value) if ok else None


def iso_apply(rot, trans, op, v):
    dim = len(v)
    r = _f32(rot).reshape(-1)
    t = _f32(trans)
    x = _f32(v)
    out = np.empty(dim, np.float32)
    lib().orc_iso_apply(dim, _p(r), _p(t), op, _p(x), _p(out))
    return out


def iso_transform_aabb(rot, trans, box):
    dim = len(trans)
    r = _f32(rot).reshape(-1)
    t = _f32(trans)
    b = _f32(box)
    out = np.empty(2 * dim, np.float32)
    lib().orc_iso_transform_aabb(dim, _p(r), _p(t), _p(b), _p(out))
    return out


def plane_rotation(dim, a, b, angle):
    """maths/isometry.rs:129-140: sin/cos evaluated in f32 like the crate."""
    r = np.eye(dim, dtype=np.float32)
    s = np.float32(np.sin(np.float32(angle)))
    c = np.float32(np.cos(np.float32(angle)))
    r[a, a] = c
    r[a, b] = -s
    r[b, a] = s
    r[b, b] = c
    return r
