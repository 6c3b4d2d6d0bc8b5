"""B200 batched-query path for spatial-query, over the C ABI in include/sq.h.

The host mirror of the crate's `gpu` feature (crates/spatial-query/src/gpu/
mod.rs) and of the Bvh batch calls it stands in for:

* ``HostBvh.build(geometry)``  -- ``Bvh::build`` (accel/bvh.rs:31-38): the
  reference median-split tree, built on the host (``sq_tree_build``).
* ``GpuRaycaster.headless(bvh, geometry)`` / ``.new(ctx, bvh, geometry)`` --
  ``GpuRaycaster::headless`` / ``new`` (gpu/mod.rs:252-324): ``None`` when
  there is no CUDA device.
* ``GpuRaycaster.refit``, ``raycast_nearest_batch`` (gpu/mod.rs:333-463), and
  the calls the WGSL path never had: ``raycast_all``, ``raycast_crossings``,
  ``shapecast_nearest``, ``shapecast_all``, ``overlap``.

Every query runs in the CUDA kernels of libsqcuda.so. There is no CPU
fallback: if the library is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsqcuda.so")

SQ_OK = 0
SQ_ERR_INVALID = 1
SQ_ERR_CUDA = 2
SQ_ERR_NO_DEVICE = 3
SQ_ERR_UNSUPPORTED = 4
SQ_ERR_DEPTH = 5
SQ_ERR_CAPACITY = 6
SQ_ERR_COMPILE = 7
NO_HIT = 0xFFFFFFFF
LAYOUT_BINARY = 0
LAYOUT_WIDE = 1
LAYOUT_QUANT = 2
LAYOUT_BINARY_REGTOP = 3
LAYOUT_BINARY_VOTE = 4
NO_SUB = 0xFFFFFFFF

NARROW = {"boxes": 0, "aabb": 0, "balls": 1, "sphere": 1, "balls_near": 2, "sphere_near": 2, "tris": 3,
          "triangle": 3}
ORDER_NEAR_FIRST = 0
ORDER_REFERENCE = 1

P = C.c_void_p


class SqError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"sq error {code}: {msg}")
        self.code = code


class _Filter(C.Structure):
    _fields_ = [("layer_mask", C.c_uint64), ("exclude", C.c_int64)]


class _Lists64(C.Structure):
    _fields_ = [("k", C.c_uint32), ("count", P), ("leaf", P), ("toi", P), ("normal", P)]


class _Hits(C.Structure):
    _fields_ = [("leaf", P), ("toi", P), ("sub_object", P), ("normal", P), ("point", P)]


class _Lists(C.Structure):
    _fields_ = [("k", C.c_uint32), ("count", P), ("leaf", P), ("toi", P), ("sub_object", P), ("normal", P)]


class _Stats(C.Structure):
    _fields_ = [("nodes_visited", C.c_uint64), ("aabb_tests", C.c_uint64), ("narrow_tests", C.c_uint64),
                ("hits", C.c_uint64)]


class _Mixed(C.Structure):
    _fields_ = [("rays", P), ("n_rays", C.c_uint32), ("ray_max_toi", C.c_float), ("ray_max_toi_per_query", P),
                ("ray_hits", _Hits), ("casts", P), ("n_casts", C.c_uint32), ("cast_max_toi", C.c_float),
                ("cast_max_toi_per_query", P), ("cast_hits", _Hits), ("regions", P), ("n_regions", C.c_uint32),
                ("region_k", C.c_uint32), ("region_count", P), ("region_leaves", P)]


class _Info(C.Structure):
    _fields_ = [("dim", C.c_int32), ("narrow", C.c_int32), ("n_nodes", C.c_uint32), ("n_prims", C.c_uint32),
                ("max_depth", C.c_uint32), ("n_interior", C.c_uint32), ("device_bytes", C.c_uint64),
                ("node_record_bytes", C.c_uint32), ("prim_record_bytes", C.c_uint32)]


_lib = None

# Every symbol include/sq.h declares, with its ctypes signature.
SIGNATURES = {
    "sq_version": (C.c_int32, []),
    "sq_ctx_create": (C.c_int32, [C.c_int32, C.POINTER(P)]),
    "sq_ctx_destroy": (C.c_int32, [P]),
    "sq_ctx_last_error": (C.c_char_p, [P]),
    "sq_ctx_stream": (P, [P]),
    "sq_ctx_set_stream": (C.c_int32, [P, P]),
    "sq_ctx_synchronize": (C.c_int32, [P]),
    "sq_ctx_set_order": (C.c_int32, [P, C.c_int32]),
    "sq_ctx_set_layout": (C.c_int32, [P, C.c_int32]),
    "sq_ctx_set_blocks_per_sm": (C.c_int32, [P, C.c_int32]),
    "sq_ctx_launch_count": (C.c_uint64, [P]),
    "sq_ctx_last_replay_count": (C.c_int32, [P, C.POINTER(C.c_uint32)]),
    "sq_ctx_set_replay_window": (C.c_int32, [P, C.c_float]),
    "sq_ctx_set_l2_persist": (C.c_int32, [P, P, C.c_uint64]),
    "sq_tree_build": (C.c_int32, [C.c_int32, C.c_uint32, P, C.c_int32, C.c_uint32, P, P, P, P, P, P]),
    "sq_prim_aabbs": (C.c_int32, [C.c_int32, C.c_int32, C.c_uint32, P, P]),
    "sq_tree_build_d": (C.c_int32, [P, C.c_int32, C.c_uint32, P, C.c_uint32, P, P, P, P, P, P]),
    "sq_tree_build_f64": (C.c_int32, [C.c_int32, C.c_uint32, P, C.c_int32, C.c_uint32, P, P, P, P, P, P]),
    "sq_prim_aabbs_f64": (C.c_int32, [C.c_int32, C.c_int32, C.c_uint32, P, P]),
    "sq_bvh_upload_f64": (C.c_int32, [P, C.c_int32, C.c_int32, C.c_uint32, P, P, P, P, C.c_uint32, P, P, C.c_uint32,
                                      P, P]),
    "sq_raycast_nearest_f64": (C.c_int32, [P, P, P, C.c_uint32, C.c_double, P, P, P, P, P, P]),
    "sq_raycast_nearest_f64_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_double, P, P, P, P, P, P]),
    "sq_raycast_all_f64": (C.c_int32, [P, P, P, C.c_uint32, C.c_double, P, P, C.c_int32, P]),
    "sq_raycast_all_f64_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_double, P, P, C.c_int32, P]),
    "sq_shapecast_nearest_f64": (C.c_int32, [P, P, P, C.c_uint32, C.c_double, P, P, P, P, P]),
    "sq_shapecast_nearest_f64_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_double, P, P, P, P, P]),
    "sq_shapecast_all_f64": (C.c_int32, [P, P, P, C.c_uint32, C.c_double, P, P, P]),
    "sq_shapecast_all_f64_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_double, P, P, P]),
    "sq_overlap_f64": (C.c_int32, [P, P, P, C.c_uint32, P, P, P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "sq_overlap_f64_d": (C.c_int32, [P, P, P, C.c_uint32, P, P, P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "sq_autotune_nearest_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, C.c_uint32, P]),
    "sq_bvh_upload_custom": (C.c_int32, [P, C.c_uint32, P, P, P, P, C.c_uint32, P, P, C.c_uint32, P, C.c_char_p,
                                         C.POINTER(P)]),
    "sq_bvh_upload": (C.c_int32, [P, C.c_int32, C.c_int32, C.c_uint32, P, P, P, P, C.c_uint32, P, P, C.c_uint32,
                                  P, P, C.POINTER(P)]),
    "sq_bvh_destroy": (C.c_int32, [P]),
    "sq_bvh_info_get": (C.c_int32, [P, C.POINTER(_Info)]),
    "sq_bvh_refit": (C.c_int32, [P, P, P]),
    "sq_bvh_refit_d": (C.c_int32, [P, P, P]),
    "sq_bvh_read_bounds": (C.c_int32, [P, P, P]),
    "sq_raycast_nearest": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P, P]),
    "sq_raycast_nearest_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P, P]),
    "sq_raycast_all": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P, P]),
    "sq_raycast_all_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P, P]),
    "sq_raycast_crossings": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_raycast_crossings_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_shapecast_nearest": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_shapecast_nearest_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_shapecast_all": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_shapecast_all_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_overlap": (C.c_int32, [P, P, P, C.c_uint32, P, P, P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "sq_overlap_d": (C.c_int32, [P, P, P, C.c_uint32, P, P, P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "sq_overlap_noalloc": (C.c_int32, [P, P, C.c_uint32, P, P, P, C.c_uint64, C.POINTER(C.c_uint64), P]),
    "sq_blas_set_upload": (C.c_int32, [P, C.c_uint32, P, P, P, P, P, P, P, P, C.POINTER(P)]),
    "sq_blas_set_destroy": (C.c_int32, [P]),
    "sq_instance_world_aabbs": (C.c_int32, [C.c_int32, C.c_int32, C.c_uint32, P, P, P, P, P, P]),
    "sq_tlas_upload": (C.c_int32, [P, C.c_int32, C.c_int32, C.c_uint32, P, P, P, P, P, C.c_uint32, P, P, P, P, P,
                                   P, P, C.POINTER(P)]),
    "sq_tlas_destroy": (C.c_int32, [P]),
    "sq_tlas_refit": (C.c_int32, [P, P, P, P, P]),
    "sq_tlas_refit_d": (C.c_int32, [P, P, P, P, P, P]),
    "sq_tlas_read_bounds": (C.c_int32, [P, P, P, P]),
    "sq_tlas_needs_rebuild": (C.c_int32, [P, P, C.c_float, C.POINTER(C.c_int32)]),
    "sq_tlas_raycast_nearest": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P, P]),
    "sq_tlas_raycast_all": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_tlas_raycast_crossings": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_tlas_shapecast_nearest": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_tlas_shapecast_all": (C.c_int32, [P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_tlas_overlap": (C.c_int32, [P, P, P, C.c_uint32, P, P, P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "sq_tlas_mixed_d": (C.c_int32, [P, P, P, P]),
    "sq_graph_begin": (C.c_int32, [P]),
    "sq_graph_end": (C.c_int32, [P, C.POINTER(P)]),
    "sq_graph_launch": (C.c_int32, [P, P]),
    "sq_graph_destroy": (C.c_int32, [P]),
    # learned guide (include/sq_guide.h)
    "sq_guide_config_default": (None, [P]),
    "sq_guide_create": (C.c_int32, [P, P, P, C.POINTER(P)]),
    "sq_guide_destroy": (C.c_int32, [P]),
    "sq_guide_get_info": (C.c_int32, [P, P]),
    "sq_guide_label_d": (C.c_int32, [P, P, C.c_uint32, C.c_float, P]),
    "sq_guide_train_step_d": (C.c_int32, [P, P, P, C.POINTER(C.c_float)]),
    "sq_guide_train_d": (C.c_int32, [P, P, P, C.c_uint32, C.c_uint32, P]),
    "sq_guide_forward_backward_d": (C.c_int32, [P, P, P, C.POINTER(C.c_float)]),
    "sq_guide_get_params": (C.c_int32, [P, P, C.c_uint64]),
    "sq_guide_set_params": (C.c_int32, [P, P, C.c_uint64]),
    "sq_guide_get_grads": (C.c_int32, [P, P, C.c_uint64]),
    "sq_guide_predict_d": (C.c_int32, [P, P, C.c_uint32, P]),
    "sq_raycast_nearest_guided_d": (C.c_int32, [P, P, P, P, C.c_uint32, C.c_float, P, P, P]),
    "sq_raycast_nearest_guided": (C.c_int32, [P, P, P, P, C.c_uint32, C.c_float, P, P]),
    "sq_guide_save": (C.c_int32, [P, P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "sq_guide_load": (C.c_int32, [P, P, C.c_size_t]),
    "sq_gemm_bf16_tn_d": (C.c_int32, [P, P, P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                      C.c_uint32]),
}

INSTANCE = {"mesh": 0, "box": 1, "ball": 2}


def lib():
    """The loaded libsqcuda.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with spatial_query_b200/build.py "
                              "(the query path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # a torch tensor (device or pinned host)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


# ---------------------------------------------------------------------------
# Host tree (Bvh::build) and leaf providers
# ---------------------------------------------------------------------------

@dataclass
class Geometry:
    """A built-in device geometry: the GpuGeometry seam (gpu/mod.rs:86-99).

    ``narrow``: "boxes" (min[D], max[D]), "balls" / "balls_near"
    (centre[D], radius) or "tris" (v0, v1, v2); ``prims`` is leaf-major.
    ``layers`` (u64 per leaf) enables the QueryFilter layer test;
    ``sub_objects`` (u32 per leaf) is returned with each hit."""
    narrow: str
    dim: int
    prims: np.ndarray
    layers: Optional[np.ndarray] = None
    sub_objects: Optional[np.ndarray] = None

    def __post_init__(self):
        self.prims = np.ascontiguousarray(self.prims, dtype=np.float32).reshape(len(self.prims), -1) \
            if len(self.prims) else np.zeros((0, self.stride), np.float32)

    @property
    def stride(self) -> int:
        n = NARROW[self.narrow]
        return 2 * self.dim if n == 0 else (9 if n == 3 else self.dim + 1)

    @property
    def leaf_count(self) -> int:
        return self.prims.shape[0]

    def world_aabbs(self) -> np.ndarray:
        out = np.empty((self.leaf_count, 2 * self.dim), np.float32)
        rc = lib().sq_prim_aabbs(self.dim, NARROW[self.narrow], self.leaf_count, _p(self.prims), _p(out))
        if rc:
            raise SqError(rc, "sq_prim_aabbs")
        return out

    def world_aabbs_f64(self, prims64: Optional[np.ndarray] = None) -> np.ndarray:
        """The leaf AABBs in f64 (sq_prim_aabbs_f64) of `prims64` (default:
        this geometry's parameters widened to double)."""
        p = np.ascontiguousarray(self.prims if prims64 is None else prims64, dtype=np.float64)
        out = np.empty((self.leaf_count, 2 * self.dim), np.float64)
        rc = lib().sq_prim_aabbs_f64(self.dim, NARROW[self.narrow], self.leaf_count, _p(p), _p(out))
        if rc:
            raise SqError(rc, "sq_prim_aabbs_f64")
        return out


@dataclass
class HostBvh:
    """The crate's host tree: tree::Node arrays and the primitive order."""
    dim: int
    bounds: np.ndarray
    child_a: np.ndarray
    child_b: np.ndarray
    prim_count: np.ndarray
    prim_indices: np.ndarray

    @property
    def node_count(self) -> int:
        return len(self.child_a)

    @classmethod
    def build_from_aabbs(cls, dim: int, aabbs: np.ndarray, threads: int = 0) -> "HostBvh":
        aabbs = _f32(aabbs).reshape(-1, 2 * dim)
        n = aabbs.shape[0]
        cap = max(2 * n - 1, 1)
        b = np.empty((cap, 2 * dim), np.float32)
        ca = np.empty(cap, np.uint32)
        cb = np.empty(cap, np.uint32)
        pc = np.empty(cap, np.uint32)
        pi = np.empty(max(n, 1), np.uint32)
        nn = C.c_uint32(0)
        rc = lib().sq_tree_build(dim, n, _p(aabbs), threads, cap, C.byref(nn), _p(b), _p(ca), _p(cb), _p(pc), _p(pi))
        if rc:
            raise SqError(rc, "sq_tree_build")
        k = nn.value
        return cls(dim, b[:k].copy(), ca[:k].copy(), cb[:k].copy(), pc[:k].copy(), pi[:n].copy())

    @classmethod
    def build(cls, geom: Geometry, threads: int = 0) -> "HostBvh":
        return cls.build_from_aabbs(geom.dim, geom.world_aabbs(), threads)

    @classmethod
    def build_f64(cls, dim: int, aabbs: np.ndarray, threads: int = 0) -> "HostBvh":
        """The crate's tree with Scalar = f64 (sq_tree_build_f64): double bounds."""
        aabbs = np.ascontiguousarray(aabbs, dtype=np.float64).reshape(-1, 2 * dim)
        n = aabbs.shape[0]
        cap = max(2 * n - 1, 1)
        b = np.empty((cap, 2 * dim), np.float64)
        ca, cb, pc = (np.empty(cap, np.uint32) for _ in range(3))
        pi = np.empty(max(n, 1), np.uint32)
        nn = C.c_uint32(0)
        rc = lib().sq_tree_build_f64(dim, n, _p(aabbs), threads, cap, C.byref(nn), _p(b), _p(ca), _p(cb), _p(pc),
                                     _p(pi))
        if rc:
            raise SqError(rc, "sq_tree_build_f64")
        k = nn.value
        return cls(dim, b[:k].copy(), ca[:k].copy(), cb[:k].copy(), pc[:k].copy(), pi[:n].copy())

    @classmethod
    def build_on_device(cls, ctx: "Context", dim: int, aabbs: np.ndarray) -> "HostBvh":
        """The same tree built on the GPU (sq_tree_build_d), read back."""
        import torch
        aabbs = _f32(aabbs).reshape(-1, 2 * dim)
        n = aabbs.shape[0]
        dev = torch.device("cuda", ctx.device)
        d_aabbs = torch.from_numpy(aabbs).to(dev)
        arrays = tree_build_d(ctx, dim, d_aabbs, n)
        torch.cuda.synchronize(dev)
        b, ca, cb, pc, pi = (t.cpu().numpy() for t in arrays)
        u = lambda a: a.view(np.uint32)
        return cls(dim, b, u(ca), u(cb), u(pc), u(pi))


def tree_build_d(ctx: "Context", dim: int, d_aabbs, n: int):
    """sq_tree_build_d on device AABBs (a CUDA tensor of n x 2*dim floats):
    (node_bounds, child_a, child_b, prim_count, prim_indices) as CUDA tensors
    cut to the node count (int32 tensors hold the u32 fields)."""
    import torch
    dev = d_aabbs.device
    cap = max(2 * n - 1, 1)
    b = torch.empty((cap, 2 * dim), dtype=torch.float32, device=dev)
    ca, cb, pc = (torch.empty(cap, dtype=torch.int32, device=dev) for _ in range(3))
    pi = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    torch.cuda.synchronize(dev)
    nn = C.c_uint32(0)
    ctx.check(lib().sq_tree_build_d(ctx.h, dim, n, C.c_void_p(d_aabbs.data_ptr()), cap, C.byref(nn),
                                    C.c_void_p(b.data_ptr()), C.c_void_p(ca.data_ptr()), C.c_void_p(cb.data_ptr()),
                                    C.c_void_p(pc.data_ptr()), C.c_void_p(pi.data_ptr())), "sq_tree_build_d")
    k = nn.value
    return b[:k], ca[:k], cb[:k], pc[:k], pi[:n]


# ---------------------------------------------------------------------------
# Device context and uploaded scene
# ---------------------------------------------------------------------------

class Context:
    """A device, a stream and the persistent-kernel bookkeeping."""

    def __init__(self, device: int = 0):
        h = P()
        rc = lib().sq_ctx_create(device, C.byref(h))
        if rc == SQ_ERR_NO_DEVICE:
            raise SqError(rc, "no CUDA device")
        if rc:
            raise SqError(rc, "sq_ctx_create")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.sq_ctx_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown may already have torn down the ctypes handles
            pass

    def check(self, rc: int, what: str):
        if rc:
            raise SqError(rc, f"{what}: {lib().sq_ctx_last_error(self.h).decode()}")

    def set_order(self, order: int):
        self.check(lib().sq_ctx_set_order(self.h, order), "set_order")

    def set_layout(self, layout: int):
        """LAYOUT_BINARY (default), LAYOUT_WIDE, LAYOUT_QUANT, LAYOUT_BINARY_REGTOP (child-pair records,
        postponed leaves, the stack's top entry in registers) or LAYOUT_BINARY_VOTE (child-pair records,
        child order by warp vote) for near-first rays."""
        self.check(lib().sq_ctx_set_layout(self.h, layout), "set_layout")

    def set_l2_persist(self, scene=None, nbytes: int = 0):
        """Keep `scene`'s node records persisting in L2 (up to nbytes set aside); no scene or 0 clears it."""
        self.check(lib().sq_ctx_set_l2_persist(self.h, scene.h if scene is not None else None, int(nbytes)),
                   "set_l2_persist")

    def set_replay_window(self, window: float):
        self.check(lib().sq_ctx_set_replay_window(self.h, window), "set_replay_window")

    def set_blocks_per_sm(self, blocks: int):
        self.check(lib().sq_ctx_set_blocks_per_sm(self.h, blocks), "set_blocks_per_sm")

    def set_stream(self, stream_ptr: int | None):
        self.check(lib().sq_ctx_set_stream(self.h, stream_ptr), "set_stream")

    @property
    def stream(self) -> int:
        return lib().sq_ctx_stream(self.h) or 0

    def synchronize(self):
        self.check(lib().sq_ctx_synchronize(self.h), "synchronize")

    @property
    def launch_count(self) -> int:
        return int(lib().sq_ctx_launch_count(self.h))

    @property
    def last_replay_count(self) -> int:
        """Queries of the last near-first nearest launch answered again in the
        reference order."""
        out = C.c_uint32(0)
        self.check(lib().sq_ctx_last_replay_count(self.h, C.byref(out)), "last_replay_count")
        return int(out.value)

    def graph_begin(self):
        """Start recording the device-pointer calls made on this context."""
        self.check(lib().sq_graph_begin(self.h), "graph_begin")

    def graph_end(self) -> "Graph":
        g = P()
        self.check(lib().sq_graph_end(self.h, C.byref(g)), "graph_end")
        return Graph(self, g)


class Graph:
    """A recorded sequence of device calls, replayed with one launch."""

    def __init__(self, ctx: Context, h):
        self.ctx, self.h = ctx, h

    def launch(self):
        self.ctx.check(lib().sq_graph_launch(self.ctx.h, self.h), "graph_launch")

    def close(self):
        if getattr(self, "h", None):
            lib().sq_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown may already have torn down the ctypes handles
            pass


@dataclass
class Hits:
    leaf: np.ndarray
    toi: np.ndarray
    normal: Optional[np.ndarray] = None
    point: Optional[np.ndarray] = None
    sub_object: Optional[np.ndarray] = None
    stats: Optional[dict] = None


@dataclass
class HitLists:
    count: np.ndarray
    leaf: np.ndarray
    toi: np.ndarray
    normal: Optional[np.ndarray] = None
    sub_object: Optional[np.ndarray] = None
    stats: Optional[dict] = None


def _filter(mask, exclude):
    if mask is None and exclude is None:
        return None
    f = _Filter()
    f.layer_mask = 0xFFFFFFFFFFFFFFFF if mask is None else mask
    f.exclude = -1 if exclude is None else exclude
    return C.byref(f)


def _stats_dict(s: _Stats) -> dict:
    return dict(nodes_visited=s.nodes_visited, aabb_tests=s.aabb_tests, narrow_tests=s.narrow_tests, hits=s.hits)


class _TuneEntry(C.Structure):
    _fields_ = [("order", C.c_int32), ("blocks_per_sm", C.c_int32), ("ms", C.c_float), ("layout", C.c_int32)]


class _TuneResult(C.Structure):
    _fields_ = [("n_entries", C.c_uint32), ("entries", _TuneEntry * 48), ("best", C.c_int32)]


class DeviceBvh:
    """An uploaded scene: child-pair node records and leaf-ordered primitive
    records in HBM (sq_bvh_upload)."""

    def __init__(self, ctx: Context, tree: HostBvh, geom: Geometry):
        if tree.dim != geom.dim:
            raise ValueError("tree and geometry dimensions differ")
        self.ctx, self.dim, self.geom = ctx, geom.dim, geom
        self._layers = None if geom.layers is None else np.ascontiguousarray(geom.layers, dtype=np.uint64)
        self._sub = None if geom.sub_objects is None else np.ascontiguousarray(geom.sub_objects, dtype=np.uint32)
        h = P()
        nn = tree.node_count
        z = np.zeros(4, np.uint32)
        ctx.check(lib().sq_bvh_upload(ctx.h, geom.dim, NARROW[geom.narrow], nn,
                                      _p(tree.bounds if nn else z), _p(tree.child_a if nn else z),
                                      _p(tree.child_b if nn else z), _p(tree.prim_count if nn else z),
                                      geom.leaf_count, _p(tree.prim_indices if nn else z),
                                      _p(geom.prims if geom.leaf_count else z), geom.stride, _p(self._layers),
                                      _p(self._sub), C.byref(h)), "sq_bvh_upload")
        self.h = h
        self.tree = tree

    def autotune_nearest_d(self, d_rays, n, max_toi, reps: int = 3) -> dict:
        """Times the order x layout x blocks-per-SM candidates on these rays, keeps the
        fastest in the context (sq_autotune_nearest_d); returns the table."""
        r = _TuneResult()
        self.ctx.check(lib().sq_autotune_nearest_d(self.ctx.h, self.h, _p(d_rays), n, float(max_toi), reps,
                                                   C.byref(r)), "autotune")
        table = [dict(order=r.entries[i].order, blocks_per_sm=r.entries[i].blocks_per_sm, ms=r.entries[i].ms,
                      layout=r.entries[i].layout) for i in range(r.n_entries)]
        return dict(best=table[r.best], table=table)

    @classmethod
    def custom(cls, ctx: Context, tree: HostBvh, prims, aabbs, source: str) -> "DeviceBvh":
        """A D = 3 scene whose narrow phase is `source` (CUDA defining
        sq_narrow, compiled at upload with NVRTC; sq_bvh_upload_custom).
        prims: [n, stride] leaf parameters; aabbs: [n, 6] the boxes the tree
        was built from."""
        prims = np.ascontiguousarray(prims, dtype=np.float32)
        if prims.ndim != 2:
            prims = prims.reshape(prims.shape[0], -1)
        aabbs = np.ascontiguousarray(aabbs, dtype=np.float32).reshape(-1, 6)
        self = cls.__new__(cls)
        self.ctx, self.dim, self.geom, self.tree = ctx, 3, None, tree
        self._layers = self._sub = None
        h = P()
        nn = tree.node_count
        z = np.zeros(4, np.uint32)
        ctx.check(lib().sq_bvh_upload_custom(ctx.h, nn, _p(tree.bounds if nn else z), _p(tree.child_a if nn else z),
                                             _p(tree.child_b if nn else z), _p(tree.prim_count if nn else z),
                                             prims.shape[0], _p(tree.prim_indices if nn else z), _p(prims),
                                             prims.shape[1], _p(aabbs), source.encode(), C.byref(h)),
                  "sq_bvh_upload_custom")
        self.h = h
        return self

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.sq_bvh_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown may already have torn down the ctypes handles
            pass

    def info(self) -> dict:
        i = _Info()
        self.ctx.check(lib().sq_bvh_info_get(self.h, C.byref(i)), "info")
        return {k: getattr(i, k) for k, _ in _Info._fields_}

    def refit(self, prims):
        prims = _f32(prims)
        self.ctx.check(lib().sq_bvh_refit(self.ctx.h, self.h, _p(prims)), "refit")

    def refit_d(self, d_prims):
        self.ctx.check(lib().sq_bvh_refit_d(self.ctx.h, self.h, _p(d_prims)), "refit_d")

    def read_bounds(self) -> np.ndarray:
        out = np.empty((max(self.tree.node_count, 1), 2 * self.dim), np.float32)
        self.ctx.check(lib().sq_bvh_read_bounds(self.ctx.h, self.h, _p(out)), "read_bounds")
        return out[: self.tree.node_count]

    # -- host-buffer queries ---------------------------------------------------

    def _nearest(self, fn, q, width, max_toi, mask, exclude, stats, outputs):
        q = _f32(q).reshape(-1, width * self.dim)
        n = q.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        h = Hits(np.empty(n, np.uint32), np.empty(n, np.float32))
        if "normal" in outputs:
            h.normal = np.empty((n, self.dim), np.float32)
        if "point" in outputs:
            h.point = np.empty((n, self.dim), np.float32)
        if "sub" in outputs:
            h.sub_object = np.empty(n, np.uint32)
        s = _Hits(_p(h.leaf), _p(h.toi), _p(h.sub_object), _p(h.normal), _p(h.point))
        args = [self.ctx.h, self.h, _p(q), n, 0.0 if per else float(max_toi), _p(mt), _filter(mask, exclude),
                C.byref(s)]
        st = _Stats() if stats else None
        if fn == "sq_raycast_nearest":
            args.append(C.byref(st) if st else None)
        self.ctx.check(getattr(lib(), fn)(*args), fn)
        if st:
            h.stats = _stats_dict(st)
        return h

    def _lists(self, fn, q, width, max_toi, k, mask, exclude, stats, outputs):
        q = _f32(q).reshape(-1, width * self.dim)
        n = q.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        h = HitLists(np.empty(n, np.uint32), np.empty((n, k), np.uint32), np.empty((n, k), np.float32))
        if "normal" in outputs:
            h.normal = np.empty((n, k, self.dim), np.float32)
        if "sub" in outputs:
            h.sub_object = np.empty((n, k), np.uint32)
        s = _Lists(k, _p(h.count), _p(h.leaf), _p(h.toi), _p(h.sub_object), _p(h.normal))
        args = [self.ctx.h, self.h, _p(q), n, 0.0 if per else float(max_toi), _p(mt), _filter(mask, exclude),
                C.byref(s)]
        st = _Stats() if stats else None
        if fn == "sq_raycast_all":
            args.append(C.byref(st) if st else None)
        self.ctx.check(getattr(lib(), fn)(*args), fn)
        if st:
            h.stats = _stats_dict(st)
        return h

    def raycast_nearest(self, rays, max_toi, mask=None, exclude=None, stats=False,
                        outputs=("normal", "point", "sub")) -> Hits:
        return self._nearest("sq_raycast_nearest", rays, 2, max_toi, mask, exclude, stats, outputs)

    def raycast_all(self, rays, max_toi, k=16, mask=None, exclude=None, stats=False,
                    outputs=("normal", "sub")) -> HitLists:
        return self._lists("sq_raycast_all", rays, 2, max_toi, k, mask, exclude, stats, outputs)

    def raycast_crossings(self, rays, max_toi, k=16, mask=None, exclude=None, outputs=("normal", "sub")) -> HitLists:
        return self._lists("sq_raycast_crossings", rays, 2, max_toi, k, mask, exclude, False, outputs)

    def shapecast_nearest(self, casts, max_toi, mask=None, exclude=None, outputs=("normal", "point", "sub")) -> Hits:
        return self._nearest("sq_shapecast_nearest", casts, 4, max_toi, mask, exclude, False, outputs)

    def shapecast_all(self, casts, max_toi, k=16, mask=None, exclude=None, outputs=("normal", "sub")) -> HitLists:
        return self._lists("sq_shapecast_all", casts, 4, max_toi, k, mask, exclude, False, outputs)

    def overlap(self, regions, mask=None, exclude=None, capacity=None):
        """CSR (offsets[n+1] u64, leaves u32), leaves ascending per query."""
        regions = _f32(regions).reshape(-1, 2 * self.dim)
        n = regions.shape[0]
        cap = capacity if capacity is not None else max(4 * n, 1024)
        while True:
            offsets = np.empty(n + 1, np.uint64)
            leaves = np.empty(max(cap, 1), np.uint32)
            total = C.c_uint64(0)
            rc = lib().sq_overlap(self.ctx.h, self.h, _p(regions), n, _filter(mask, exclude), _p(offsets),
                                  _p(leaves), cap, C.byref(total))
            if rc == SQ_ERR_CAPACITY:
                cap = int(total.value)
                continue
            self.ctx.check(rc, "sq_overlap")
            return offsets, leaves[: int(total.value)]

    # -- device-buffer queries (torch tensors; async on the context stream) -----

    def raycast_nearest_d(self, d_rays, n, max_toi, d_leaf, d_toi=None, d_normal=None, d_point=None, d_sub=None,
                          d_max_toi=None, mask=None, exclude=None, stats=False):
        s = _Hits(_p(d_leaf), _p(d_toi), _p(d_sub), _p(d_normal), _p(d_point))
        st = _Stats() if stats else None
        self.ctx.check(lib().sq_raycast_nearest_d(self.ctx.h, self.h, _p(d_rays), n, float(max_toi), _p(d_max_toi),
                                                  _filter(mask, exclude), C.byref(s),
                                                  C.byref(st) if st else None), "sq_raycast_nearest_d")
        return _stats_dict(st) if st else None

    def raycast_all_d(self, d_rays, n, max_toi, k, d_count, d_leaf, d_toi, d_normal=None, d_sub=None,
                      d_max_toi=None, mask=None, exclude=None):
        s = _Lists(k, _p(d_count), _p(d_leaf), _p(d_toi), _p(d_sub), _p(d_normal))
        self.ctx.check(lib().sq_raycast_all_d(self.ctx.h, self.h, _p(d_rays), n, float(max_toi), _p(d_max_toi),
                                              _filter(mask, exclude), C.byref(s), None), "sq_raycast_all_d")

    def shapecast_nearest_d(self, d_casts, n, max_toi, d_leaf, d_toi=None, d_normal=None, d_point=None, d_sub=None,
                            d_max_toi=None, mask=None, exclude=None):
        s = _Hits(_p(d_leaf), _p(d_toi), _p(d_sub), _p(d_normal), _p(d_point))
        self.ctx.check(lib().sq_shapecast_nearest_d(self.ctx.h, self.h, _p(d_casts), n, float(max_toi),
                                                    _p(d_max_toi), _filter(mask, exclude), C.byref(s)),
                       "sq_shapecast_nearest_d")

    def overlap_d(self, d_regions, n, d_offsets, d_leaves, capacity, mask=None, exclude=None) -> int:
        total = C.c_uint64(0)
        rc = lib().sq_overlap_d(self.ctx.h, self.h, _p(d_regions), n, _filter(mask, exclude), _p(d_offsets),
                                _p(d_leaves), capacity, C.byref(total))
        if rc != SQ_ERR_CAPACITY:
            self.ctx.check(rc, "sq_overlap_d")
        return int(total.value)


# ---------------------------------------------------------------------------
# GpuRaycaster: the crate's gpu-feature API (gpu/mod.rs:229-463)
# ---------------------------------------------------------------------------

@dataclass
class GpuHit:
    """One ray's nearest hit (gpu/mod.rs:104-114) plus the sub-object."""
    leaf: int
    time_of_impact: float
    point: np.ndarray
    normal: np.ndarray
    sub_object: Optional[int] = None


class DeviceBvh64:
    """An f64 scene (sq_bvh_upload_f64): the crate's `f64` feature on the
    device. `tree` is a HostBvh with double bounds (HostBvh.build_f64);
    `prims64` the leaf parameters in double."""

    def __init__(self, ctx: Context, tree: HostBvh, geom: Geometry, prims64: Optional[np.ndarray] = None):
        self.ctx, self.dim, self.geom = ctx, geom.dim, geom
        self.prims64 = np.ascontiguousarray(geom.prims if prims64 is None else prims64, dtype=np.float64)
        self._layers = None if geom.layers is None else np.ascontiguousarray(geom.layers, dtype=np.uint64)
        bounds = np.ascontiguousarray(tree.bounds, dtype=np.float64)
        h = P()
        nn = tree.node_count
        z = np.zeros(4, np.uint32)
        zd = np.zeros(4, np.float64)
        ctx.check(lib().sq_bvh_upload_f64(ctx.h, geom.dim, NARROW[geom.narrow], nn, _p(bounds if nn else zd),
                                          _p(tree.child_a if nn else z), _p(tree.child_b if nn else z),
                                          _p(tree.prim_count if nn else z), geom.leaf_count,
                                          _p(tree.prim_indices if nn else z),
                                          _p(self.prims64 if geom.leaf_count else zd), geom.stride,
                                          _p(self._layers), C.byref(h)), "sq_bvh_upload_f64")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.sq_bvh_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown may already have torn down the ctypes handles
            pass

    def raycast_nearest(self, rays, max_toi, mask=None, exclude=None, stats=False) -> Hits:
        """rays: [n, 2D] doubles; max_toi a scalar or one per ray."""
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 2 * self.dim)
        n = rays.shape[0]
        per = np.ndim(max_toi) > 0
        mt = np.ascontiguousarray(max_toi, dtype=np.float64) if per else None
        leaf = np.empty(n, np.uint32)
        toi = np.empty(n, np.float64)
        nrm = np.empty((n, self.dim), np.float64)
        st = _Stats() if stats else None
        self.ctx.check(lib().sq_raycast_nearest_f64(self.ctx.h, self.h, _p(rays), n, 0.0 if per else float(max_toi),
                                                    _p(mt), _filter(mask, exclude), _p(leaf), _p(toi), _p(nrm),
                                                    C.byref(st) if st is not None else None),
                       "sq_raycast_nearest_f64")
        sd = None if st is None else dict(nodes_visited=st.nodes_visited, aabb_tests=st.aabb_tests,
                                          narrow_tests=st.narrow_tests, hits=st.hits)
        return Hits(leaf, toi, nrm, None, None, sd)

    def _limits(self, max_toi):
        per = np.ndim(max_toi) > 0
        return (0.0 if per else float(max_toi)), (np.ascontiguousarray(max_toi, dtype=np.float64) if per else None)

    def _lists(self, fn, q, width, max_toi, k, mask, exclude, extra=()):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, width * self.dim)
        n = q.shape[0]
        mt0, mt = self._limits(max_toi)
        out = HitLists(np.empty(n, np.uint32), np.full((n, k), NO_HIT, np.uint32), np.zeros((n, k), np.float64),
                       np.zeros((n, k, self.dim), np.float64))
        o = _Lists64(k, _p(out.count), _p(out.leaf), _p(out.toi), _p(out.normal))
        self.ctx.check(getattr(lib(), fn)(self.ctx.h, self.h, _p(q), n, mt0, _p(mt), _filter(mask, exclude), *extra,
                                          C.byref(o)), fn)
        return out

    def raycast_all(self, rays, max_toi, k=16, mask=None, exclude=None) -> "HitLists":
        """raycast_all with Scalar = f64: the first k hits per ray in hit order, full counts."""
        return self._lists("sq_raycast_all_f64", rays, 2, max_toi, k, mask, exclude, (0,))

    def raycast_crossings(self, rays, max_toi, k=16, mask=None, exclude=None) -> "HitLists":
        return self._lists("sq_raycast_all_f64", rays, 2, max_toi, k, mask, exclude, (1,))

    def shapecast_all(self, casts, max_toi, k=16, mask=None, exclude=None) -> "HitLists":
        """casts: [n, 4D] doubles (origin, dir, probe.min, probe.max)."""
        return self._lists("sq_shapecast_all_f64", casts, 4, max_toi, k, mask, exclude)

    def shapecast_nearest(self, casts, max_toi, mask=None, exclude=None) -> Hits:
        casts = np.ascontiguousarray(casts, dtype=np.float64).reshape(-1, 4 * self.dim)
        n = casts.shape[0]
        mt0, mt = self._limits(max_toi)
        leaf = np.empty(n, np.uint32)
        toi = np.empty(n, np.float64)
        nrm = np.empty((n, self.dim), np.float64)
        self.ctx.check(lib().sq_shapecast_nearest_f64(self.ctx.h, self.h, _p(casts), n, mt0, _p(mt),
                                                      _filter(mask, exclude), _p(leaf), _p(toi), _p(nrm)),
                       "sq_shapecast_nearest_f64")
        return Hits(leaf, toi, nrm, None, None, None)

    def overlap(self, regions, mask=None, exclude=None, capacity=None):
        """CSR (offsets[n+1] u64, leaves u32) of double regions [n, 2D], leaves ascending per region."""
        regions = np.ascontiguousarray(regions, dtype=np.float64).reshape(-1, 2 * self.dim)
        n = regions.shape[0]
        cap = capacity if capacity is not None else max(4 * n, 1024)
        while True:
            offsets = np.empty(n + 1, np.uint64)
            leaves = np.empty(max(cap, 1), np.uint32)
            total = C.c_uint64(0)
            rc = lib().sq_overlap_f64(self.ctx.h, self.h, _p(regions), n, _filter(mask, exclude), _p(offsets),
                                      _p(leaves), cap, C.byref(total))
            if rc == SQ_ERR_CAPACITY and total.value > cap:
                cap = int(total.value)
                continue
            self.ctx.check(rc, "sq_overlap_f64")
            return offsets, leaves[: int(total.value)]


class GpuRaycaster:
    """Drop-in for ``spatial_query::gpu::GpuRaycaster``."""

    def __init__(self, ctx: Context, bvh: HostBvh, geom: Geometry):
        self.ctx = ctx
        self.scene = DeviceBvh(ctx, bvh, geom)

    @classmethod
    def new(cls, ctx: Context, bvh: HostBvh, geom: Geometry) -> "GpuRaycaster":
        return cls(ctx, bvh, geom)

    @classmethod
    def headless(cls, bvh: HostBvh, geom: Geometry, device: int = 0) -> Optional["GpuRaycaster"]:
        """A raycaster on its own context, or None when no CUDA device exists."""
        try:
            ctx = Context(device)
        except SqError as e:
            if e.code == SQ_ERR_NO_DEVICE:
                return None
            raise
        return cls(ctx, bvh, geom)

    def refit(self, bvh: HostBvh, geom: Geometry):
        """New leaf parameters for the same topology; the refit runs on the device."""
        self.scene.refit(geom.prims)

    def raycast_nearest_batch(self, rays, max_toi: float) -> list:
        """One Optional[GpuHit] per ray, in ray order (gpu/mod.rs:348)."""
        rays = _f32(rays).reshape(-1, 2 * self.scene.dim)
        if rays.shape[0] == 0:
            return []
        h = self.scene.raycast_nearest(rays, max_toi)
        out = []
        for i in range(rays.shape[0]):
            if h.leaf[i] == NO_HIT:
                out.append(None)
            else:
                sub = None if h.sub_object[i] == NO_SUB else int(h.sub_object[i])
                out.append(GpuHit(int(h.leaf[i]), float(h.toi[i]), h.point[i].copy(), h.normal[i].copy(), sub))
        return out

    # the batch forms of the crate's other queries
    def raycast_all(self, rays, max_toi, k=16, **kw):
        return self.scene.raycast_all(rays, max_toi, k, **kw)

    def raycast_crossings(self, rays, max_toi, k=16, **kw):
        return self.scene.raycast_crossings(rays, max_toi, k, **kw)

    def shapecast_nearest(self, casts, max_toi, **kw):
        return self.scene.shapecast_nearest(casts, max_toi, **kw)

    def shapecast_all(self, casts, max_toi, k=16, **kw):
        return self.scene.shapecast_all(casts, max_toi, k, **kw)

    def overlap(self, regions, **kw):
        return self.scene.overlap(regions, **kw)


# ---------------------------------------------------------------------------
# Two-level scenes (accel/tlas.rs)
# ---------------------------------------------------------------------------

class BlasSet:
    """Triangle meshes with their own host trees, uploaded once and shared by
    every mesh instance (the lower level of a two-level scene)."""

    def __init__(self, ctx: Context, meshes: list, threads: int = 0):
        self.ctx = ctx
        self.trees = []
        node_off, tri_off = [0], [0]
        bounds, ca, cb, pc, pi, tris = [], [], [], [], [], []
        for m in meshes:
            g = Geometry("tris", 3, m)
            t = HostBvh.build(g, threads)
            self.trees.append(t)
            bounds.append(t.bounds.reshape(-1, 6))
            ca.append(t.child_a)
            cb.append(t.child_b)
            pc.append(t.prim_count)
            pi.append(t.prim_indices[: g.leaf_count])
            tris.append(g.prims)
            node_off.append(node_off[-1] + t.node_count)
            tri_off.append(tri_off[-1] + g.leaf_count)
        cat = lambda xs, dt, shape: (np.ascontiguousarray(np.concatenate(xs), dtype=dt) if xs and sum(len(x) for x in xs)
                                     else np.zeros(shape, dt))
        self._arrays = [np.asarray(node_off, np.uint32), cat(bounds, np.float32, (1, 6)), cat(ca, np.uint32, 1),
                        cat(cb, np.uint32, 1), cat(pc, np.uint32, 1), np.asarray(tri_off, np.uint32),
                        cat(pi, np.uint32, 1), cat(tris, np.float32, (1, 9))]
        h = P()
        a = self._arrays
        ctx.check(lib().sq_blas_set_upload(ctx.h, len(meshes), _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), _p(a[4]),
                                           _p(a[5]), _p(a[6]), _p(a[7]), C.byref(h)), "sq_blas_set_upload")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().sq_blas_set_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown may already have torn down the ctypes handles
            pass


def instance_world_aabbs(kind: str, dim: int, rot, trans, param, blas_id=None, blas: BlasSet | None = None):
    n = len(trans)
    rot, trans, param = _f32(rot), _f32(trans), _f32(param)
    bid = None if blas_id is None else np.ascontiguousarray(blas_id, dtype=np.uint32)
    out = np.empty((n, 2 * dim), np.float32)
    rc = lib().sq_instance_world_aabbs(dim, INSTANCE[kind], n, _p(rot), _p(trans), _p(param), _p(bid),
                                       blas.h if blas else None, _p(out))
    if rc:
        raise SqError(rc, "sq_instance_world_aabbs")
    return out


class DeviceTlas:
    """Tlas::build over instances, uploaded (sq_tlas_upload)."""

    def __init__(self, ctx: Context, kind: str, dim: int, rot, trans, param, blas_id=None, blas: BlasSet | None = None,
                 layers=None, sub_objects=None, threads: int = 0):
        self.ctx, self.kind, self.dim, self.blas = ctx, kind, dim, blas
        self.rot, self.trans, self.param = _f32(rot), _f32(trans), _f32(param)
        self.blas_id = None if blas_id is None else np.ascontiguousarray(blas_id, dtype=np.uint32)
        self.n = len(self.trans)
        world = instance_world_aabbs(kind, dim, self.rot, self.trans, self.param, self.blas_id, blas)
        self.tree = HostBvh.build_from_aabbs(dim, world, threads)
        self._layers = None if layers is None else np.ascontiguousarray(layers, dtype=np.uint64)
        self._sub = None if sub_objects is None else np.ascontiguousarray(sub_objects, dtype=np.uint32)
        t = self.tree
        nn = t.node_count
        z = np.zeros(4, np.uint32)
        h = P()
        ctx.check(lib().sq_tlas_upload(ctx.h, dim, INSTANCE[kind], self.n, _p(self.rot), _p(self.trans),
                                       _p(self.param), _p(self.blas_id), blas.h if blas else None, nn,
                                       _p(t.bounds if nn else z), _p(t.child_a if nn else z),
                                       _p(t.child_b if nn else z), _p(t.prim_count if nn else z),
                                       _p(t.prim_indices if nn else z), _p(self._layers), _p(self._sub), C.byref(h)),
                  "sq_tlas_upload")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().sq_tlas_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown may already have torn down the ctypes handles
            pass

    def refit(self, trans, rot=None, param=None):
        self.trans = _f32(trans)
        r = None if rot is None else _f32(rot)
        pr = None if param is None else _f32(param)
        self.ctx.check(lib().sq_tlas_refit(self.ctx.h, self.h, _p(r), _p(self.trans), _p(pr)), "sq_tlas_refit")

    def refit_d(self, d_rot=None, d_trans=None, d_delta=None, d_param=None):
        self.ctx.check(lib().sq_tlas_refit_d(self.ctx.h, self.h, _p(d_rot), _p(d_trans), _p(d_delta), _p(d_param)),
                       "sq_tlas_refit_d")

    def read_bounds(self):
        nb = np.empty((max(self.tree.node_count, 1), 2 * self.dim), np.float32)
        wa = np.empty((max(self.n, 1), 2 * self.dim), np.float32)
        self.ctx.check(lib().sq_tlas_read_bounds(self.ctx.h, self.h, _p(nb), _p(wa)), "sq_tlas_read_bounds")
        return nb[: self.tree.node_count], wa[: self.n]

    def needs_rebuild(self, factor: float) -> bool:
        out = C.c_int32(0)
        self.ctx.check(lib().sq_tlas_needs_rebuild(self.ctx.h, self.h, factor, C.byref(out)), "needs_rebuild")
        return bool(out.value)

    def _nearest(self, fn, q, width, max_toi, mask, exclude, stats):
        q = _f32(q).reshape(-1, width * self.dim)
        n = q.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        h = Hits(np.empty(n, np.uint32), np.empty(n, np.float32), np.empty((n, self.dim), np.float32),
                 np.empty((n, self.dim), np.float32), np.empty(n, np.uint32))
        s = _Hits(_p(h.leaf), _p(h.toi), _p(h.sub_object), _p(h.normal), _p(h.point))
        args = [self.ctx.h, self.h, _p(q), n, 0.0 if per else float(max_toi), _p(mt), _filter(mask, exclude),
                C.byref(s)]
        st = _Stats() if stats else None
        if fn == "sq_tlas_raycast_nearest":
            args.append(C.byref(st) if st else None)
        self.ctx.check(getattr(lib(), fn)(*args), fn)
        if st:
            h.stats = _stats_dict(st)
        return h

    def _lists(self, fn, q, width, max_toi, k, mask, exclude):
        q = _f32(q).reshape(-1, width * self.dim)
        n = q.shape[0]
        per = np.ndim(max_toi) > 0
        mt = _f32(max_toi) if per else None
        h = HitLists(np.empty(n, np.uint32), np.empty((n, k), np.uint32), np.empty((n, k), np.float32),
                     np.empty((n, k, self.dim), np.float32), np.empty((n, k), np.uint32))
        s = _Lists(k, _p(h.count), _p(h.leaf), _p(h.toi), _p(h.sub_object), _p(h.normal))
        self.ctx.check(getattr(lib(), fn)(self.ctx.h, self.h, _p(q), n, 0.0 if per else float(max_toi), _p(mt),
                                          _filter(mask, exclude), C.byref(s)), fn)
        return h

    def raycast_nearest(self, rays, max_toi, mask=None, exclude=None, stats=False) -> Hits:
        return self._nearest("sq_tlas_raycast_nearest", rays, 2, max_toi, mask, exclude, stats)

    def raycast_all(self, rays, max_toi, k=16, mask=None, exclude=None) -> HitLists:
        return self._lists("sq_tlas_raycast_all", rays, 2, max_toi, k, mask, exclude)

    def raycast_crossings(self, rays, max_toi, k=16, mask=None, exclude=None) -> HitLists:
        return self._lists("sq_tlas_raycast_crossings", rays, 2, max_toi, k, mask, exclude)

    def shapecast_nearest(self, casts, max_toi, mask=None, exclude=None) -> Hits:
        return self._nearest("sq_tlas_shapecast_nearest", casts, 4, max_toi, mask, exclude, False)

    def shapecast_all(self, casts, max_toi, k=16, mask=None, exclude=None) -> HitLists:
        return self._lists("sq_tlas_shapecast_all", casts, 4, max_toi, k, mask, exclude)

    def overlap(self, regions, mask=None, exclude=None, capacity=None):
        regions = _f32(regions).reshape(-1, 2 * self.dim)
        n = regions.shape[0]
        cap = capacity if capacity is not None else max(4 * n, 1024)
        while True:
            offsets = np.empty(n + 1, np.uint64)
            leaves = np.empty(max(cap, 1), np.uint32)
            total = C.c_uint64(0)
            rc = lib().sq_tlas_overlap(self.ctx.h, self.h, _p(regions), n, _filter(mask, exclude), _p(offsets),
                                       _p(leaves), cap, C.byref(total))
            if rc == SQ_ERR_CAPACITY:
                cap = int(total.value)
                continue
            self.ctx.check(rc, "sq_tlas_overlap")
            return offsets, leaves[: int(total.value)]

    def mixed_d(self, rays=None, n_rays=0, ray_max_toi=0.0, ray_out=None, casts=None, n_casts=0, cast_max_toi=0.0,
                cast_max_toi_per_query=None, cast_out=None, regions=None, n_regions=0, region_k=0, region_count=None,
                region_leaves=None, mask=None, exclude=None):
        """One persistent launch over device buffers (torch tensors). ray_out /
        cast_out: dicts of leaf, toi, normal, point, sub tensors."""
        ro = ray_out or {}
        co = cast_out or {}
        m = _Mixed(_p(rays), n_rays, ray_max_toi, None,
                   _Hits(_p(ro.get("leaf")), _p(ro.get("toi")), _p(ro.get("sub")), _p(ro.get("normal")),
                         _p(ro.get("point"))),
                   _p(casts), n_casts, cast_max_toi, _p(cast_max_toi_per_query),
                   _Hits(_p(co.get("leaf")), _p(co.get("toi")), _p(co.get("sub")), _p(co.get("normal")),
                         _p(co.get("point"))),
                   _p(regions), n_regions, region_k, _p(region_count), _p(region_leaves))
        self.ctx.check(lib().sq_tlas_mixed_d(self.ctx.h, self.h, C.byref(m), _filter(mask, exclude)),
                       "sq_tlas_mixed_d")


# ---------------------------------------------------------------------------
# Learned guide (include/sq_guide.h)
# ---------------------------------------------------------------------------

class _GuideConfig(C.Structure):
    _fields_ = [("depth", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float), ("weight_decay", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("seed", C.c_uint64)]


class _GuideInfo(C.Structure):
    _fields_ = [("n_buckets", C.c_uint32), ("n_out", C.c_uint32), ("hidden", C.c_uint32), ("inputs", C.c_uint32),
                ("n_params", C.c_uint64), ("steps", C.c_uint32)]


class Guide:
    """The learned guide of a D = 3 scene: an MLP that predicts, per ray, the
    bucket (subtree at ``depth``) holding its nearest hit, trained and run on
    the GPU; ``raycast_nearest_guided_d`` returns the same hits as the plain
    query. Device arrays are torch tensors on the scene's device."""

    def __init__(self, scene: "DeviceBvh", depth: int = 12, batch: int = 8192, lr: float = 1e-3,
                 weight_decay: float = 0.01, seed: int = 0):
        cfg = _GuideConfig()
        lib().sq_guide_config_default(C.byref(cfg))
        cfg.depth, cfg.batch, cfg.lr, cfg.weight_decay, cfg.seed = depth, batch, lr, weight_decay, seed
        h = P()
        scene.ctx.check(lib().sq_guide_create(scene.ctx.h, scene.h, C.byref(cfg), C.byref(h)), "guide_create")
        self.h, self.scene, self.ctx, self.batch = h, scene, scene.ctx, batch

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.sq_guide_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown may already have torn down the ctypes handles
            pass

    def info(self) -> dict:
        i = _GuideInfo()
        self.ctx.check(lib().sq_guide_get_info(self.h, C.byref(i)), "guide_info")
        return {k: getattr(i, k) for k, _ in _GuideInfo._fields_}

    def label_d(self, d_rays, n, max_toi, d_labels):
        self.ctx.check(lib().sq_guide_label_d(self.h, _p(d_rays), n, float(max_toi), _p(d_labels)), "guide_label")

    def train_step_d(self, d_rays, d_labels) -> float:
        loss = C.c_float(0.0)
        self.ctx.check(lib().sq_guide_train_step_d(self.h, _p(d_rays), _p(d_labels), C.byref(loss)), "train_step")
        return float(loss.value)

    def train_d(self, d_rays, d_labels, n, epochs) -> np.ndarray:
        losses = np.zeros(max(epochs, 1), np.float32)
        self.ctx.check(lib().sq_guide_train_d(self.h, _p(d_rays), _p(d_labels), n, epochs, _p(losses)), "train")
        return losses[:epochs]

    def forward_backward_d(self, d_rays, d_labels) -> float:
        loss = C.c_float(0.0)
        self.ctx.check(lib().sq_guide_forward_backward_d(self.h, _p(d_rays), _p(d_labels), C.byref(loss)),
                       "forward_backward")
        return float(loss.value)

    def _vec(self, fn) -> np.ndarray:
        out = np.empty(self.info()["n_params"], np.float32)
        self.ctx.check(getattr(lib(), fn)(self.h, _p(out), out.size), fn)
        return out

    def get_params(self) -> np.ndarray:
        return self._vec("sq_guide_get_params")

    def get_grads(self) -> np.ndarray:
        return self._vec("sq_guide_get_grads")

    def set_params(self, v):
        v = _f32(v)
        self.ctx.check(lib().sq_guide_set_params(self.h, _p(v), v.size), "set_params")

    def predict_d(self, d_rays, n, d_bucket):
        self.ctx.check(lib().sq_guide_predict_d(self.h, _p(d_rays), n, _p(d_bucket)), "predict")

    def raycast_nearest_guided_d(self, d_rays, n, max_toi, d_leaf, d_toi=None, d_normal=None, d_bucket=None,
                                 stats=False):
        s = _Hits(_p(d_leaf), _p(d_toi), None, _p(d_normal), None)
        st = _Stats() if stats else None
        self.ctx.check(lib().sq_raycast_nearest_guided_d(self.ctx.h, self.scene.h, self.h, _p(d_rays), n,
                                                          float(max_toi), _p(d_bucket), C.byref(s),
                                                          C.byref(st) if st else None), "raycast_nearest_guided_d")
        return _stats_dict(st) if st else None

    def raycast_nearest_guided(self, rays, max_toi) -> "Hits":
        rays = _f32(rays).reshape(-1, 6)
        n = rays.shape[0]
        h = Hits(np.empty(n, np.uint32), np.empty(n, np.float32))
        h.normal = np.empty((n, 3), np.float32)
        h.point = np.empty((n, 3), np.float32)
        s = _Hits(_p(h.leaf), _p(h.toi), None, _p(h.normal), _p(h.point))
        self.ctx.check(lib().sq_raycast_nearest_guided(self.ctx.h, self.scene.h, self.h, _p(rays), n,
                                                        float(max_toi), C.byref(s), None), "raycast_nearest_guided")
        return h

    def save(self) -> bytes:
        size = C.c_size_t(0)
        self.ctx.check(lib().sq_guide_save(self.h, None, 0, C.byref(size)), "save")
        buf = (C.c_uint8 * size.value)()
        self.ctx.check(lib().sq_guide_save(self.h, buf, size.value, C.byref(size)), "save")
        return bytes(buf)

    def load(self, blob: bytes):
        buf = (C.c_uint8 * len(blob)).from_buffer_copy(blob)
        self.ctx.check(lib().sq_guide_load(self.h, buf, len(blob)), "load")


def gemm_bf16_tn_d(ctx: Context, a, b, c, m, n, k, lda, ldb, ldc):
    """C[m x n] (f32) = A[m x k] * B[n x k]^T on the tcgen05 GEMM (bf16 torch tensors)."""
    ctx.check(lib().sq_gemm_bf16_tn_d(ctx.h, _p(a), _p(b), _p(c), m, n, k, lda, ldb, ldc), "gemm_bf16_tn_d")
