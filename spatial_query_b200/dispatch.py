"""Backend selection for batched nearest-ray queries, with this library as
the `Gpu` backend: the crate's Dispatcher and cost model
(crates/spatial-query/src/dispatch.rs) restated, plus the B200 cost
constants `calibrate_gpu` measures.

The CPU and draw-pass constants are the crate's (dispatch.rs:40-78).
`REFERENCE_GPU` holds the crate's constants for its wgpu backend
(dispatch.rs:62-78, measured on its reference machine); `B200` holds this
library's, measured by `calibrate_gpu` on a B200 through the host-buffer
call (sq_raycast_nearest: rays copied in, launch, hits copied out), the same
per-batch shape as the crate's (a fixed cost plus a per-ray cost growing
with depth squared).
"""
from __future__ import annotations

import ctypes as C
import enum
import math
import time
from dataclasses import dataclass, replace
from typing import List, Optional

import numpy as np


class BackendKind(enum.Enum):
    """dispatch.rs:122-152."""
    CPU = "Cpu"
    DRAW_PASS = "DrawPass"
    GPU = "Gpu"


@dataclass(frozen=True)
class QueryContext:
    """The shape of a batch request (dispatch.rs:154-220)."""
    batch_size: int
    distinct_directions: int
    scene_leaves: int
    device_available: bool = False
    require_deterministic: bool = False
    narrow_cost_hint: float = 1.0

    def with_device(self, available: bool) -> "QueryContext":
        return replace(self, device_available=available)

    def with_narrow_cost(self, hint: float) -> "QueryContext":
        return replace(self, narrow_cost_hint=max(hint, 0.0))

    def deterministic(self, required: bool) -> "QueryContext":
        return replace(self, require_deterministic=required)


@dataclass(frozen=True)
class GpuCosts:
    """gpu_batch_us = fixed_us + batch * (traversal + hint * narrow) * depth^2."""
    fixed_us: float
    traversal_us_per_level2: float
    narrow_us_per_level2: float
    source: str


# The crate's constants (dispatch.rs:40-78).
CPU_TRAVERSAL_US_PER_LEVEL2 = 0.0020
CPU_NARROW_US_PER_LEVEL2 = 0.0078
DRAW_PASS_READBACK_US = 0.5
DRAW_PASS_US_PER_LEAF = 0.002
REFERENCE_GPU = GpuCosts(1350.0, 0.00004, 0.000153, "the crate's wgpu backend (dispatch.rs:62-78)")

# This library on one B200, measured by calibrate_gpu (100,000 leaves,
# 1,048,576-ray batches, median of 5, host buffers in and out; two runs gave
# 45.9 / 46.6 us fixed, 7.71e-6 / 7.63e-6 and 8.3e-7 / 5.7e-7 us per level^2).
# The CPU/GPU crossover at 100,000 leaves moves from the crate's 512 rays to 32.
B200 = GpuCosts(46.0, 0.0000077, 0.0000007,
                "calibrate_gpu on a B200: sq_raycast_nearest with host buffers, 100,000 box / ball leaves")


def depth(leaves: int) -> float:
    """log2(leaves + 1), at least 1 (dispatch.rs:80-84)."""
    return max(math.log2(leaves + 1), 1.0)


def cpu_batch_us(ctx: QueryContext) -> float:
    d = depth(ctx.scene_leaves)
    return ctx.batch_size * (CPU_TRAVERSAL_US_PER_LEVEL2 + ctx.narrow_cost_hint * CPU_NARROW_US_PER_LEVEL2) * d * d


def gpu_batch_us(ctx: QueryContext, costs: GpuCosts = B200) -> float:
    d = depth(ctx.scene_leaves)
    per_ray = (costs.traversal_us_per_level2 + ctx.narrow_cost_hint * costs.narrow_us_per_level2) * d * d
    return costs.fixed_us + ctx.batch_size * per_ray


def draw_pass_batch_us(ctx: QueryContext) -> float:
    extra = max(ctx.distinct_directions - 1, 0)
    return DRAW_PASS_READBACK_US + extra * DRAW_PASS_US_PER_LEAF * ctx.scene_leaves


class CudaBackend:
    """QueryBackend<3, G> (dispatch.rs:222-240) for an uploaded scene
    (DeviceBvh): kind Gpu, serves a request when a device is available, costs
    `gpu_batch_us` with this library's constants, answers through
    sq_raycast_nearest (the crate's hits, bit for bit)."""

    def __init__(self, scene, costs: GpuCosts = B200):
        self.scene = scene
        self.costs = costs

    def kind(self) -> BackendKind:
        return BackendKind.GPU

    def can_serve(self, ctx: QueryContext) -> bool:
        return ctx.device_available

    def estimate_cost(self, ctx: QueryContext) -> float:
        return gpu_batch_us(ctx, self.costs)

    def raycast_nearest_batch(self, rays, max_toi: float, mask=None, exclude=None):
        return self.scene.raycast_nearest(rays, max_toi, mask=mask, exclude=exclude)


class Dispatcher:
    """Chooses among registered backends per batch (dispatch.rs:276-346): the
    first backend is the mandatory CPU fallback (the consumer's own CPU
    traversal); a forced kind wins over everything, a deterministic request
    pins CPU, otherwise the cheapest backend that can serve the request."""

    def __init__(self, cpu_backend):
        self.backends: List = [cpu_backend]
        self.forced: Optional[BackendKind] = None

    def register(self, backend) -> None:
        self.backends.append(backend)

    def force(self, kind: Optional[BackendKind]) -> None:
        self.forced = kind

    def select(self, ctx: QueryContext) -> BackendKind:
        if self.forced is not None:
            return self.forced
        if ctx.require_deterministic:
            return BackendKind.CPU
        best = None
        for b in self.backends:
            if not b.can_serve(ctx):
                continue
            c = b.estimate_cost(ctx)
            if best is None or c < best[0]:  # min_by keeps the first of equal costs
                best = (c, b)
        return best[1].kind() if best else BackendKind.CPU

    def raycast_nearest_batch(self, rays, max_toi: float, ctx: QueryContext, **kw):
        ctx = replace(ctx, batch_size=len(rays))
        kind = self.select(ctx)
        backend = next(b for b in self.backends if b.kind() == kind)
        return kind, backend.raycast_nearest_batch(rays, max_toi, **kw)


def crossover_batch(leaves: int, costs: GpuCosts = B200, hint: float = 1.0) -> int:
    """The smallest power-of-two scattered batch the model sends to the GPU
    rather than the CPU (the quantity dispatch tests pin)."""
    k = 1
    while True:
        ctx = QueryContext(1 << k, 1 << k, leaves, device_available=True, narrow_cost_hint=hint)
        if gpu_batch_us(ctx, costs) < cpu_batch_us(ctx):
            return 1 << k
        k += 1


def calibrate_gpu(ctx, leaves: int = 100_000, batch: int = 1 << 20, reps: int = 5) -> GpuCosts:
    """Measures this library's GpuCosts on the current device: the fixed cost
    is a one-ray host-buffer call; the per-ray parts come from full batches
    over `leaves` box leaves (traversal: a box leaf's narrow test is its own
    slab) and ball leaves (traversal + one cheap analytic narrow test, hint 1),
    each reduced by depth(leaves)^2 as the crate's model has it."""
    from . import HostBvh, Geometry, DeviceBvh, _Hits, lib, scenes

    rng = scenes.Rng(0xD15_0A7C)
    centres = rng.range(-40.0, 40.0, (leaves, 3)).astype(np.float32)
    org = rng.range(-50.0, 50.0, (batch, 3)).astype(np.float32)
    rays = np.ascontiguousarray(np.concatenate([org, scenes.normalize_rows(-org)], axis=1), dtype=np.float32)
    kinds = {
        "boxes": np.concatenate([centres - 1.0, centres + 1.0], axis=1),
        "balls": np.concatenate([centres, np.ones((leaves, 1), np.float32)], axis=1),
    }
    leaf = np.empty(batch, np.uint32)
    toi = np.empty(batch, np.float32)

    def timed_call(scene, r, n):
        hits = _Hits()
        hits.leaf = leaf.ctypes.data_as(C.c_void_p)
        hits.toi = toi.ctypes.data_as(C.c_void_p)
        fn = lib().sq_raycast_nearest
        args = (ctx.h, scene.h, r.ctypes.data_as(C.c_void_p), n, C.c_float(500.0), None, None, C.byref(hits), None)
        ctx.check(fn(*args), "sq_raycast_nearest")  # warm
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            ctx.check(fn(*args), "sq_raycast_nearest")
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)) * 1e6

    per_ray = {}
    fixed = None
    for name, prims in kinds.items():
        geom = Geometry(name, 3, np.ascontiguousarray(prims, dtype=np.float32))
        scene = DeviceBvh(ctx, HostBvh.build(geom), geom)
        one = timed_call(scene, rays[:1].copy(), 1)
        fixed = one if fixed is None else min(fixed, one)
        per_ray[name] = (timed_call(scene, rays, batch) - one) / batch
        scene.close()
    d2 = depth(leaves) ** 2
    trav = per_ray["boxes"] / d2
    narrow = max(per_ray["balls"] - per_ray["boxes"], 0.0) / d2
    return GpuCosts(fixed, trav, narrow, f"calibrate_gpu: {leaves} leaves, {batch}-ray batches, median of {reps}")
