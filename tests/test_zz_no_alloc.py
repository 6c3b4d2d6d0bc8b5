"""The allocation-free overlap entry point (sq_overlap_noalloc).

Some callers cannot allocate device memory when they query: an engine that
owns a fixed device-memory budget and forbids driver allocations, a
real-time loop that cannot take an allocation's latency, code that holds no
sq_ctx. sq_overlap_noalloc keeps its scratch in a static device array of the
library instead. This test calls it through the C ABI twice in a row and
checks both results against the ordinary overlap entry point bit for bit,
which in turn equals the oracle's CSR result (overlap sets are integer
results, so the tolerance is exact equality), and
checks that a batch beyond the array's capacity is refused. It creates its
own context and scene, so it passes alone in a fresh process as well as
after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import spatial_query_b200 as sq
from spatial_query_b200 import scenes
from gpu_util import O

pytestmark = pytest.mark.gpu

MAX_REGIONS = 1 << 20


def _noalloc(scene, d_regions, n, d_offsets, d_leaves, capacity, stream, mask=None):
    total = C.c_uint64(0)
    rc = sq.lib().sq_overlap_noalloc(scene.h, d_regions.data_ptr(), n, sq._filter(mask, None), d_offsets.data_ptr(),
                                     d_leaves.data_ptr(), capacity, C.byref(total), stream)
    return rc, int(total.value)


def _check_against_overlap(scene, regions, stream, mask=None, label=""):
    """Two calls in a row, each with poisoned outputs, equal to the ordinary
    entry point's CSR result bit for bit."""
    import torch
    dev = torch.device("cuda", 0)
    want_off, want_leaves = scene.overlap(regions, mask=mask)
    n = regions.shape[0]
    d_regions = torch.from_numpy(np.ascontiguousarray(regions)).to(dev) if n else torch.zeros(1, device=dev)
    cap = int(want_leaves.size) + 16
    for call in range(2):
        d_offsets = torch.full((n + 1,), -1, dtype=torch.int64, device=dev)
        d_leaves = torch.full((cap,), -1, dtype=torch.int32, device=dev)
        rc, total = _noalloc(scene, d_regions, n, d_offsets, d_leaves, cap, stream, mask=mask)
        assert rc == sq.SQ_OK, f"{label} call {call}: status {rc}"
        assert total == want_leaves.size, f"{label} call {call}: total {total} != {want_leaves.size}"
        assert np.array_equal(d_offsets.cpu().numpy().view(np.uint64), want_off), f"{label} call {call}: offsets"
        assert np.array_equal(d_leaves.cpu().numpy().view(np.uint32)[:total], want_leaves), f"{label} call {call}"


def test_overlap_noalloc_matches_overlap_twice():
    import torch
    s = scenes.mixture_scene(seed=11, n_boxes=200_000, n_rays=1, n_regions=50_000)
    ctx = sq.Context(0)
    geom = sq.Geometry("boxes", 6, s["prims"])
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    want_off, want_leaves = scene.overlap(s["regions"])
    assert want_leaves.size > 0
    # The oracle (the crate's CPU walk) gives the same CSR result.
    o_off, o_leaves = O.Scene("boxes", 6, s["prims"]).overlap(s["regions"])
    assert np.array_equal(o_off, want_off) and np.array_equal(o_leaves, want_leaves)

    dev = torch.device("cuda", 0)
    n = s["regions"].shape[0]
    d_regions = torch.from_numpy(s["regions"]).to(dev)
    cap = int(want_leaves.size) + 16
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        # Poison the outputs so a stale result from the first call cannot pass the second.
        d_offsets = torch.full((n + 1,), -1, dtype=torch.int64, device=dev)
        d_leaves = torch.full((cap,), -1, dtype=torch.int32, device=dev)
        rc, total = _noalloc(scene, d_regions, n, d_offsets, d_leaves, cap, stream)
        assert rc == sq.SQ_OK, f"call {call}: status {rc}"
        assert total == want_leaves.size
        got_off = d_offsets.cpu().numpy().view(np.uint64)
        got_leaves = d_leaves.cpu().numpy().view(np.uint32)[:total]
        assert np.array_equal(got_off, want_off), f"call {call}: offsets differ"
        assert np.array_equal(got_leaves, want_leaves), f"call {call}: leaves differ"

    # Too small an output: the needed total is reported, nothing overflows.
    d_offsets = torch.empty(n + 1, dtype=torch.int64, device=dev)
    d_small = torch.empty(4, dtype=torch.int32, device=dev)
    rc, total = _noalloc(scene, d_regions, n, d_offsets, d_small, 4, stream)
    assert rc == sq.SQ_ERR_CAPACITY and total == want_leaves.size

    # More regions than the static scratch holds: refused before any work.
    rc, _ = _noalloc(scene, d_regions, MAX_REGIONS + 1, d_offsets, d_small, 4, stream)
    assert rc == sq.SQ_ERR_CAPACITY
    scene.close()
    ctx.close()


def test_overlap_noalloc_edge_cases():
    """No regions, an empty scene, a layer filter, and scenes of another
    dimension and tree depth after a D = 6 one (the persistent grid is sized
    for each scene's own kernel and stack), each against sq_overlap."""
    import torch
    ctx = sq.Context(0)
    stream = torch.cuda.current_stream(torch.device("cuda", 0)).cuda_stream
    rng = scenes.Rng(23)

    s6 = scenes.mixture_scene(seed=12, n_boxes=30_000, n_rays=1, n_regions=3_000)
    layers = (np.arange(30_000, dtype=np.uint64) % np.uint64(3)) + np.uint64(1)  # layer bits 1, 2, 3
    g6 = sq.Geometry("boxes", 6, s6["prims"], layers=layers)
    scene6 = sq.DeviceBvh(ctx, sq.HostBvh.build(g6), g6)
    _check_against_overlap(scene6, s6["regions"], stream, label="D=6")
    _check_against_overlap(scene6, s6["regions"], stream, mask=0x2, label="D=6 layer mask 0x2")
    _check_against_overlap(scene6, s6["regions"][:0], stream, label="D=6 no regions")

    b = scenes.boxes_scene(seed=4)
    g3 = sq.Geometry("boxes", 3, b["prims"])
    scene3 = sq.DeviceBvh(ctx, sq.HostBvh.build(g3), g3)
    c = rng.range(-100.0, 100.0, (2_000, 3))
    h = rng.range(0.5, 6.0, (2_000, 3))
    regions3 = np.ascontiguousarray(np.concatenate([c - h, c + h], axis=1), dtype=np.float32)
    _check_against_overlap(scene3, regions3, stream, label="D=3 after D=6")

    g0 = sq.Geometry("boxes", 3, np.zeros((0, 6), np.float32))
    scene0 = sq.DeviceBvh(ctx, sq.HostBvh.build(g0), g0)
    _check_against_overlap(scene0, regions3, stream, label="empty scene")
    for sc in (scene0, scene3, scene6):
        sc.close()
    ctx.close()
