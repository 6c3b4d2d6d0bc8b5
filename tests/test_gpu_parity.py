"""CUDA path == CPU oracle, bit for bit, on the spatial-query test-suite's own
scenes (crates/spatial-query/tests/*.rs), through the C ABI.

Each test replays a reference test's scenes and rays, runs them through
libsqcuda.so and compares leaf, toi, normal, point and sub-object bit
patterns with the oracle. Nearest queries run in both traversal orders; in
the reference order the per-batch QueryStats counters match too."""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_csr, assert_same_lists, assert_same_nearest, ctx, pair
from refscenes import (axis_ray, conformance_balls, conformance_rays, differential_cases, line_balls, point,
                       random_balls, ray_new)
from spatial_query_b200.scenes import Rng

pytestmark = pytest.mark.gpu

ORDERS = [sq.ORDER_NEAR_FIRST, sq.ORDER_REFERENCE]


@pytest.fixture(params=ORDERS, ids=["near_first", "reference_order"])
def order(request):
    ctx().set_order(request.param)
    yield request.param
    ctx().set_order(sq.ORDER_NEAR_FIRST)


@pytest.mark.parametrize("dim,seed,n,lo,hi", [(3, 0xABCD_1234, 64, -60.0, 60.0), (2, 0x2222_2222, 48, -60.0, 60.0),
                                              (4, 0x4444_4444, 48, -40.0, 40.0)])
def test_differential_scenes(dim, seed, n, lo, hi, order):
    """tests/differential.rs:120-162 on the GPU: nearest and all hits."""
    for prims, ray in differential_cases(dim, seed, n, lo, hi):
        sub = np.arange(prims.shape[0], dtype=np.uint32)
        o, g = pair("balls", dim, prims, sub=sub)
        assert_same_nearest(o.nearest(ray, 500.0), g.raycast_nearest(ray, 500.0), label="nearest")
        assert_same_lists(o.all(ray, 500.0, k=64), g.raycast_all(ray, 500.0, k=64), label="all")


def test_edge_cases(order):
    """differential.rs:164-211: empty scene, single ball t = 4, miss, clip, ties."""
    ray = axis_ray()
    o, g = pair("balls", 3, np.zeros((0, 4), np.float32))
    assert g.raycast_nearest(ray, 100.0).leaf[0] == sq.NO_HIT
    assert g.raycast_all(ray, 100.0).count[0] == 0
    o, g = pair("balls", 3, np.array([[5, 0, 0, 1]], np.float32))
    h = g.raycast_nearest(ray, 100.0)
    assert h.leaf[0] == 0 and abs(h.toi[0] - 4.0) < 1e-4
    assert g.raycast_nearest(np.array([0, 0, 0, -1, 0, 0], np.float32), 100.0).leaf[0] == sq.NO_HIT
    assert g.raycast_nearest(ray, 3.0).leaf[0] == sq.NO_HIT
    o, g = pair("balls", 3, np.array([[5, 0, 0, 1], [5, 0, 0, 1]], np.float32))
    a = g.raycast_all(ray, 100.0)
    assert a.count[0] == 2 and list(a.leaf[0, :2]) == [0, 1]
    assert g.raycast_nearest(ray, 100.0).leaf[0] == 0
    assert g.raycast_nearest(np.zeros((0, 6), np.float32), 100.0).leaf.size == 0


def test_coincident_leaf_of_many_prims(order):
    """tree.rs:145-148: a leaf of 37 coincident balls (more than LEAF_SIZE)."""
    prims = np.tile(np.array([[10, 0, 0, 1]], np.float32), (37, 1))
    prims[:, 3] = np.linspace(0.5, 2.0, 37, dtype=np.float32)
    o, g = pair("balls", 3, prims)
    rays = np.stack([ray_new(np.zeros(3, np.float32), np.array([1, dy, 0], np.float32))
                     for dy in np.linspace(-0.1, 0.1, 64)])
    assert_same_nearest(o.nearest(rays, 100.0), g.raycast_nearest(rays, 100.0))
    assert_same_lists(o.all(rays, 100.0, k=40), g.raycast_all(rays, 100.0, k=40))


def test_conformance_batches(order):
    """conformance.rs:106-181: batch of 256 / 500 rays, near-root balls."""
    for nb, sb, nr, sr in [(600, 0xC0FF_EE12_3456_789A, 256, 0x0BAD_F00D_DEAD_BEEF),
                           (800, 0x1234_5678_9ABC_DEF0, 500, 0xFACE_B00C_1357_9BDF),
                           (400, 0xAAAA_5555_AAAA_5555, 120, 0x3141_5926_5358_9793)]:
        prims = conformance_balls(nb, sb)
        o, g = pair("balls_near", 3, prims, sub=np.arange(nb, dtype=np.uint32))
        rays = conformance_rays(nr, sr)
        ref = o.nearest(rays, 200.0, threads=1)
        got = g.raycast_nearest(rays, 200.0)
        assert_same_nearest(ref, got)
        # Repeated runs are bitwise identical (conformance.rs:117-122).
        again = g.raycast_nearest(rays, 200.0)
        assert np.array_equal(got.leaf, again.leaf) and np.array_equal(got.toi.view(np.uint32),
                                                                       again.toi.view(np.uint32))


def test_reference_order_replays_cpu_counters():
    """In the reference order the GPU makes the CPU's decisions one for one, so
    the QueryStats counters (accel/stats.rs:41-50) agree exactly."""
    ctx().set_order(sq.ORDER_REFERENCE)
    try:
        prims = conformance_balls(600, 0xC0FF_EE12_3456_789A)
        o, g = pair("balls_near", 3, prims)
        rays = conformance_rays(256, 0x0BAD_F00D_DEAD_BEEF)
        ref = o.nearest(rays, 200.0, stats=True)
        got = g.raycast_nearest(rays, 200.0, stats=True)
        assert_same_nearest(ref, got)
        want = ref.stats.sum(axis=0)
        assert [got.stats[k] for k in ("nodes_visited", "aabb_tests", "narrow_tests", "hits")] == list(want)
    finally:
        ctx().set_order(sq.ORDER_NEAR_FIRST)


def test_counters_known_answers():
    """stats.rs:106-162: all-hits 1/1/3/3, nearest 1/1/3/1, miss 1/1/0/0."""
    o, g = pair("balls_near", 3, line_balls(3, 0.5))
    h = g.raycast_all(axis_ray(), 100.0, stats=True)
    assert h.count[0] == 3 and list(h.stats.values()) == [1, 1, 3, 3]
    ctx().set_order(sq.ORDER_REFERENCE)
    n = g.raycast_nearest(axis_ray(), 100.0, stats=True)
    ctx().set_order(sq.ORDER_NEAR_FIRST)
    assert n.leaf[0] == 0 and list(n.stats.values()) == [1, 1, 3, 1]
    m = g.raycast_all(np.array([0, 0, 0, 0, 0, 1], np.float32), 100.0, stats=True)
    assert m.count[0] == 0 and list(m.stats.values()) == [1, 1, 0, 0]
    o, g = pair("balls_near", 3, line_balls(40, 0.5))
    a = g.raycast_all(axis_ray(), 100.0, k=40, stats=True)
    ref = o.all(axis_ray(), 100.0, k=40, stats=True)
    assert list(a.stats.values()) == list(ref.stats.sum(axis=0))


def _labelled(n):
    return dict(layers=(np.uint64(1) << (np.arange(n, dtype=np.uint64) % np.uint64(2))),
                sub=(np.arange(n, dtype=np.uint32) * 10 + 1))


def test_filter_and_sub_objects(order):
    """result_identity.rs:123-217: layer filter sets and sub-object survival."""
    L = _labelled(12)
    o, g = pair("balls", 3, line_balls(12, 0.6), **L)
    full = g.raycast_all(axis_ray(), 100.0, k=12)
    assert list(full.leaf[0]) == list(range(12))
    even = g.raycast_all(axis_ray(), 100.0, k=12, mask=0b01)
    odd = g.raycast_all(axis_ray(), 100.0, k=12, mask=0b10)
    assert list(even.leaf[0, :even.count[0]]) == [0, 2, 4, 6, 8, 10]
    assert list(odd.leaf[0, :odd.count[0]]) == [1, 3, 5, 7, 9, 11]
    assert all(full.sub_object[0, j] == full.leaf[0, j] * 10 + 1 for j in range(12))
    _, lv = g.overlap(np.array([0, -1, -1, 30, 1, 1], np.float32), mask=0b01)
    assert list(lv) == [0, 2, 4, 6, 8, 10]
    n = g.raycast_nearest(axis_ray(), 100.0, exclude=0)
    assert n.leaf[0] == 1 and n.sub_object[0] == 11
    cast = np.concatenate([axis_ray(), np.full(3, -0.5, np.float32), np.full(3, 0.5, np.float32)])
    c = g.shapecast_nearest(cast, 100.0)
    assert c.sub_object[0] == c.leaf[0] * 10 + 1
    assert_same_nearest(o.shapecast_nearest(cast, 100.0), c)
    assert_same_lists(o.shapecast_all(cast, 100.0, k=12), g.shapecast_all(cast, 100.0, k=12))


PROBE = np.float32(0.75)


def ball_cast(origin, d, r=PROBE):
    dn = ray_new(origin, d)
    return np.concatenate([dn, np.full(3, -r, np.float32), np.full(3, r, np.float32)]).astype(np.float32)


def test_shapecast_scenes(order):
    """shape_overlap.rs:153-231: swept balls, nearest and all, and t = 8.25."""
    rng = Rng(0x5EED_C0DE)
    for _ in range(200):
        prims = random_balls(rng, 64, 3, -30.0, 30.0, 0.5, 2.0)
        cast = ball_cast(point(rng, 3, -50.0, 50.0), point(rng, 3, -1.0, 1.0))
        if not np.any(cast[3:6]):
            continue
        o, g = pair("balls", 3, prims)
        assert_same_nearest(o.shapecast_nearest(cast, 500.0), g.shapecast_nearest(cast, 500.0))
        assert_same_lists(o.shapecast_all(cast, 500.0, k=64), g.shapecast_all(cast, 500.0, k=64))
    o, g = pair("balls", 3, np.array([[10, 0, 0, 1]], np.float32))
    h = g.shapecast_nearest(ball_cast(np.zeros(3, np.float32), np.array([1, 0, 0], np.float32)), 100.0)
    assert h.leaf[0] == 0 and abs(h.toi[0] - 8.25) < 1e-4 and abs(h.normal[0, 0] + 1.0) < 1e-4


def test_overlap_scenes():
    """shape_overlap.rs:237-281: the [0] / [0, 1] sets and random regions."""
    o, g = pair("balls", 3, np.array([[0, 0, 0, 1], [5, 0, 0, 1], [100, 0, 0, 1]], np.float32))
    assert list(g.overlap(np.array([-1.5, -1.5, -1.5, 1.5, 1.5, 1.5], np.float32))[1]) == [0]
    assert list(g.overlap(np.array([-1.5, -1.5, -1.5, 4.0, 1.5, 1.5], np.float32))[1]) == [0, 1]
    rng = Rng(0x0BEE_F00D)
    for _ in range(200):
        prims = random_balls(rng, 96, 3, -30.0, 30.0, 0.5, 2.0)
        c = point(rng, 3, -30.0, 30.0)
        hh = point(rng, 3, 1.0, 6.0)
        region = np.concatenate([c - hh, c + hh])
        o, g = pair("balls", 3, prims)
        assert_same_csr(o.overlap(region), g.overlap(region))


@pytest.mark.parametrize("dim,seed,n", [(3, 0xC0FF_EE11, 64), (2, 0x2D2D_2D2D, 48)])
def test_crossing_scenes(dim, seed, n):
    """crossings.rs:113-173: entry 8 / exit 12, and random shells."""
    o, g = pair("balls", 3, np.array([[10, 0, 0, 2]], np.float32))
    h = g.raycast_crossings(axis_ray(), 100.0)
    assert h.count[0] == 2 and abs(h.toi[0, 0] - 8) < 1e-4 and abs(h.toi[0, 1] - 12) < 1e-4
    assert abs(h.normal[0, 0, 0] + 1) < 1e-4 and abs(h.normal[0, 1, 0] - 1) < 1e-4
    rng = Rng(seed)
    for _ in range(200):
        prims = random_balls(rng, n, dim, -30.0, 30.0, 1.0, 4.0)
        ray = ray_new(point(rng, dim, -40.0, 40.0), point(rng, dim, -1.0, 1.0))
        if not np.any(ray[dim:]):
            continue
        o, g = pair("balls", dim, prims)
        assert_same_lists(o.all(ray, 500.0, k=2 * n, crossings=True), g.raycast_crossings(ray, 500.0, k=2 * n))


def test_gpu_suite_scene(order):
    """tests/gpu.rs:222-240: 1,500 spheres x 2,000 rays -- here bit-exact, not
    within the wgpu path's 1e-3 tolerance."""
    rng = Rng(0xC0FF_EE00_1234_5678)
    raw = rng.take(4 * 1500).reshape(1500, 4)
    from spatial_query_b200.scenes import f32_range
    prims = np.concatenate([f32_range(raw[:, :3], -18.0, 18.0), f32_range(raw[:, 3:], 0.5, 1.6)], axis=1)
    o, g = pair("balls_near", 3, prims)
    rays = conformance_rays(2000, 0x0BAD_F00D_1111_2222, -30.0, 30.0, -6.0, 6.0)
    assert_same_nearest(o.nearest(rays, 200.0), g.raycast_nearest(rays, 200.0))


def test_refit_matches_oracle_refit():
    """two_level.rs:404-432 / gpu.rs:242-263: move the balls, refit on the
    device, and match the oracle's refit tree and its queries."""
    rng = Rng(0x1357_9BDF)
    centers = np.stack([point(rng, 3, -30.0, 30.0) for _ in range(150)])
    prims = np.concatenate([centers, np.ones((150, 1), np.float32)], axis=1)
    o, g = pair("balls_near", 3, prims)
    for _ in range(8):
        centers = centers + np.stack([point(rng, 3, -2.0, 2.0) for _ in range(150)])
        prims = np.concatenate([centers, np.ones((150, 1), np.float32)], axis=1)
        o.refit(prims)
        g.refit(prims)
        assert np.array_equal(g.read_bounds(), o.tree()["bounds"])
        rays = []
        for _ in range(40):
            r = ray_new(point(rng, 3, -40.0, 40.0), point(rng, 3, -1.0, 1.0))
            if np.any(r[3:]):
                rays.append(r)
        rays = np.stack(rays)
        assert_same_nearest(o.nearest(rays, 300.0), g.raycast_nearest(rays, 300.0))


def test_gpuraycaster_api_mirror():
    """GpuRaycaster::headless / raycast_nearest_batch / refit (gpu/mod.rs)."""
    prims = conformance_balls(300, 7)
    geom = sq.Geometry("balls_near", 3, prims)
    bvh = sq.HostBvh.build(geom)
    rc = sq.GpuRaycaster.headless(bvh, geom)
    assert rc is not None
    assert rc.raycast_nearest_batch(np.zeros((0, 6), np.float32), 100.0) == []
    rays = conformance_rays(64, 9)
    hits = rc.raycast_nearest_batch(rays, 200.0)
    o = O.Scene("balls_near", 3, prims).nearest(rays, 200.0)
    for i, h in enumerate(hits):
        if o.leaf[i] == O.NO_HIT:
            assert h is None
        else:
            assert h.leaf == o.leaf[i] and np.float32(h.time_of_impact) == o.toi[i]
    moved = prims.copy()
    moved[:, :3] += np.array([5.0, -3.0, 2.0], np.float32)
    geom2 = sq.Geometry("balls_near", 3, moved)
    rc.refit(bvh, geom2)
    o2 = O.Scene("balls_near", 3, prims)
    o2.refit(moved)
    h2 = rc.scene.raycast_nearest(rays, 200.0)
    assert_same_nearest(o2.nearest(rays, 200.0), h2)


def test_per_query_max_toi(order):
    prims = conformance_balls(500, 11)
    o, g = pair("balls", 3, prims)
    rays = conformance_rays(512, 12)
    mt = Rng(13).range(0.0, 60.0, 512)
    assert_same_nearest(o.nearest(rays, mt), g.raycast_nearest(rays, mt))
    assert_same_lists(o.all(rays, mt, k=8), g.raycast_all(rays, mt, k=8))


def test_uncertified_answers_are_answered_again():
    """Flat triangles in z = const planes: the triangle test's toi can land an
    ulp before the slab entry of the triangle's flat AABB, an answer the
    near-first walk cannot certify. Those rays are answered again in the
    crate's order (by the same lane, in the same launch); every answer is the
    oracle's, for plain and seeded-free host and device calls alike."""
    from spatial_query_b200.scenes import normalize_rows
    rng = Rng(77)
    n, m = 20000, 65536
    z = np.floor(rng.range(0.0, 40.0, n)).astype(np.float32)
    v0 = np.stack([rng.range(-50.0, 50.0, n), rng.range(-50.0, 50.0, n), z], 1)
    v1 = v0 + np.stack([rng.range(0.5, 5.0, n), rng.range(-2.0, 2.0, n), np.zeros(n, np.float32)], 1)
    v2 = v0 + np.stack([rng.range(-2.0, 2.0, n), rng.range(0.5, 5.0, n), np.zeros(n, np.float32)], 1)
    prims = np.ascontiguousarray(np.concatenate([v0, v1, v2], 1), dtype=np.float32)
    o = np.stack([rng.range(-60.0, 60.0, m), rng.range(-60.0, 60.0, m), np.full(m, 80.0, np.float32)], 1)
    d = normalize_rows(np.stack([rng.range(-0.3, 0.3, m), rng.range(-0.3, 0.3, m), -np.ones(m, np.float32)], 1))
    rays = np.ascontiguousarray(np.concatenate([o, d], 1), dtype=np.float32)
    oscene, g = pair("tris", 3, prims)
    ref = oscene.nearest(rays, 500.0)
    assert (ref.leaf != O.NO_HIT).mean() > 0.3
    ctx().set_order(sq.ORDER_NEAR_FIRST)
    got = g.raycast_nearest(rays, 500.0)
    assert ctx().last_replay_count > 0
    assert_same_nearest(ref, got, label="flat triangles, near-first with replays")
    g.close()
