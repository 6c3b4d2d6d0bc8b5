"""Pins the CPU oracle to the spatial-query crate's own tests.

Every test here restates an assertion of crates/spatial-query/tests/*.rs
against the oracle: the known answers (toi 4, 8, 8.25, 12, overlap sets,
counters, filter sets, sub-objects) and the randomised BVH == naive parity on
the same SplitMix64 seeds. The reference cannot be compiled in this image (no
Rust toolchain), so these are what pin the restatement.
"""
import math

import numpy as np
import pytest

import oracle as O
from refscenes import (TAU32, axis_ray, conformance_balls, conformance_rays, differential_cases, line_balls,
                       plane_rotation, point, random_balls, random_oriented_boxes, ray_new)
from spatial_query_b200.scenes import Rng

NO = O.NO_HIT


def _same_nearest(a: O.Hits, b: O.Hits):
    assert np.array_equal(a.leaf, b.leaf)
    hit = a.leaf != NO
    assert np.array_equal(a.toi[hit].view(np.uint32), b.toi[hit].view(np.uint32))


def _same_lists(a: O.HitLists, b: O.HitLists):
    assert np.array_equal(a.count, b.count)
    assert np.array_equal(a.leaf, b.leaf)
    assert np.array_equal(a.toi.view(np.uint32), b.toi.view(np.uint32))


# -- tests/differential.rs ---------------------------------------------------

@pytest.mark.parametrize("dim,seed,n,lo,hi", [(3, 0xABCD_1234, 64, -60.0, 60.0), (2, 0x2222_2222, 48, -60.0, 60.0),
                                              (4, 0x4444_4444, 48, -40.0, 40.0)])
def test_bvh_matches_naive(dim, seed, n, lo, hi):
    """differential.rs:120-162 (balls, sub-object = leaf, far root inside)."""
    for prims, ray in differential_cases(dim, seed, n, lo, hi):
        sc = O.Scene("balls", dim, prims, sub=np.arange(prims.shape[0], dtype=np.uint32))
        _same_nearest(sc.nearest(ray, 500.0), sc.nearest(ray, 500.0, naive=True))
        _same_lists(sc.all(ray, 500.0, k=64), sc.all(ray, 500.0, k=64, naive=True))


def test_edge_cases():
    """differential.rs:164-194."""
    ray = np.array([0, 0, 0, 1, 0, 0], np.float32)
    empty = O.Scene("balls", 3, np.zeros((0, 4), np.float32))
    assert empty.nearest(ray, 100.0).leaf[0] == NO
    assert empty.all(ray, 100.0).count[0] == 0
    one = O.Scene("balls", 3, np.array([[5, 0, 0, 1]], np.float32))
    h = one.nearest(ray, 100.0)
    assert h.leaf[0] == 0 and abs(h.toi[0] - 4.0) < 1e-4
    away = np.array([0, 0, 0, -1, 0, 0], np.float32)
    assert one.nearest(away, 100.0).leaf[0] == NO
    assert one.nearest(ray, 3.0).leaf[0] == NO


def test_all_hits_sorted_and_ordered_by_leaf_on_ties():
    """differential.rs:196-211: equal toi resolves by leaf."""
    sc = O.Scene("balls", 3, np.array([[5, 0, 0, 1], [5, 0, 0, 1]], np.float32))
    h = sc.all(axis_ray(), 100.0)
    assert h.count[0] == 2 and list(h.leaf[0, :2]) == [0, 1]
    assert h.toi[0, 0] <= h.toi[0, 1]


# -- tests/conformance.rs ----------------------------------------------------

def test_sequential_batch_is_bitwise_repeatable():
    """conformance.rs:106-123 (near-root balls)."""
    sc = O.Scene("balls_near", 3, conformance_balls(600, 0xC0FF_EE12_3456_789A),
                 sub=np.arange(600, dtype=np.uint32))
    rays = conformance_rays(256, 0x0BAD_F00D_DEAD_BEEF)
    ref = sc.nearest(rays, 200.0, threads=1)
    assert np.any(ref.leaf != NO) and np.any(ref.leaf == NO)
    for _ in range(50):
        again = sc.nearest(rays, 200.0, threads=1)
        _same_nearest(ref, again)
        assert np.array_equal(ref.normal.view(np.uint32), again.normal.view(np.uint32))


def test_parallel_batch_matches_sequential_across_thread_counts():
    """conformance.rs:125-145."""
    sc = O.Scene("balls_near", 3, conformance_balls(800, 0x1234_5678_9ABC_DEF0))
    rays = conformance_rays(500, 0xFACE_B00C_1357_9BDF)
    seq = sc.nearest(rays, 200.0, threads=1)
    for t in [1, 2, 3, 4, 7, 8, 16, 999]:
        par = sc.nearest(rays, 200.0, threads=t)
        _same_nearest(seq, par)
        assert np.array_equal(seq.normal, par.normal) and np.array_equal(seq.point, par.point)


def test_parallel_batch_handles_empty_and_single_ray():
    """conformance.rs:147-161."""
    sc = O.Scene("balls_near", 3, conformance_balls(50, 0x0000_0000_DEAD_C0DE))
    assert sc.nearest(np.zeros((0, 6), np.float32), 200.0, threads=8).leaf.size == 0
    rays = conformance_rays(1, 0x5EED_5EED_5EED_5EED)
    _same_nearest(sc.nearest(rays, 200.0, threads=1), sc.nearest(rays, 200.0, threads=8))


def test_parallel_batch_matches_single_ray_nearest():
    """conformance.rs:163-180."""
    sc = O.Scene("balls_near", 3, conformance_balls(400, 0xAAAA_5555_AAAA_5555))
    rays = conformance_rays(120, 0x3141_5926_5358_9793)
    batch = sc.nearest(rays, 200.0, threads=4)
    for i in range(rays.shape[0]):
        one = sc.nearest(rays[i], 200.0, threads=1)
        assert one.leaf[0] == batch.leaf[i]
        if one.leaf[0] != NO:
            assert one.toi[0] == batch.toi[i]


# -- tests/two_level.rs ------------------------------------------------------

def test_isometry_rotation_and_inverse():
    """two_level.rs:180-190."""
    rot = plane_rotation(3, 0, 1, np.float32(math.pi / 2))
    t = np.zeros(3, np.float32)
    r = O.iso_apply(rot, t, 0, np.array([1, 0, 0], np.float32))
    assert abs(r[0]) < 1e-6 and abs(r[1] - 1) < 1e-6 and abs(r[2]) < 1e-6
    back = O.iso_apply(rot, t, 1, r)
    assert abs(back[0] - 1) < 1e-6 and abs(back[1]) < 1e-6


def test_transform_aabb_of_rotated_box():
    """two_level.rs:192-205: extents cos45 + sin45 on x and y, 1 on z."""
    rot = plane_rotation(3, 0, 1, np.float32(math.pi / 4))
    w = O.iso_transform_aabb(rot, np.array([10, 0, 0], np.float32), np.array([-.5, -.5, -.5, .5, .5, .5], np.float32))
    ext = w[3:] - w[:3]
    diag = 2.0 * np.float32(1 / math.sqrt(2))
    assert abs(ext[0] - diag) < 1e-5 and abs(ext[1] - diag) < 1e-5 and abs(ext[2] - 1.0) < 1e-5
    assert abs((w[0] + w[3]) * 0.5 - 10.0) < 1e-5


def test_end_to_end_hit_point_and_normal():
    """two_level.rs:207-224: unit box at x = 5 entered at x = 4, normal -x."""
    sc = O.TlasScene("box", 3, np.eye(3, dtype=np.float32)[None], np.array([[5, 0, 0]], np.float32),
                     np.array([[1, 1, 1]], np.float32))
    h = sc.nearest(axis_ray(), 100.0)
    assert h.leaf[0] == 0 and abs(h.toi[0] - 4.0) < 1e-4
    assert abs(h.point[0, 0] - 4.0) < 1e-4 and abs(h.normal[0, 0] + 1.0) < 1e-4


@pytest.mark.parametrize("dim,seed,n,lo", [(3, 0x7ABC_1234, 64, -60.0), (2, 0x2020_2020, 48, -60.0)])
def test_tlas_matches_naive(dim, seed, n, lo):
    """two_level.rs:263-287 (oriented boxes)."""
    rng = Rng(seed)
    for _ in range(200):
        rot, trans, halves = random_oriented_boxes(rng, n, dim)
        ray = ray_new(point(rng, dim, lo, -lo), point(rng, dim, -1.0, 1.0))
        if not np.any(ray[dim:]):
            continue
        sc = O.TlasScene("box", dim, rot, trans, halves)
        a, b = sc.nearest(ray, 500.0), sc.nearest(ray, 500.0, naive=True)
        _same_nearest(a, b)
        al = sc.all(ray, 500.0, k=n)
        # naive_all (two_level.rs:156-174): every instance hit, sorted.
        hits = []
        for i in range(n):
            one = O.TlasScene("box", dim, rot[i:i + 1], trans[i:i + 1], halves[i:i + 1])
            h = one.nearest(ray, 500.0)
            if h.leaf[0] != NO:
                hits.append((h.toi[0], i))
        hits.sort(key=lambda x: (x[0], x[1]))
        assert al.count[0] == len(hits)
        assert [int(x) for x in al.leaf[0, :len(hits)]] == [i for _, i in hits]


def test_refit_matches_rebuild_when_instances_move():
    """two_level.rs:289-332: move every instance, deform every 7th, refit."""
    rng = Rng(0xF00D_5EED)
    rot, trans, halves = random_oriented_boxes(rng, 200, 3)
    sc = O.TlasScene("box", 3, rot, trans, halves)
    for frame in range(10):
        for i in range(200):
            trans[i] = trans[i] + point(rng, 3, -1.5, 1.5)
            if i % 7 == 0:
                halves[i] = halves[i] * np.float32(1.05)
        sc.refit(trans, param=halves)
        rebuilt = O.TlasScene("box", 3, rot, trans, halves)
        rays = []
        for _ in range(40):
            r = ray_new(point(rng, 3, -60.0, 60.0), point(rng, 3, -1.0, 1.0))
            if np.any(r[3:]):
                rays.append(r)
        rays = np.stack(rays)
        a, b, n = sc.nearest(rays, 500.0), rebuilt.nearest(rays, 500.0), rebuilt.nearest(rays, 500.0, naive=True)
        _same_nearest(a, b)
        _same_nearest(a, n)


def test_needs_rebuild_triggers_after_spreading_instances():
    """two_level.rs:334-362."""
    rng = Rng(0xCAFE_1111)
    n = 128
    trans = np.stack([point(rng, 3, -2.0, 2.0) for _ in range(n)])
    rot = np.repeat(np.eye(3, dtype=np.float32)[None], n, axis=0)
    halves = np.full((n, 3), 0.5, np.float32)
    sc = O.TlasScene("box", 3, rot, trans, halves)
    assert not sc.needs_rebuild(2.0)
    spread = np.stack([point(rng, 3, -500.0, 500.0) for _ in range(n)])
    sc.refit(spread)
    assert sc.needs_rebuild(2.0)


def test_bvh_refit_matches_rebuild():
    """two_level.rs:404-432 (unit balls, near root)."""
    rng = Rng(0x1357_9BDF)
    centers = np.stack([point(rng, 3, -30.0, 30.0) for _ in range(150)])
    prims = np.concatenate([centers, np.ones((150, 1), np.float32)], axis=1)
    sc = O.Scene("balls_near", 3, prims)
    for _ in range(8):
        for i in range(150):
            centers[i] = centers[i] + point(rng, 3, -2.0, 2.0)
        prims = np.concatenate([centers, np.ones((150, 1), np.float32)], axis=1)
        sc.refit(prims)
        rebuilt = O.Scene("balls_near", 3, prims)
        rays = []
        for _ in range(40):
            r = ray_new(point(rng, 3, -40.0, 40.0), point(rng, 3, -1.0, 1.0))
            if np.any(r[3:]):
                rays.append(r)
        _same_nearest(sc.nearest(np.stack(rays), 300.0), rebuilt.nearest(np.stack(rays), 300.0))


# -- tests/shape_overlap.rs --------------------------------------------------

PROBE = np.float32(0.75)


def ball_cast(origin, d, r=PROBE):
    dn = ray_new(origin, d)
    return np.concatenate([dn, np.full(3, -r, np.float32), np.full(3, r, np.float32)]).astype(np.float32)


def test_bvh_shapecast_matches_naive():
    """shape_overlap.rs:153-181."""
    rng = Rng(0x5EED_C0DE)
    for _ in range(200):
        prims = random_balls(rng, 64, 3, -30.0, 30.0, 0.5, 2.0)
        cast = ball_cast(point(rng, 3, -50.0, 50.0), point(rng, 3, -1.0, 1.0))
        if not np.any(cast[3:6]):
            continue
        sc = O.Scene("balls", 3, prims)
        _same_nearest(sc.shapecast_nearest(cast, 500.0), sc.shapecast_nearest(cast, 500.0, naive=True))
        _same_lists(sc.shapecast_all(cast, 500.0, k=64), sc.shapecast_all(cast, 500.0, k=64, naive=True))


def test_swept_ball_stops_at_nearest_surface():
    """shape_overlap.rs:183-231: toi 8.25, normal -x, fine-step march agrees."""
    sc = O.Scene("balls", 3, np.array([[10, 0, 0, 1]], np.float32))
    cast = ball_cast(np.zeros(3, np.float32), np.array([1, 0, 0], np.float32))
    h = sc.shapecast_nearest(cast, 100.0)
    assert h.leaf[0] == 0 and abs(h.toi[0] - 8.25) < 1e-4 and abs(h.normal[0, 0] + 1.0) < 1e-4
    t, step = 0.0, 0.001
    while abs(t - 10.0) > 1.75:
        t += step
    assert abs(h.toi[0] - t) < 2 * step


def test_overlap_returns_exactly_intersecting_balls():
    """shape_overlap.rs:237-262: sets [0] and [0, 1]."""
    sc = O.Scene("balls", 3, np.array([[0, 0, 0, 1], [5, 0, 0, 1], [100, 0, 0, 1]], np.float32))
    off, lv = sc.overlap(np.array([-1.5, -1.5, -1.5, 1.5, 1.5, 1.5], np.float32))
    assert list(lv) == [0]
    off, lv = sc.overlap(np.array([-1.5, -1.5, -1.5, 4.0, 1.5, 1.5], np.float32))
    assert list(lv) == [0, 1]


def test_bvh_overlap_matches_naive():
    """shape_overlap.rs:264-281."""
    rng = Rng(0x0BEE_F00D)
    for _ in range(200):
        prims = random_balls(rng, 96, 3, -30.0, 30.0, 0.5, 2.0)
        c = point(rng, 3, -30.0, 30.0)
        hh = point(rng, 3, 1.0, 6.0)
        region = np.concatenate([c - hh, c + hh])
        sc = O.Scene("balls", 3, prims)
        a = sc.overlap(region)
        b = sc.overlap(region, naive=True)
        assert list(a[1]) == list(b[1])


def _ball_instances(rng, n):
    trans = np.stack([point(rng, 3, -30.0, 30.0) for _ in range(n)])
    radii = rng.range(0.5, 2.0, n)
    return trans, radii


def test_tlas_shapecast_matches_naive_via_ball_bvh():
    """shape_overlap.rs:344-381."""
    rng = Rng(0x1234_ABCD)
    for _ in range(150):
        trans, radii = _ball_instances(rng, 48)
        inst = O.TlasScene("ball", 3, np.repeat(np.eye(3, dtype=np.float32)[None], 48, 0), trans, radii)
        balls = O.Scene("balls", 3, np.concatenate([trans, radii[:, None]], axis=1))
        cast = ball_cast(point(rng, 3, -50.0, 50.0), point(rng, 3, -1.0, 1.0))
        if not np.any(cast[3:6]):
            continue
        _same_nearest(balls.shapecast_nearest(cast, 500.0, naive=True), inst.shapecast_nearest(cast, 500.0))
        _same_lists(balls.shapecast_all(cast, 500.0, k=48, naive=True), inst.shapecast_all(cast, 500.0, k=48))


def test_tlas_overlap_matches_naive_via_ball_bvh():
    """shape_overlap.rs:383-411."""
    rng = Rng(0x9999_5555)
    for _ in range(150):
        trans, radii = _ball_instances(rng, 64)
        inst = O.TlasScene("ball", 3, np.repeat(np.eye(3, dtype=np.float32)[None], 64, 0), trans, radii)
        balls = O.Scene("balls", 3, np.concatenate([trans, radii[:, None]], axis=1))
        c = point(rng, 3, -30.0, 30.0)
        hh = point(rng, 3, 1.0, 6.0)
        region = np.concatenate([c - hh, c + hh])
        assert list(balls.overlap(region, naive=True)[1]) == list(inst.overlap(region)[1])


# -- tests/crossings.rs ------------------------------------------------------

def test_crossings_report_entry_and_exit():
    """crossings.rs:113-135: toi 8 (normal -x) and 12 (normal +x)."""
    sc = O.Scene("balls", 3, np.array([[10, 0, 0, 2]], np.float32))
    h = sc.all(axis_ray(), 100.0, crossings=True)
    assert h.count[0] == 2
    assert abs(h.toi[0, 0] - 8.0) < 1e-4 and abs(h.normal[0, 0, 0] + 1.0) < 1e-4
    assert abs(h.toi[0, 1] - 12.0) < 1e-4 and abs(h.normal[0, 1, 0] - 1.0) < 1e-4


@pytest.mark.parametrize("dim,seed,n", [(3, 0xC0FF_EE11, 64), (2, 0x2D2D_2D2D, 48)])
def test_crossings_match_naive(dim, seed, n):
    """crossings.rs:149-173."""
    rng = Rng(seed)
    for _ in range(200):
        prims = random_balls(rng, n, dim, -30.0, 30.0, 1.0, 4.0)
        ray = ray_new(point(rng, dim, -40.0, 40.0), point(rng, dim, -1.0, 1.0))
        if not np.any(ray[dim:]):
            continue
        sc = O.Scene("balls", dim, prims)
        _same_lists(sc.all(ray, 500.0, k=2 * n, crossings=True), sc.all(ray, 500.0, k=2 * n, crossings=True, naive=True))


def test_default_crossings_reproduce_all_hits():
    """crossings.rs:210-232: a single-hit provider's crossings == all hits."""
    rng = Rng(0x5011_D000)
    prims = random_balls(rng, 80, 3, -25.0, 25.0, 1.0, 3.0)
    sc = O.Scene("balls_near", 3, prims)  # no crossings override
    for _ in range(100):
        ray = ray_new(point(rng, 3, -35.0, 35.0), point(rng, 3, -1.0, 1.0))
        if not np.any(ray[3:]):
            continue
        _same_lists(sc.all(ray, 500.0, k=80), sc.all(ray, 500.0, k=80, crossings=True))


def test_tlas_crossings_match_single_level_oracle():
    """crossings.rs:286-320."""
    rng = Rng(0x7717_9999)
    for _ in range(150):
        centers = np.stack([point(rng, 3, -30.0, 30.0) for _ in range(48)])
        radii = rng.range(1.0, 4.0, 48)
        inst = O.TlasScene("ball", 3, np.repeat(np.eye(3, dtype=np.float32)[None], 48, 0), centers, radii)
        shells = O.Scene("balls", 3, np.concatenate([centers, radii[:, None]], axis=1))
        ray = ray_new(point(rng, 3, -40.0, 40.0), point(rng, 3, -1.0, 1.0))
        if not np.any(ray[3:]):
            continue
        _same_lists(shells.all(ray, 500.0, k=96, crossings=True, naive=True),
                    inst.all(ray, 500.0, k=96, crossings=True))


# -- tests/stats.rs ----------------------------------------------------------

def test_structural_stats():
    """stats.rs:62-100."""
    s = O.Scene("balls_near", 3, line_balls(3, 0.5)).stats()
    assert (s["node_count"], s["leaf_count"], s["prim_count"], s["max_depth"]) == (1, 1, 3, 1)
    s = O.Scene("balls_near", 3, line_balls(50, 0.5)).stats()
    assert s["prim_count"] == 50 and 1 <= s["leaf_count"] < s["node_count"]
    assert 1 <= s["max_depth"] <= s["node_count"] and math.isfinite(s["quality"]) and s["quality"] >= 0
    s = O.Scene("balls_near", 3, np.zeros((0, 4), np.float32)).stats()
    assert (s["node_count"], s["leaf_count"], s["prim_count"], s["max_depth"]) == (0, 0, 0, 0)


def test_counters_are_exact():
    """stats.rs:106-162: all-hits 1/1/3/3, nearest 1/1/3/1, miss 1/1/0/0."""
    sc = O.Scene("balls_near", 3, line_balls(3, 0.5))
    h = sc.all(axis_ray(), 100.0, stats=True)
    assert h.count[0] == 3 and list(h.stats[0]) == [1, 1, 3, 3]
    n = sc.nearest(axis_ray(), 100.0, stats=True)
    assert n.leaf[0] == 0 and list(n.stats[0]) == [1, 1, 3, 1]
    m = sc.all(np.array([0, 0, 0, 0, 0, 1], np.float32), 100.0, stats=True)
    assert m.count[0] == 0 and list(m.stats[0]) == [1, 1, 0, 0]


def test_stats_path_matches_plain_path_and_repeats():
    """stats.rs:164-185."""
    sc = O.Scene("balls_near", 3, line_balls(40, 0.5))
    a = sc.all(axis_ray(), 100.0, k=40, stats=True)
    b = sc.all(axis_ray(), 100.0, k=40, stats=True)
    _same_lists(a, sc.all(axis_ray(), 100.0, k=40))
    assert np.array_equal(a.stats, b.stats)
    assert a.stats[0, 0] > 1 and a.stats[0, 0] <= a.stats[0, 2] + sc.stats()["node_count"]


# -- tests/result_identity.rs ------------------------------------------------

def _labelled(n):
    return dict(layers=(np.uint64(1) << (np.arange(n, dtype=np.uint64) % np.uint64(2))),
                sub=(np.arange(n, dtype=np.uint32) * 10 + 1))


def test_filter_selects_exactly_the_accepted_complement():
    """result_identity.rs:123-163."""
    sc = O.Scene("balls", 3, line_balls(12, 0.6), **_labelled(12))
    full = list(sc.all(axis_ray(), 100.0, k=12).leaf[0])
    even = sc.all(axis_ray(), 100.0, k=12, mask=0b01)
    odd = sc.all(axis_ray(), 100.0, k=12, mask=0b10)
    assert full == list(range(12))
    assert list(even.leaf[0, :even.count[0]]) == [0, 2, 4, 6, 8, 10]
    assert list(odd.leaf[0, :odd.count[0]]) == [1, 3, 5, 7, 9, 11]
    nv = sc.all(axis_ray(), 100.0, k=12, mask=0b01, naive=True)
    assert list(nv.leaf[0, :nv.count[0]]) == [0, 2, 4, 6, 8, 10]


def test_filter_applies_to_overlap_too():
    """result_identity.rs:165-180."""
    sc = O.Scene("balls", 3, line_balls(12, 0.6), **_labelled(12))
    _, lv = sc.overlap(np.array([0, -1, -1, 30, 1, 1], np.float32), mask=0b01)
    assert list(lv) == [0, 2, 4, 6, 8, 10]


def test_sub_object_survives_bvh_ray_and_shapecast():
    """result_identity.rs:186-217 (probe radius 0.5)."""
    sc = O.Scene("balls", 3, line_balls(8, 0.6), **_labelled(8))
    n = sc.nearest(axis_ray(), 100.0)
    assert n.sub[0] == n.leaf[0] * 10 + 1
    a = sc.all(axis_ray(), 100.0, k=8)
    assert all(a.sub[0, j] == a.leaf[0, j] * 10 + 1 for j in range(a.count[0]))
    cast = ball_cast(np.zeros(3, np.float32), np.array([1, 0, 0], np.float32), np.float32(0.5))
    c = sc.shapecast_nearest(cast, 100.0)
    assert c.leaf[0] != NO and c.sub[0] == c.leaf[0] * 10 + 1
    ca = sc.shapecast_all(cast, 100.0, k=8)
    assert all(ca.sub[0, j] == ca.leaf[0, j] * 10 + 1 for j in range(ca.count[0]))
    nv = sc.nearest(axis_ray(), 100.0, naive=True)
    assert nv.sub[0] == nv.leaf[0] * 10 + 1


def test_sub_object_survives_tlas_ray():
    """result_identity.rs:251-270."""
    trans = np.zeros((6, 3), np.float32)
    trans[:, 0] = 2.0 * (np.arange(6, dtype=np.float32) + 1)
    inst = O.TlasScene("ball", 3, np.repeat(np.eye(3, dtype=np.float32)[None], 6, 0), trans,
                       np.full(6, 0.6, np.float32), sub=np.arange(6, dtype=np.uint32) * 10 + 1)
    n = inst.nearest(axis_ray(), 100.0)
    assert n.sub[0] == n.leaf[0] * 10 + 1
    a = inst.all(axis_ray(), 100.0, k=6)
    assert all(a.sub[0, j] == a.leaf[0, j] * 10 + 1 for j in range(a.count[0]))


# -- the GPU test suite's CPU half (tests/gpu.rs:222-275 scenes) -------------

def test_gpu_suite_scenes_hit_and_miss():
    """gpu.rs:222-240: the 1,500-sphere / 2,000-ray batch really hits and misses."""
    rng = Rng(0xC0FF_EE00_1234_5678)
    raw = rng.take(4 * 1500).reshape(1500, 4)
    from spatial_query_b200.scenes import f32_range
    prims = np.concatenate([f32_range(raw[:, :3], -18.0, 18.0), f32_range(raw[:, 3:], 0.5, 1.6)], axis=1)
    sc = O.Scene("balls_near", 3, prims)
    rays = conformance_rays(2000, 0x0BAD_F00D_1111_2222, -30.0, 30.0, -6.0, 6.0)
    h = sc.nearest(rays, 200.0)
    assert np.any(h.leaf != NO) and np.any(h.leaf == NO)


# -- crates/viewport-lib-query/src/lib.rs (mesh instances, ray_triangle) -------

def _cube_tlas(trans, scale=None):
    from refscenes import cube_mesh, mesh_instances
    cube = cube_mesh(2.0)
    rot, t, s, bid = mesh_instances(trans, scale)
    blas = O.BlasSet(np.array([0, cube.shape[0]], np.uint64), cube)
    return O.TlasScene("mesh", 3, rot, t, s, blas_id=bid, blas=blas), blas


def test_ray_hits_registered_cube_with_face_and_id():
    """lib.rs:338-366: a cube of edge 2 at x = 5; a +x ray from the origin hits
    its near face at toi 4 (within 1e-3) with a normal along x and a face
    sub-object; the instance is the one registered (pick id 42)."""
    pick_ids = np.array([42], np.uint32)
    sc, _ = _cube_tlas([[5.0, 0.0, 0.0]])
    h = sc.nearest(ray_new(np.zeros(3, np.float32), np.array([1, 0, 0], np.float32))[None], 100.0)
    assert h.leaf[0] != NO and pick_ids[h.leaf[0]] == 42
    assert abs(float(h.toi[0]) - (5.0 + -1.0)) < 1e-3
    assert abs(float(h.normal[0, 0])) > 0.9
    assert h.sub[0] != NO and h.sub[0] < 12  # a face of the 12-triangle cube


def test_nearest_instance_wins():
    """lib.rs:368-380: cubes at x = 10 (pick 100) and x = 5 (pick 200): 200."""
    pick_ids = np.array([100, 200], np.uint32)
    sc, _ = _cube_tlas([[10.0, 0.0, 0.0], [5.0, 0.0, 0.0]])
    h = sc.nearest(ray_new(np.zeros(3, np.float32), np.array([1, 0, 0], np.float32))[None], 100.0)
    assert h.leaf[0] != NO and pick_ids[h.leaf[0]] == 200


def test_ray_pointing_away_misses():
    """lib.rs:382-392: a -x ray from the origin misses the cube at x = 5."""
    sc, _ = _cube_tlas([[5.0, 0.0, 0.0]])
    h = sc.nearest(ray_new(np.zeros(3, np.float32), np.array([-1, 0, 0], np.float32))[None], 100.0)
    assert h.leaf[0] == NO


def test_scaled_instance_reports_world_distance():
    """lib.rs:394-430: the cube scaled 3x at x = 20: world toi 20 + 3 * -1 = 17
    (within 1e-2), not the local-space distance."""
    sc, _ = _cube_tlas([[20.0, 0.0, 0.0]], scale=[3.0])
    h = sc.nearest(ray_new(np.zeros(3, np.float32), np.array([1, 0, 0], np.float32))[None], 100.0)
    assert h.leaf[0] == 0
    assert abs(float(h.toi[0]) - 17.0) < 1e-2
