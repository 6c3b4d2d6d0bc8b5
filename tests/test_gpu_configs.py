"""CUDA path == CPU oracle on the benchmark workloads at full size.

* boxes: D = 3, 10,000 boxes, 65,536 rays from a radius-200 shell (seed 0).
* terrain: 1,048,576 height-field triangles, 1,048,576 rays (half coherent,
  half incoherent), nearest and all-hits (k = 16), t_max 2000 (seed 1).
* mixture: D = 6, 2,097,152 Gaussian-mixture boxes; rays and overlap
  regions (seed 3).
Also size-independent properties at full size: the first all-hits entry is
the nearest hit, and a query hits iff its list is non-empty."""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_csr, assert_same_lists, assert_same_nearest, ctx, pair
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def boxes():
    s = scenes.boxes_scene(seed=0)
    o, g = pair("boxes", 3, s["prims"])
    return s, o, g


@pytest.fixture(scope="module")
def terrain():
    s = scenes.terrain_scene(seed=1)
    o, g = pair("tris", 3, s["prims"])
    return s, o, g


@pytest.mark.parametrize("order", [sq.ORDER_NEAR_FIRST, sq.ORDER_REFERENCE])
def test_boxes_nearest(boxes, order):
    s, o, g = boxes
    ctx().set_order(order)
    try:
        ref = o.nearest(s["rays"], s["max_toi"], stats=order == sq.ORDER_REFERENCE)
        got = g.raycast_nearest(s["rays"], s["max_toi"], stats=order == sq.ORDER_REFERENCE)
    finally:
        ctx().set_order(sq.ORDER_NEAR_FIRST)
    assert (ref.leaf != O.NO_HIT).mean() > 0.1
    assert_same_nearest(ref, got, label="boxes nearest")
    if order == sq.ORDER_REFERENCE:
        assert list(got.stats.values()) == list(ref.stats.sum(axis=0))


def test_boxes_all_casts_overlaps(boxes):
    s, o, g = boxes
    assert_same_lists(o.all(s["rays"], s["max_toi"], k=16), g.raycast_all(s["rays"], s["max_toi"], k=16))
    rng = scenes.Rng(100)
    n = 8192
    org = rng.range(-150.0, 150.0, (n, 3))
    d = scenes.normalize_rows(rng.normal64((n, 3)).astype(np.float32))
    h = rng.range(0.1, 5.0, (n, 3))
    casts = np.concatenate([org, d, -h, h], axis=1)
    lens = rng.range(0.0, 300.0, n)
    assert_same_nearest(o.shapecast_nearest(casts, lens), g.shapecast_nearest(casts, lens), label="box casts")
    assert_same_lists(o.shapecast_all(casts, lens, k=8), g.shapecast_all(casts, lens, k=8), label="box casts all")
    c = rng.range(-100.0, 100.0, (n, 3))
    e = rng.range(0.5, 10.0, (n, 3))
    regions = np.concatenate([c - e, c + e], axis=1)
    assert_same_csr(o.overlap(regions), g.overlap(regions), label="box overlaps")


@pytest.mark.parametrize("dim", [2, 4])
def test_boxes_other_dims(dim):
    s = scenes.boxes_scene(seed=10 + dim, n_boxes=20000, n_rays=16384, dim=dim)
    o, g = pair("boxes", dim, s["prims"])
    assert_same_nearest(o.nearest(s["rays"], s["max_toi"]), g.raycast_nearest(s["rays"], s["max_toi"]))
    assert_same_lists(o.all(s["rays"], s["max_toi"], k=8), g.raycast_all(s["rays"], s["max_toi"], k=8))


@pytest.mark.parametrize("order", [sq.ORDER_NEAR_FIRST, sq.ORDER_REFERENCE])
def test_terrain_nearest_full(terrain, order):
    s, o, g = terrain
    ctx().set_order(order)
    try:
        got = g.raycast_nearest(s["rays"], s["max_toi"])
    finally:
        ctx().set_order(sq.ORDER_NEAR_FIRST)
    ref = o.nearest(s["rays"], s["max_toi"])
    assert (ref.leaf != O.NO_HIT).mean() > 0.5
    assert_same_nearest(ref, got, label="terrain nearest")


def test_terrain_all_hits_full(terrain):
    s, o, g = terrain
    ref = o.all(s["rays"], s["max_toi"], k=16)
    got = g.raycast_all(s["rays"], s["max_toi"], k=16)
    assert_same_lists(ref, got, label="terrain all-hits")
    # Properties: list head == nearest; hit iff non-empty.
    near = g.raycast_nearest(s["rays"], s["max_toi"])
    has = got.count > 0
    assert np.array_equal(has, near.leaf != sq.NO_HIT)
    assert np.array_equal(got.leaf[has, 0], near.leaf[has])
    assert np.array_equal(got.toi[has, 0].view(np.uint32), near.toi[has].view(np.uint32))


def test_terrain_refit():
    """Lift and tilt the small terrain, refit on the device, compare the tree
    bounds and the queries with the oracle's refit."""
    s = scenes.terrain_scene(seed=5, nx=128, ny=64, n_coherent=4096, n_incoherent=4096)
    o, g = pair("tris", 3, s["prims"])
    moved = s["prims"].copy()
    moved[:, 2::3] += np.float32(3.5) + np.float32(0.01) * moved[:, 0::3]
    o.refit(moved)
    g.refit(moved)
    assert np.array_equal(g.read_bounds(), o.tree()["bounds"])
    assert_same_nearest(o.nearest(s["rays"], s["max_toi"]), g.raycast_nearest(s["rays"], s["max_toi"]))


def test_mixture_d6():
    s = scenes.mixture_scene(seed=3)
    o, g = pair("boxes", 6, s["prims"])
    rays = s["rays"][:262144]
    assert_same_nearest(o.nearest(rays, s["max_toi"]), g.raycast_nearest(rays, s["max_toi"]), label="d6 nearest")
    assert_same_csr(o.overlap(s["regions"]), g.overlap(s["regions"]), label="d6 overlaps")
