"""The device tree build (sq_tree_build_d) against the host restatement of
tree::build (sq_tree_build, accel/tree.rs:39-49, 112-163): the same node
arrays and primitive order on the configs' scenes, on small counts around
the leaf size, on ties (the stable sort keeps the parent's order), on
coincident centroids (a leaf of more than four), on -0 / +0 centroids
(total_cmp puts -0 first), and in 2, 4 and 6 dimensions. Bounds compare
equal as numbers (a zero bound may differ in sign: f32::min / max leave it
open). A scene uploaded from the device-built tree answers as the oracle.
"""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_nearest
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sq.Context(0)
    yield c
    c.close()


def assert_same_tree(h, d, label):
    assert h.node_count == d.node_count, f"{label}: node count {h.node_count} vs {d.node_count}"
    assert np.array_equal(h.child_a, d.child_a), f"{label}: child_a"
    assert np.array_equal(h.child_b, d.child_b), f"{label}: child_b"
    assert np.array_equal(h.prim_count, d.prim_count), f"{label}: prim_count"
    assert np.array_equal(h.prim_indices, d.prim_indices), f"{label}: prim_indices"
    assert np.array_equal(h.bounds, d.bounds), f"{label}: bounds"


def check(ctx, dim, aabbs, label):
    h = sq.HostBvh.build_from_aabbs(dim, aabbs)
    d = sq.HostBvh.build_on_device(ctx, dim, aabbs)
    assert_same_tree(h, d, label)
    return h, d


def boxes(rng, n, dim, lo=-100.0, hi=100.0, he=(0.25, 2.0)):
    c = rng.range(lo, hi, (n, dim))
    e = rng.range(he[0], he[1], (n, dim))
    return np.ascontiguousarray(np.concatenate([c - e, c + e], axis=1), dtype=np.float32)


def test_config1_boxes(ctx):
    s = scenes.boxes_scene(seed=0)
    geom = sq.Geometry("boxes", 3, s["prims"])
    h, d = check(ctx, 3, geom.world_aabbs(), "config 1")
    assert h.node_count == 7711  # the crate's tree for 10,000 distinct centroids


def test_terrain_million(ctx):
    s = scenes.terrain_scene(seed=1)
    geom = sq.Geometry("tris", 3, s["prims"])
    h, d = check(ctx, 3, geom.world_aabbs(), "terrain 1M")
    assert h.node_count == 524287


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 9, 17, 33, 1000, 4097])
def test_small_counts(ctx, n):
    check(ctx, 3, boxes(scenes.Rng(100 + n), n, 3), f"n={n}")


def test_ties_keep_parent_order(ctx):
    # centroids on a coarse integer grid: every axis has many equal keys
    rng = scenes.Rng(7)
    n = 5000
    c = np.floor(rng.range(0.0, 6.0, (n, 3))).astype(np.float32)
    e = rng.range(0.1, 0.4, (n, 3)).astype(np.float32)
    check(ctx, 3, np.concatenate([c - e, c + e], axis=1), "ties")


def test_coincident_centroids(ctx):
    rng = scenes.Rng(8)
    same = np.tile(np.array([[1.0, 2.0, 3.0, 2.0, 3.0, 4.0]], np.float32), (50, 1))
    other = boxes(rng, 40, 3)
    a = np.concatenate([same, other, same[:13]], axis=0)
    h, _ = check(ctx, 3, a, "coincident")
    assert (h.prim_count > 4).any()  # the coincident group stays one leaf
    h, _ = check(ctx, 3, same, "all coincident")
    assert h.node_count == 1 and h.prim_count[0] == 50


def test_signed_zero_centroids(ctx):
    # centroids -0 and +0 on the widest axis: total_cmp orders -0 first
    n = 64
    lo = np.zeros((n, 3), np.float32)
    hi = np.zeros((n, 3), np.float32)
    lo[:, 0] = np.where(np.arange(n) % 2 == 0, -0.0, 0.0)
    hi[:, 0] = lo[:, 0]
    lo[:, 1] = np.arange(n, dtype=np.float32) * 0.0  # all zero on y
    lo[:, 2] = (np.arange(n) % 3).astype(np.float32) * 0.1
    hi[:, 2] = lo[:, 2] + 0.1
    a = np.concatenate([lo, hi], axis=1)
    a[::5, 0] = -1.0  # some spread on x
    a[::7, 3] = 2.0
    check(ctx, 3, a, "signed zeros")


@pytest.mark.parametrize("dim", [2, 4, 6])
def test_other_dimensions(ctx, dim):
    check(ctx, dim, boxes(scenes.Rng(20 + dim), 20000, dim), f"D={dim}")


def test_device_tree_answers_as_oracle(ctx):
    s = scenes.boxes_scene(seed=3, n_boxes=6000, n_rays=8192)
    geom = sq.Geometry("boxes", 3, s["prims"])
    d = sq.HostBvh.build_on_device(ctx, 3, geom.world_aabbs())
    scene = sq.DeviceBvh(ctx, d, geom)
    got = scene.raycast_nearest(s["rays"], s["max_toi"])
    ref = O.Scene("boxes", 3, s["prims"]).nearest(s["rays"], s["max_toi"])
    assert_same_nearest(ref, got, label="device-built tree")
    scene.close()
