"""The host tree build in f64 (sq_tree_build_f64, tree::build with
Scalar = f64) equals the oracle's f64 build: the same nodes, children and
primitive order, and bounds that agree once both are narrowed to f32 (the
oracle exports them so)."""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from spatial_query_b200 import scenes


def same_tree64(geom):
    t = sq.HostBvh.build_f64(geom.dim, geom.world_aabbs_f64())
    o = O.Scene(geom.narrow, geom.dim, geom.prims, prec=64).tree()
    assert t.node_count == len(o["child_a"])
    assert np.array_equal(t.child_a, o["child_a"])
    assert np.array_equal(t.child_b, o["child_b"])
    assert np.array_equal(t.prim_count, o["prim_count"])
    assert np.array_equal(t.prim_indices[: geom.leaf_count], o["prim_indices"])
    assert np.array_equal(t.bounds.astype(np.float32), o["bounds"])
    return t


@pytest.mark.parametrize("dim", [2, 3, 4, 6])
def test_boxes_f64_tree(dim):
    s = scenes.boxes_scene(seed=40 + dim, n_boxes=4000, n_rays=1, dim=dim)
    same_tree64(sq.Geometry("boxes", dim, s["prims"]))


def test_balls_and_triangles_f64_tree():
    rng = scenes.Rng(5)
    c = rng.range(-30.0, 30.0, (3000, 3))
    r = rng.range(0.1, 2.0, (3000, 1))
    same_tree64(sq.Geometry("balls", 3, np.concatenate([c, r], axis=1)))
    s = scenes.terrain_scene(seed=6, nx=64, ny=32, n_coherent=8, n_incoherent=8)
    same_tree64(sq.Geometry("tris", 3, s["prims"]))


def test_f64_tree_differs_from_f32_where_precision_does():
    # descending centroids 1e7 + k/4: distinct in f64 (the sort reverses them),
    # tied in groups in f32 (the stable sort keeps each group's input order)
    n = 64
    c = (1.0e7 + np.arange(n)[::-1] / 4.0).astype(np.float64)
    boxes = np.stack([c, np.zeros(n), np.zeros(n), c + 0.5, np.ones(n), np.ones(n)], axis=1)
    t64 = sq.HostBvh.build_f64(3, boxes)
    t32 = sq.HostBvh.build_from_aabbs(3, boxes.astype(np.float32))
    assert t64.node_count > 1
    assert not (t64.node_count == t32.node_count and np.array_equal(t64.prim_indices, t32.prim_indices))
