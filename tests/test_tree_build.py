"""The product's host tree build (sq_tree_build) reproduces the crate's
tree::build (accel/tree.rs:39-163) exactly: same nodes, bounds, children
and primitive order as the oracle, including the degenerate all-coincident
leaf and the stable tie order of equal centroids."""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from spatial_query_b200 import scenes


def same_tree(geom: sq.Geometry, threads=0):
    t = sq.HostBvh.build(geom, threads=threads)
    o = O.Scene(geom.narrow, geom.dim, geom.prims).tree()
    assert t.node_count == len(o["child_a"])
    assert np.array_equal(t.bounds, o["bounds"])
    assert np.array_equal(t.child_a, o["child_a"])
    assert np.array_equal(t.child_b, o["child_b"])
    assert np.array_equal(t.prim_count, o["prim_count"])
    assert np.array_equal(t.prim_indices[: geom.leaf_count], o["prim_indices"])
    return t


@pytest.mark.parametrize("n", [0, 1, 3, 4, 5, 17, 1000])
def test_small_trees(n):
    rng = scenes.Rng(n + 7)
    c = rng.range(-10.0, 10.0, (n, 3))
    r = rng.range(0.1, 1.0, n)
    same_tree(sq.Geometry("balls", 3, np.concatenate([c, r[:, None]], axis=1)))


@pytest.mark.parametrize("dim", [2, 3, 4, 6])
def test_boxes_any_dim(dim):
    s = scenes.boxes_scene(seed=dim, n_boxes=5000, n_rays=1, dim=dim)
    same_tree(sq.Geometry("boxes", dim, s["prims"]))


def test_coincident_centroids_stay_one_leaf():
    # tree.rs:145-148: all centroids equal -> a single leaf of any size.
    prims = np.tile(np.array([[1, 2, 3, 0.5]], np.float32), (37, 1))
    t = same_tree(sq.Geometry("balls", 3, prims))
    assert t.node_count == 1 and t.prim_count[0] == 37


def test_grid_ties_keep_stable_order():
    # A height field puts many equal centroid coordinates on each axis.
    s = scenes.terrain_scene(seed=5, nx=64, ny=32, n_coherent=1, n_incoherent=1)
    for threads in (1, 8):
        same_tree(sq.Geometry("tris", 3, s["prims"]), threads=threads)


def test_full_terrain_tree():
    """1,048,576 triangles: the benchmark tree itself."""
    s = scenes.terrain_scene(seed=1, n_coherent=1, n_incoherent=1)
    t = same_tree(sq.Geometry("tris", 3, s["prims"]))
    assert t.node_count == 524287
