"""Host side of the two-level path: instance world AABBs
(Isometry::transform_aabb, maths/isometry.rs:84-97) and the Tlas tree built
over them equal the oracle's Tlas::build (accel/tlas.rs:35-45) bit for bit."""
import numpy as np

import oracle as O
import spatial_query_b200 as sq
from refscenes import random_oriented_boxes
from spatial_query_b200 import scenes


def tlas_tree(kind, dim, rot, trans, param, blas_id=None, oblas=None):
    o = O.TlasScene(kind, dim, rot, trans, param, blas_id=blas_id, blas=oblas)
    return o, o.tree()


def test_box_instances_world_aabbs_and_tree():
    for dim, seed in [(3, 0x7ABC_1234), (2, 0x2020_2020)]:
        rot, trans, halves = random_oriented_boxes(scenes.Rng(seed), 64, dim)
        w = sq.instance_world_aabbs("box", dim, rot, trans, halves)
        _, ot = tlas_tree("box", dim, rot, trans, halves)
        assert np.array_equal(w, ot["world_aabbs"])
        t = sq.HostBvh.build_from_aabbs(dim, w)
        assert np.array_equal(t.bounds, ot["bounds"]) and np.array_equal(t.prim_indices, ot["prim_indices"])
        assert np.array_equal(t.child_a, ot["child_a"]) and np.array_equal(t.prim_count, ot["prim_count"])


def test_ball_instance_world_aabbs():
    rng = scenes.Rng(0x1234_ABCD)
    trans = rng.range(-30.0, 30.0, (48, 3))
    radii = rng.range(0.5, 2.0, 48)
    rot = np.repeat(np.eye(3, dtype=np.float32)[None], 48, 0)
    w = sq.instance_world_aabbs("ball", 3, rot, trans, radii)
    _, ot = tlas_tree("ball", 3, rot, trans, radii)
    assert np.array_equal(w, ot["world_aabbs"])
