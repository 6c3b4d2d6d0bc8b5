"""L2-persisting node records (sq_ctx_set_l2_persist): with a scene's node
records marked persisting for the context's stream, nearest rays in both
orders still return the oracle's answers bit for bit (leaf, toi, normal),
also through the chunked host-buffer call that uses the context's second
lane; clearing the window (and giving a bad scene handle) behaves."""
import numpy as np
import pytest

import spatial_query_b200 as sq
from gpu_util import O, assert_same_nearest
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu


def test_persisting_node_records_keep_answers():
    s = scenes.terrain_scene(seed=12, nx=256, ny=128, n_coherent=32768, n_incoherent=32768)
    geom = sq.Geometry("tris", 3, s["prims"])
    tree = sq.HostBvh.build(geom)
    ctx = sq.Context(0)
    scene = sq.DeviceBvh(ctx, tree, geom)
    ref = O.Scene("tris", 3, s["prims"]).nearest(s["rays"], s["max_toi"])
    ctx.set_l2_persist(scene, 8 << 20)
    for order in (sq.ORDER_NEAR_FIRST, sq.ORDER_REFERENCE):
        ctx.set_order(order)
        got = scene.raycast_nearest(s["rays"], s["max_toi"], outputs=("normal",))
        assert_same_nearest(ref, got, label=f"persisting, order {order}")
    ctx.set_order(sq.ORDER_NEAR_FIRST)
    # 2^20 rays: the chunked host-buffer path, on the context and its second lane
    big = np.ascontiguousarray(np.concatenate([s["rays"]] * 16))
    got = scene.raycast_nearest(big, s["max_toi"], outputs=("normal",))
    ref_big = O.Scene("tris", 3, s["prims"]).nearest(big[:65536], s["max_toi"])
    assert np.array_equal(got.leaf[:65536], ref_big.leaf)
    assert np.array_equal(np.asarray(got.toi[:65536]).view(np.uint32), np.asarray(ref_big.toi).view(np.uint32))
    assert np.array_equal(got.leaf[65536:131072], got.leaf[:65536])
    ctx.set_l2_persist()
    got = scene.raycast_nearest(s["rays"], s["max_toi"], outputs=("normal",))
    assert_same_nearest(ref, got, label="cleared")
    scene.close()
    ctx.close()


def test_l2_persist_rejects_bad_arguments():
    assert sq.lib().sq_ctx_set_l2_persist(None, None, 0) == sq.SQ_ERR_INVALID
