"""Host-buffer calls large enough to run in chunks (rays copied in on one
stream while earlier chunks are walked, alternately on the context's stream
and on its second lane, and their hits copied out on another) return exactly
what the device-pointer calls and the oracle return: plain nearest with every
output and per-ray limits, in both traversal orders and both node layouts
(the second lane takes the context's settings), and the learned-seeded
call."""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_nearest
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def setup():
    s = scenes.terrain_scene(seed=11, nx=512, ny=256)  # 262,144 triangles, 262,144 rays
    rays = np.ascontiguousarray(np.concatenate([s["rays"]] * 4))  # 1,048,576 rays: four chunks
    ctx = sq.Context(0)
    geom = sq.Geometry("tris", 3, s["prims"], sub_objects=np.arange(s["prims"].shape[0], dtype=np.uint32) * 3)
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    yield s, rays, ctx, geom, scene
    scene.close()
    ctx.close()


def test_chunked_plain_equals_oracle(setup):
    s, rays, ctx, geom, scene = setup
    mt = scenes.Rng(12).range(5.0, s["max_toi"], rays.shape[0]).astype(np.float32)
    got = scene.raycast_nearest(rays, mt, outputs=("normal", "point", "sub"))
    o = O.Scene("tris", 3, s["prims"], sub=geom.sub_objects)
    ref = o.nearest(rays, mt)
    assert (ref.leaf != O.NO_HIT).mean() > 0.3
    assert_same_nearest(ref, got, label="chunked host call")


@pytest.mark.parametrize("order,layout", [(sq.ORDER_REFERENCE, sq.LAYOUT_BINARY), (sq.ORDER_NEAR_FIRST, sq.LAYOUT_WIDE)])
def test_chunked_settings_reach_both_lanes(setup, order, layout):
    s, rays, ctx, geom, scene = setup
    ctx.set_order(order)
    ctx.set_layout(layout)
    try:
        launches0 = ctx.launch_count
        got = scene.raycast_nearest(rays, s["max_toi"], outputs=("normal",))
        assert ctx.launch_count - launches0 >= 4  # every chunk's launches are counted, both lanes'
    finally:
        ctx.set_order(sq.ORDER_NEAR_FIRST)
        ctx.set_layout(sq.LAYOUT_BINARY)
    ref = O.Scene("tris", 3, s["prims"]).nearest(rays, s["max_toi"])
    assert_same_nearest(ref, got, label=f"chunked host call, order {order}, layout {layout}")


def test_chunked_guided_equals_device_call(setup):
    import torch
    s, rays, ctx, geom, scene = setup
    guide = sq.Guide(scene, depth=10, batch=256, seed=4)
    host = guide.raycast_nearest_guided(rays, s["max_toi"])
    n = rays.shape[0]
    d_rays = torch.from_numpy(rays).to(DEV)
    leaf = torch.empty(n, dtype=torch.int32, device=DEV)
    toi = torch.empty(n, dtype=torch.float32, device=DEV)
    nrm = torch.empty((n, 3), dtype=torch.float32, device=DEV)
    torch.cuda.synchronize()
    guide.raycast_nearest_guided_d(d_rays, n, s["max_toi"], leaf, toi, nrm)
    ctx.synchronize()
    assert np.array_equal(host.leaf, leaf.cpu().numpy().view(np.uint32))
    assert np.array_equal(host.toi.view(np.uint32), toi.cpu().numpy().view(np.uint32))
    assert np.array_equal(host.normal.view(np.uint32), nrm.cpu().numpy().view(np.uint32))
    ref = O.Scene("tris", 3, s["prims"]).nearest(rays, s["max_toi"])
    assert np.array_equal(ref.leaf, host.leaf)
    guide.close()
