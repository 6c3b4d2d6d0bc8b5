"""A consumer narrow phase compiled at upload time (sq_bvh_upload_custom).

The reference's `gpu` feature takes the consumer's narrow phase as WGSL
source (GpuGeometry, crates/spatial-query/src/gpu/mod.rs:69-99). Here the
consumer's CUDA `sq_narrow` is compiled with NVRTC into the traversal
kernels. The test narrow phase restates the near-root ball test of the
reference's GPU tests (tests/gpu.rs:92-106) in the library's exact maths, so
its answers must equal the oracle's `balls_near` provider bit for bit, in
both traversal orders, for nearest and all-hits queries; a wider leaf
record (stride 7, extra floats ignored) gives the same answers; a source
that does not compile reports SQ_ERR_COMPILE with the compiler's log; the
queries a consumer narrow phase cannot serve report SQ_ERR_UNSUPPORTED.
"""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_lists, assert_same_nearest
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu

BALL_NEAR = """
// The near-root ball test of tests/gpu.rs:92-106: prim = centre[3], radius.
__device__ bool sq_narrow(const float* prim, uint32_t leaf, const float* ro, const float* rd, float max_toi,
                          float* toi, float* normal) {
  float oc[3];
  for (int i = 0; i < 3; ++i) oc[i] = fsub(ro[i], prim[i]);
  const float b = pdot<3>(oc, rd);
  const float c = fsub(pdot<3>(oc, oc), fmul(prim[3], prim[3]));
  const float disc = fsub(fmul(b, b), c);
  if (disc < 0.f) return false;
  const float t = fsub(-b, fsqrt(disc));
  if (t < 0.f || t > max_toi) return false;
  *toi = t;
  float p[3];
  ray_at<3>(ro, rd, t, p);
  for (int i = 0; i < 3; ++i) normal[i] = fsub(p[i], prim[i]);
  normalize_or_zero<3>(normal);
  return true;
}
"""


@pytest.fixture(scope="module")
def ctx():
    c = sq.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def balls():
    rng = scenes.Rng(77)
    n = 6000
    c = rng.range(-50.0, 50.0, (n, 3))
    r = rng.range(0.2, 2.0, (n, 1))
    prims = np.ascontiguousarray(np.concatenate([c, r], axis=1), dtype=np.float32)
    m = 20000
    org = rng.range(-80.0, 80.0, (m, 3))
    d = scenes.normalize_rows(rng.normal64((m, 3)).astype(np.float32))
    rays = np.ascontiguousarray(np.concatenate([org, d], axis=1), dtype=np.float32)
    geom = sq.Geometry("balls_near", 3, prims)
    return prims, geom.world_aabbs(), rays


@pytest.mark.parametrize("order", [sq.ORDER_NEAR_FIRST, sq.ORDER_REFERENCE])
def test_custom_ball_equals_oracle(ctx, balls, order):
    prims, aabbs, rays = balls
    tree = sq.HostBvh.build_from_aabbs(3, aabbs)
    g = sq.DeviceBvh.custom(ctx, tree, prims, aabbs, BALL_NEAR)
    o = O.Scene("balls_near", 3, prims)
    ctx.set_order(order)
    try:
        got = g.raycast_nearest(rays, 120.0, outputs=("normal", "point"))
    finally:
        ctx.set_order(sq.ORDER_NEAR_FIRST)
    ref = o.nearest(rays, 120.0)
    assert (ref.leaf != O.NO_HIT).mean() > 0.2
    assert_same_nearest(ref, got, sub=False, label="custom balls nearest")
    assert_same_lists(o.all(rays, 120.0, k=8), g.raycast_all(rays, 120.0, k=8, outputs=("normal",)),
                      label="custom balls all")
    g.close()


def test_custom_wider_record_same_answers(ctx, balls):
    prims, aabbs, rays = balls
    tree = sq.HostBvh.build_from_aabbs(3, aabbs)
    wide = np.concatenate([prims, np.full((prims.shape[0], 3), 7.5, np.float32)], axis=1)
    g4 = sq.DeviceBvh.custom(ctx, tree, prims, aabbs, BALL_NEAR)
    g7 = sq.DeviceBvh.custom(ctx, tree, wide, aabbs, BALL_NEAR)
    a, b = g4.raycast_nearest(rays, 120.0), g7.raycast_nearest(rays, 120.0)
    assert np.array_equal(a.leaf, b.leaf)
    assert np.array_equal(a.toi.view(np.uint32), b.toi.view(np.uint32))
    g4.close()
    g7.close()


def test_custom_errors(ctx, balls):
    prims, aabbs, rays = balls
    tree = sq.HostBvh.build_from_aabbs(3, aabbs)
    with pytest.raises(sq.SqError) as e:
        sq.DeviceBvh.custom(ctx, tree, prims, aabbs, "__device__ bool sq_narrow( this is not CUDA")
    assert e.value.code == sq.SQ_ERR_COMPILE and "did not compile" in str(e.value)
    g = sq.DeviceBvh.custom(ctx, tree, prims, aabbs, BALL_NEAR)
    casts = np.concatenate([rays[:16], np.full((16, 3), -0.5, np.float32), np.full((16, 3), 0.5, np.float32)],
                           axis=1)
    with pytest.raises(sq.SqError) as e:
        g.shapecast_nearest(casts, 10.0)
    assert e.value.code == sq.SQ_ERR_UNSUPPORTED
    with pytest.raises(sq.SqError) as e:
        g.overlap(np.concatenate([aabbs[:4, :3] - 1, aabbs[:4, 3:] + 1], axis=1))
    assert e.value.code == sq.SQ_ERR_UNSUPPORTED
    g.close()
