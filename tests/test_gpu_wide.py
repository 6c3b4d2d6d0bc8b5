"""Four-wide node records (SQ_LAYOUT_WIDE, near-first nearest rays), their
quantised copies (SQ_LAYOUT_QUANT: child boxes as 8-bit steps rounded
outward) and the child-pair walk with postponed leaves and the stack's top
entry in registers (SQ_LAYOUT_BINARY_REGTOP) and the child-pair walk with
the warp-vote child order (SQ_LAYOUT_BINARY_VOTE) against the child-pair
records and the oracle: the same
leaf, toi, normal and sub-object bit for bit on boxes in 2, 3, 4 and 6
dimensions, balls, triangles, with per-ray limits and a layer filter, on
trees whose root is a leaf or has leaf children, and after a device refit
(the four-wide boxes are refreshed from the refit binary records)."""
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
    c.set_layout(sq.LAYOUT_BINARY)
    c.close()


@pytest.fixture(params=[sq.LAYOUT_WIDE, sq.LAYOUT_QUANT, sq.LAYOUT_BINARY_REGTOP, sq.LAYOUT_BINARY_VOTE],
                ids=["wide", "quant", "regtop", "vote"])
def layout(request):
    return request.param


def both(ctx, scene, rays, max_toi, layout=sq.LAYOUT_WIDE, **kw):
    out = {}
    for lay in (sq.LAYOUT_BINARY, layout):
        ctx.set_layout(lay)
        out[lay] = scene.raycast_nearest(rays, max_toi, outputs=("normal", "sub"), **kw)
    ctx.set_layout(sq.LAYOUT_BINARY)
    return out[sq.LAYOUT_BINARY], out[layout]


@pytest.mark.parametrize("dim", [2, 3, 4, 6])
def test_boxes(ctx, dim, layout):
    s = scenes.boxes_scene(seed=80 + dim, n_boxes=20000, n_rays=32768, dim=dim)
    geom = sq.Geometry("boxes", dim, s["prims"])
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    binary, wide = both(ctx, scene, s["rays"], s["max_toi"], layout=layout)
    ref = O.Scene("boxes", dim, s["prims"]).nearest(s["rays"], s["max_toi"])
    assert_same_nearest(ref, wide, label=f"wide boxes D={dim}")
    assert_same_nearest(ref, binary, label=f"binary boxes D={dim}")
    scene.close()


def test_triangles_limits_and_filter(ctx, layout):
    s = scenes.terrain_scene(seed=9, nx=256, ny=128, n_coherent=32768, n_incoherent=32768)
    n = s["prims"].shape[0]
    layers = (np.arange(n) % 4 + 1).astype(np.uint64)
    sub = (np.arange(n) * 7).astype(np.uint32)
    geom = sq.Geometry("tris", 3, s["prims"], layers=layers, sub_objects=sub)
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    mt = scenes.Rng(90).range(5.0, 2000.0, s["rays"].shape[0]).astype(np.float32)
    o = O.Scene("tris", 3, s["prims"], layers=layers, sub=sub)
    binary, wide = both(ctx, scene, s["rays"], mt, mask=0b1010, exclude=123, layout=layout)
    ref = o.nearest(s["rays"], mt, mask=0b1010, exclude=123)
    assert (ref.leaf != sq.NO_HIT).mean() > 0.3
    assert_same_nearest(ref, wide, label="wide triangles")
    assert_same_nearest(ref, binary, label="binary triangles")
    scene.close()


@pytest.mark.parametrize("kind", ["balls", "balls_near"])
def test_balls(ctx, kind, layout):
    rng = scenes.Rng(91)
    n = 30000
    prims = np.concatenate([rng.range(-80.0, 80.0, (n, 3)), rng.range(0.2, 2.5, (n, 1))], axis=1).astype(np.float32)
    o = rng.range(-120.0, 120.0, (32768, 3))
    d = scenes.normalize_rows(rng.range(-60.0, 60.0, (32768, 3)) - o)
    rays = np.ascontiguousarray(np.concatenate([o, d], axis=1), dtype=np.float32)
    geom = sq.Geometry(kind, 3, prims)
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    _, wide = both(ctx, scene, rays, 500.0, layout=layout)
    assert_same_nearest(O.Scene(kind, 3, prims).nearest(rays, 500.0), wide, label=f"wide {kind}")
    scene.close()


@pytest.mark.parametrize("n", [1, 3, 5, 6, 9, 40])
def test_small_trees(ctx, n, layout):
    # root a leaf (n <= 4), root with leaf children (5..8), mixed
    s = scenes.boxes_scene(seed=200 + n, n_boxes=n, n_rays=4096)
    geom = sq.Geometry("boxes", 3, s["prims"])
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    binary, wide = both(ctx, scene, s["rays"], s["max_toi"], layout=layout)
    ref = O.Scene("boxes", 3, s["prims"]).nearest(s["rays"], s["max_toi"])
    assert_same_nearest(ref, wide, label=f"wide n={n}")
    scene.close()


def test_refit_refreshes_wide_records(ctx, layout):
    s = scenes.boxes_scene(seed=92, n_boxes=20000, n_rays=32768)
    geom = sq.Geometry("boxes", 3, s["prims"])
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    moved = s["prims"] + scenes.Rng(93).range(-3.0, 3.0, (20000, 1)).astype(np.float32)
    scene.refit(moved)
    o = O.Scene("boxes", 3, s["prims"])
    o.refit(moved)
    binary, wide = both(ctx, scene, s["rays"], s["max_toi"], layout=layout)
    ref = o.nearest(s["rays"], s["max_toi"])
    assert_same_nearest(ref, wide, label="wide after refit")
    assert_same_nearest(ref, binary, label="binary after refit")
    scene.close()
