"""Nearest rays with the crate's f64 feature on the device
(sq_raycast_nearest_f64) against the oracle's f64 build: the same leaf,
the same f64 time of impact bit for bit, the same normal (compared after
narrowing to f32, as the oracle reports it) and the same QueryStats
counters, for boxes in 2, 3, 4 and 6 dimensions, balls (both roots and
near root only) and triangles; with a per-ray limit and a layer filter; and
on large coordinates where the f32 path's answers move but the f64 path
still matches the f64 CPU build. Inputs are f32 values widened to f64 on
both sides."""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sq.Context(0)
    yield c
    c.close()


def run(ctx, geom, rays, max_toi, mask=None, exclude=None):
    tree = sq.HostBvh.build_f64(geom.dim, geom.world_aabbs_f64())
    scene = sq.DeviceBvh64(ctx, tree, geom)
    got = scene.raycast_nearest(rays.astype(np.float64), max_toi if np.ndim(max_toi) == 0 else
                                np.asarray(max_toi, np.float64), mask=mask, exclude=exclude, stats=True)
    o = O.Scene(geom.narrow, geom.dim, geom.prims, layers=geom.layers, prec=64)
    kw = {}
    if mask is not None:
        kw["mask"] = mask
    if exclude is not None:
        kw["exclude"] = exclude
    ref = o.nearest(rays, max_toi, stats=True, **kw)
    scene.close()
    return ref, got


def same(ref, got, label):
    assert np.array_equal(ref.leaf, got.leaf), f"{label}: leaf differs on {(ref.leaf != got.leaf).sum()} rays"
    assert np.array_equal(ref.toi.view(np.uint64), got.toi.view(np.uint64)), f"{label}: f64 toi"
    assert np.array_equal(ref.normal.view(np.uint32), got.normal.astype(np.float32).view(np.uint32)), f"{label}: normal"
    s = ref.stats.sum(axis=0)
    assert [int(x) for x in s] == [got.stats["nodes_visited"], got.stats["aabb_tests"], got.stats["narrow_tests"],
                                   got.stats["hits"]], f"{label}: counters"


@pytest.mark.parametrize("dim", [2, 3, 4, 6])
def test_boxes(ctx, dim):
    s = scenes.boxes_scene(seed=60 + dim, n_boxes=10000, n_rays=16384, dim=dim)
    prims = s["prims"]
    if dim >= 4:  # widen the boxes so that rays in 4 and 6 dimensions still hit some
        c, h = (prims[:, :dim] + prims[:, dim:]) / 2, (prims[:, dim:] - prims[:, :dim]) / 2
        prims = np.ascontiguousarray(np.concatenate([c - 6 * h, c + 6 * h], axis=1), dtype=np.float32)
    ref, got = run(ctx, sq.Geometry("boxes", dim, prims), s["rays"], s["max_toi"])
    assert (ref.leaf != sq.NO_HIT).sum() > 200  # sparse in 4 and 6 dimensions
    same(ref, got, f"boxes D={dim}")


@pytest.mark.parametrize("kind", ["balls", "balls_near"])
def test_balls(ctx, kind):
    rng = scenes.Rng(61)
    n = 8000
    prims = np.concatenate([rng.range(-60.0, 60.0, (n, 3)), rng.range(0.3, 3.0, (n, 1))], axis=1).astype(np.float32)
    o = rng.range(-100.0, 100.0, (16384, 3))
    d = scenes.normalize_rows(rng.range(-50.0, 50.0, (16384, 3)) - o)
    rays = np.ascontiguousarray(np.concatenate([o, d], axis=1), dtype=np.float32)
    ref, got = run(ctx, sq.Geometry(kind, 3, prims), rays, 400.0)
    assert (ref.leaf != sq.NO_HIT).mean() > 0.2
    same(ref, got, kind)


def test_triangles_per_ray_limit(ctx):
    s = scenes.terrain_scene(seed=7, nx=128, ny=64, n_coherent=8192, n_incoherent=8192)
    rng = scenes.Rng(62)
    mt = rng.range(10.0, 2000.0, s["rays"].shape[0]).astype(np.float32)
    ref, got = run(ctx, sq.Geometry("tris", 3, s["prims"]), s["rays"], mt)
    assert (ref.leaf != sq.NO_HIT).mean() > 0.3
    same(ref, got, "triangles")


def test_layer_filter(ctx):
    s = scenes.boxes_scene(seed=63, n_boxes=5000, n_rays=8192)
    layers = (np.arange(5000) % 3 + 1).astype(np.uint64)  # 1, 2, 3
    geom = sq.Geometry("boxes", 3, s["prims"], layers=layers)
    ref, got = run(ctx, geom, s["rays"], s["max_toi"], mask=0b10, exclude=17)
    same(ref, got, "filter")


def test_large_coordinates(ctx):
    # boxes near 1e6: the f32 path's tois move by its rounding, the f64 path's match the f64 CPU build
    s = scenes.boxes_scene(seed=64, n_boxes=5000, n_rays=8192)
    off = np.float32(1.0e6)
    prims = s["prims"] + off
    rays = s["rays"].copy()
    rays[:, :3] += off
    geom = sq.Geometry("boxes", 3, prims)
    ref, got = run(ctx, geom, rays, s["max_toi"])
    same(ref, got, "large coordinates")
    f32 = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom).raycast_nearest(rays, s["max_toi"])
    hit = (ref.leaf != sq.NO_HIT) & (f32.leaf == ref.leaf)
    assert hit.mean() > 0.2
    assert (f32.toi[hit].astype(np.float64) != got.toi[hit]).mean() > 0.5


def test_f32_and_f64_scenes_stay_apart(ctx):
    s = scenes.boxes_scene(seed=65, n_boxes=100, n_rays=4)
    geom = sq.Geometry("boxes", 3, s["prims"])
    s64 = sq.DeviceBvh64(ctx, sq.HostBvh.build_f64(3, geom.world_aabbs_f64()), geom)
    with pytest.raises(sq.SqError) as e:  # an f32 entry point on an f64 scene
        ctx.check(sq.lib().sq_bvh_refit(ctx.h, s64.h, sq._p(geom.prims)), "refit")
    assert e.value.code == sq.SQ_ERR_UNSUPPORTED
    s32 = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    leaf = np.empty(4, np.uint32)
    rc = sq.lib().sq_raycast_nearest_f64(ctx.h, s32.h, sq._p(s["rays"].astype(np.float64)), 4, 10.0, None, None,
                                         sq._p(leaf), None, None, None)
    assert rc == sq.SQ_ERR_UNSUPPORTED
    s64.close()
    s32.close()


# -- lists, casts and overlap with Scalar = f64 ---------------------------------

def scene64(ctx, geom):
    return sq.DeviceBvh64(ctx, sq.HostBvh.build_f64(geom.dim, geom.world_aabbs_f64()), geom)


def same_lists64(ref, got, label):
    assert np.array_equal(ref.count, got.count), f"{label}: counts differ on {(ref.count != got.count).sum()}"
    k = ref.leaf.shape[1]
    mask = np.arange(k)[None, :] < np.minimum(ref.count, k)[:, None]
    assert np.array_equal(ref.leaf[mask], got.leaf[mask]), f"{label}: list leaves"
    assert np.array_equal(ref.toi[mask].view(np.uint64), got.toi[mask].view(np.uint64)), f"{label}: f64 list toi"
    assert np.array_equal(ref.normal[mask].view(np.uint32), got.normal[mask].astype(np.float32).view(np.uint32)), \
        f"{label}: list normals"


def same_nearest64(ref, got, label):
    assert np.array_equal(ref.leaf, got.leaf), f"{label}: leaf differs on {(ref.leaf != got.leaf).sum()}"
    assert np.array_equal(ref.toi.view(np.uint64), got.toi.view(np.uint64)), f"{label}: f64 toi"
    assert np.array_equal(ref.normal.view(np.uint32), got.normal.astype(np.float32).view(np.uint32)), \
        f"{label}: normals"


def box_casts(rng, n, dim, lo, hi, hlo, hhi):
    o = rng.range(lo, hi, (n, dim))
    d = scenes.normalize_rows(rng.range(-1.0, 1.0, (n, dim)))
    h = rng.range(hlo, hhi, (n, dim))
    return np.ascontiguousarray(np.concatenate([o, d, -h, h], axis=1), dtype=np.float32)


def regions(rng, n, dim, lo, hi, hlo, hhi):
    c = rng.range(lo, hi, (n, dim))
    h = rng.range(hlo, hhi, (n, dim))
    return np.ascontiguousarray(np.concatenate([c - h, c + h], axis=1), dtype=np.float32)


@pytest.mark.parametrize("dim", [2, 3, 6])
def test_lists_casts_overlap_boxes(ctx, dim):
    s = scenes.boxes_scene(seed=70 + dim, n_boxes=8000, n_rays=4096, dim=dim)
    prims = s["prims"]
    if dim >= 4:
        c, h = (prims[:, :dim] + prims[:, dim:]) / 2, (prims[:, dim:] - prims[:, :dim]) / 2
        prims = np.ascontiguousarray(np.concatenate([c - 6 * h, c + 6 * h], axis=1), dtype=np.float32)
    geom = sq.Geometry("boxes", dim, prims)
    o = O.Scene("boxes", dim, prims, prec=64)
    g = scene64(ctx, geom)
    rng = scenes.Rng(80 + dim)
    rays = s["rays"]
    ra = o.all(rays, s["max_toi"], k=16)
    assert (ra.count > 0).sum() > 50 and (dim >= 4 or (ra.count > 1).sum() > 50)
    same_lists64(ra, g.raycast_all(rays.astype(np.float64), s["max_toi"], k=16), f"all D={dim}")
    casts = box_casts(rng, 4096, dim, -120.0, 120.0, 0.2, 3.0)
    lens = rng.range(0.0, 300.0, 4096).astype(np.float32)
    cn = o.shapecast_nearest(casts, lens)
    assert (cn.leaf != O.NO_HIT).sum() > (50 if dim < 4 else 10)  # sparse in 6 dimensions
    same_nearest64(cn, g.shapecast_nearest(casts.astype(np.float64), lens.astype(np.float64)), f"cast D={dim}")
    same_lists64(o.shapecast_all(casts, lens, k=8), g.shapecast_all(casts.astype(np.float64), lens.astype(np.float64),
                                                                      k=8), f"cast all D={dim}")
    reg = regions(rng, 4096, dim, -100.0, 100.0, 0.5, 12.0)
    want = o.overlap(reg)
    assert want[1].size > (100 if dim < 4 else 10)
    got = g.overlap(reg.astype(np.float64))
    assert np.array_equal(want[0], got[0]) and np.array_equal(want[1], got[1]), f"overlap D={dim}"
    g.close()


@pytest.mark.parametrize("kind", ["balls", "balls_near"])
def test_crossings_casts_overlap_balls(ctx, kind):
    rng = scenes.Rng(90)
    n = 6000
    prims = np.concatenate([rng.range(-60.0, 60.0, (n, 3)), rng.range(0.3, 3.0, (n, 1))], axis=1).astype(np.float32)
    o0 = rng.range(-100.0, 100.0, (4096, 3))
    d = scenes.normalize_rows(rng.range(-50.0, 50.0, (4096, 3)) - o0)
    rays = np.ascontiguousarray(np.concatenate([o0, d], axis=1), dtype=np.float32)
    geom = sq.Geometry(kind, 3, prims)
    o = O.Scene(kind, 3, prims, prec=64)
    g = scene64(ctx, geom)
    cr = o.all(rays, 400.0, k=24, crossings=True)
    assert (cr.count >= 2).sum() > 50
    same_lists64(cr, g.raycast_crossings(rays.astype(np.float64), 400.0, k=24), f"{kind} crossings")
    same_lists64(o.all(rays, 400.0, k=24), g.raycast_all(rays.astype(np.float64), 400.0, k=24), f"{kind} all")
    # ball casts: the probe's max[0] is the swept radius
    casts = box_casts(rng, 4096, 3, -80.0, 80.0, 0.5, 0.5)
    cn = o.shapecast_nearest(casts, 200.0)
    assert (cn.leaf != O.NO_HIT).sum() > 100
    same_nearest64(cn, g.shapecast_nearest(casts.astype(np.float64), 200.0), f"{kind} cast")
    reg = regions(rng, 4096, 3, -60.0, 60.0, 0.5, 8.0)
    want = o.overlap(reg)
    got = g.overlap(reg.astype(np.float64))
    assert np.array_equal(want[0], got[0]) and np.array_equal(want[1], got[1]), f"{kind} overlap"
    g.close()


def test_triangles_lists_casts_overlap_filter(ctx):
    s = scenes.terrain_scene(seed=8, nx=96, ny=64, n_coherent=4096, n_incoherent=4096)
    layers = (np.arange(s["prims"].shape[0]) % 3 + 1).astype(np.uint64)
    geom = sq.Geometry("tris", 3, s["prims"], layers=layers)
    o = O.Scene("tris", 3, s["prims"], layers=layers, prec=64)
    g = scene64(ctx, geom)
    rng = scenes.Rng(91)
    rays = s["rays"]
    same_lists64(o.all(rays, s["max_toi"], k=16), g.raycast_all(rays.astype(np.float64), s["max_toi"], k=16),
                 "tri all")
    same_lists64(o.all(rays, s["max_toi"], k=16, mask=0b10), g.raycast_all(rays.astype(np.float64), s["max_toi"],
                                                                            k=16, mask=0b10), "tri all filtered")
    lo, hi = s["prims"].reshape(-1, 3).min(axis=0), s["prims"].reshape(-1, 3).max(axis=0)
    o0 = rng.range(0.0, 1.0, (4096, 3)) * (hi - lo) + lo
    o0[:, 2] = hi[2] + 5.0
    d = scenes.normalize_rows(np.concatenate([rng.range(-0.3, 0.3, (4096, 2)), -np.ones((4096, 1))], axis=1))
    h = rng.range(0.2, 2.0, (4096, 3))
    casts = np.ascontiguousarray(np.concatenate([o0, d, -h, h], axis=1), dtype=np.float32)
    cn = o.shapecast_nearest(casts, 500.0)
    assert (cn.leaf != O.NO_HIT).mean() > 0.5
    same_nearest64(cn, g.shapecast_nearest(casts.astype(np.float64), 500.0), "tri cast")
    same_lists64(o.shapecast_all(casts, 500.0, k=8), g.shapecast_all(casts.astype(np.float64), 500.0, k=8),
                 "tri cast all")
    c = rng.range(0.0, 1.0, (2048, 3)) * (hi - lo) + lo
    hh = rng.range(0.5, 6.0, (2048, 3))
    reg = np.ascontiguousarray(np.concatenate([c - hh, c + hh], axis=1), dtype=np.float32)
    want = o.overlap(reg, mask=0b101)
    got = g.overlap(reg.astype(np.float64), mask=0b101)
    assert want[1].size > 100
    assert np.array_equal(want[0], got[0]) and np.array_equal(want[1], got[1]), "tri overlap filtered"
    g.close()


def test_f64_lists_empty_scene_and_no_queries(ctx):
    geom = sq.Geometry("boxes", 3, np.zeros((0, 6), np.float32))
    g = scene64(ctx, geom)
    r = g.raycast_all(np.array([[0, 0, 0, 1, 0, 0]], np.float64), 10.0, k=4)
    assert r.count[0] == 0
    off, lv = g.overlap(np.array([[-1, -1, -1, 1, 1, 1]], np.float64))
    assert list(off) == [0, 0] and lv.size == 0
    c = g.shapecast_nearest(np.zeros((0, 12), np.float64), 10.0)
    assert c.leaf.size == 0
    g.close()
