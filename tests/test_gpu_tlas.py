"""Two-level path on the GPU == the oracle's Tlas (accel/tlas.rs), bit for
bit: the reference's two-level test scenes (oriented boxes, ball instances,
shells, labelled instances), the instanced-mesh workload with in-kernel BLAS
descent, the mixed persistent launch, device refit and a CUDA-graph frame."""
import math

import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_csr, assert_same_lists, assert_same_nearest, ctx
from refscenes import axis_ray, point, random_oriented_boxes, ray_new
from spatial_query_b200 import scenes
from spatial_query_b200.scenes import Rng

pytestmark = pytest.mark.gpu

EYE3 = np.eye(3, dtype=np.float32)


@pytest.fixture(params=[sq.ORDER_NEAR_FIRST, sq.ORDER_REFERENCE], ids=["near_first", "reference_order"])
def order(request):
    ctx().set_order(request.param)
    yield request.param
    ctx().set_order(sq.ORDER_NEAR_FIRST)


def tpair(kind, dim, rot, trans, param, layers=None, sub=None):
    o = O.TlasScene(kind, dim, rot, trans, param, layers=layers, sub=sub)
    g = sq.DeviceTlas(ctx(), kind, dim, rot, trans, param, layers=layers, sub_objects=sub)
    return o, g


def test_end_to_end_hit_point_and_normal():
    """two_level.rs:207-224."""
    o, g = tpair("box", 3, EYE3[None], np.array([[5, 0, 0]], np.float32), np.ones((1, 3), np.float32))
    h = g.raycast_nearest(axis_ray(), 100.0)
    assert h.leaf[0] == 0 and abs(h.toi[0] - 4) < 1e-4 and abs(h.point[0, 0] - 4) < 1e-4
    assert abs(h.normal[0, 0] + 1) < 1e-4


@pytest.mark.parametrize("dim,seed,n", [(3, 0x7ABC_1234, 64), (2, 0x2020_2020, 48)])
def test_oriented_box_scenes(dim, seed, n, order):
    """two_level.rs:263-287: nearest and all hits."""
    rng = Rng(seed)
    for _ in range(200):
        rot, trans, halves = random_oriented_boxes(rng, n, dim)
        ray = ray_new(point(rng, dim, -60.0, 60.0), point(rng, dim, -1.0, 1.0))
        if not np.any(ray[dim:]):
            continue
        o, g = tpair("box", dim, rot, trans, halves)
        assert_same_nearest(o.nearest(ray, 500.0), g.raycast_nearest(ray, 500.0), sub=False)
        assert_same_lists(o.all(ray, 500.0, k=n), g.raycast_all(ray, 500.0, k=n), sub=False)


def test_refit_matches_rebuild_when_instances_move():
    """two_level.rs:289-332: move every instance, deform every 7th, refit on
    the device; bounds, world AABBs and queries match the oracle's refit."""
    rng = Rng(0xF00D_5EED)
    rot, trans, halves = random_oriented_boxes(rng, 200, 3)
    o, g = tpair("box", 3, rot, trans, halves)
    for frame in range(10):
        for i in range(200):
            trans[i] = trans[i] + point(rng, 3, -1.5, 1.5)
            if i % 7 == 0:
                halves[i] = halves[i] * np.float32(1.05)
        o.refit(trans, param=halves)
        g.refit(trans, param=halves)
        nb, wa = g.read_bounds()
        ot = o.tree()
        assert np.array_equal(nb, ot["bounds"]) and np.array_equal(wa, ot["world_aabbs"])
        rays = []
        for _ in range(40):
            r = ray_new(point(rng, 3, -60.0, 60.0), point(rng, 3, -1.0, 1.0))
            if np.any(r[3:]):
                rays.append(r)
        rays = np.stack(rays)
        assert_same_nearest(o.nearest(rays, 500.0), g.raycast_nearest(rays, 500.0), sub=False)


def test_needs_rebuild_triggers_after_spreading_instances():
    """two_level.rs:334-362."""
    rng = Rng(0xCAFE_1111)
    n = 128
    trans = np.stack([point(rng, 3, -2.0, 2.0) for _ in range(n)])
    rot = np.repeat(EYE3[None], n, 0)
    o, g = tpair("box", 3, rot, trans, np.full((n, 3), 0.5, np.float32))
    assert not g.needs_rebuild(2.0)
    spread = np.stack([point(rng, 3, -500.0, 500.0) for _ in range(n)])
    g.refit(spread)
    assert g.needs_rebuild(2.0)


def _ball_instances(rng, n):
    trans = np.stack([point(rng, 3, -30.0, 30.0) for _ in range(n)])
    return trans, rng.range(0.5, 2.0, n)


def test_ball_instance_casts_and_overlaps(order):
    """shape_overlap.rs:344-411."""
    rng = Rng(0x1234_ABCD)
    for _ in range(150):
        trans, radii = _ball_instances(rng, 48)
        o, g = tpair("ball", 3, np.repeat(EYE3[None], 48, 0), trans, radii)
        dn = ray_new(point(rng, 3, -50.0, 50.0), point(rng, 3, -1.0, 1.0))
        cast = np.concatenate([dn, np.full(3, -0.75, np.float32), np.full(3, 0.75, np.float32)])
        if not np.any(cast[3:6]):
            continue
        assert_same_nearest(o.shapecast_nearest(cast, 500.0), g.shapecast_nearest(cast, 500.0), sub=False)
        assert_same_lists(o.shapecast_all(cast, 500.0, k=48), g.shapecast_all(cast, 500.0, k=48), sub=False)
    rng = Rng(0x9999_5555)
    for _ in range(150):
        trans, radii = _ball_instances(rng, 64)
        o, g = tpair("ball", 3, np.repeat(EYE3[None], 64, 0), trans, radii)
        c = point(rng, 3, -30.0, 30.0)
        hh = point(rng, 3, 1.0, 6.0)
        region = np.concatenate([c - hh, c + hh])
        assert_same_csr(o.overlap(region), g.overlap(region))


def test_ball_instance_crossings():
    """crossings.rs:286-320."""
    rng = Rng(0x7717_9999)
    for _ in range(150):
        centers = np.stack([point(rng, 3, -30.0, 30.0) for _ in range(48)])
        radii = rng.range(1.0, 4.0, 48)
        o, g = tpair("ball", 3, np.repeat(EYE3[None], 48, 0), centers, radii)
        ray = ray_new(point(rng, 3, -40.0, 40.0), point(rng, 3, -1.0, 1.0))
        if not np.any(ray[3:]):
            continue
        assert_same_lists(o.all(ray, 500.0, k=96, crossings=True), g.raycast_crossings(ray, 500.0, k=96), sub=False)


def test_sub_object_survives_tlas_ray():
    """result_identity.rs:251-270."""
    trans = np.zeros((6, 3), np.float32)
    trans[:, 0] = 2.0 * (np.arange(6, dtype=np.float32) + 1)
    sub = np.arange(6, dtype=np.uint32) * 10 + 1
    o, g = tpair("ball", 3, np.repeat(EYE3[None], 6, 0), trans, np.full(6, 0.6, np.float32), sub=sub)
    n = g.raycast_nearest(axis_ray(), 100.0)
    assert n.sub_object[0] == n.leaf[0] * 10 + 1
    a = g.raycast_all(axis_ray(), 100.0, k=6)
    assert all(a.sub_object[0, j] == a.leaf[0, j] * 10 + 1 for j in range(a.count[0]))
    assert_same_nearest(o.nearest(axis_ray(), 100.0), n)


def test_reference_order_counters_match():
    ctx().set_order(sq.ORDER_REFERENCE)
    try:
        rng = Rng(0x7ABC_1234)
        rot, trans, halves = random_oriented_boxes(rng, 256, 3)
        o, g = tpair("box", 3, rot, trans, halves)
        rays = np.stack([ray_new(point(rng, 3, -60.0, 60.0), point(rng, 3, -1.0, 1.0)) for _ in range(500)])
        ref = o.nearest(rays, 500.0, stats=True)
        got = g.raycast_nearest(rays, 500.0, stats=True)
        assert_same_nearest(ref, got, sub=False)
        assert list(got.stats.values()) == list(ref.stats.sum(axis=0))
    finally:
        ctx().set_order(sq.ORDER_NEAR_FIRST)


# -- instanced meshes (the two-level benchmark scene) -------------------------

def mesh_pair(s):
    oblas = O.BlasSet(s["blas_offsets"], s["blas_tris"])
    o = O.TlasScene("mesh", 3, s["rot"], s["trans"], s["scale"], blas_id=s["blas_id"], blas=oblas)
    blas = sq.BlasSet(ctx(), s["meshes"])
    g = sq.DeviceTlas(ctx(), "mesh", 3, s["rot"], s["trans"], s["scale"], blas_id=s["blas_id"], blas=blas)
    return oblas, o, blas, g


@pytest.fixture(scope="module")
def small_instanced():
    s = scenes.instanced_scene(seed=7, n_instances=256, n_blas=4, n_rays=20000, n_casts=4096, n_regions=4096,
                               n_frames=12, blas_lo=2000, blas_hi=20000)
    return (s,) + mesh_pair(s)


def test_mesh_instances_small(small_instanced, order):
    s, oblas, o, blas, g = small_instanced
    _, wa = g.read_bounds()
    assert np.array_equal(wa, o.tree()["world_aabbs"])
    ref = o.nearest(s["rays"], s["max_toi"])
    assert (ref.leaf != O.NO_HIT).mean() > 0.05
    assert_same_nearest(ref, g.raycast_nearest(s["rays"], s["max_toi"]), label="mesh nearest")
    assert_same_lists(o.all(s["rays"], s["max_toi"], k=8), g.raycast_all(s["rays"], s["max_toi"], k=8),
                      label="mesh all")
    assert_same_lists(o.all(s["rays"], s["max_toi"], k=8, crossings=True),
                      g.raycast_crossings(s["rays"], s["max_toi"], k=8), label="mesh crossings")
    assert_same_nearest(o.shapecast_nearest(s["casts"], s["cast_len"]),
                        g.shapecast_nearest(s["casts"], s["cast_len"]), label="mesh casts")
    assert_same_csr(o.overlap(s["regions"]), g.overlap(s["regions"]), label="mesh overlaps")


def test_mixed_launch_and_graph_frames(small_instanced):
    """One persistent launch over rays + casts + regions equals the separate
    queries; a captured frame (translation steps + refit + mixed launch)
    replays to the oracle's refit scene each frame."""
    import torch
    s, oblas, o, blas, g = small_instanced
    c = ctx()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.ExternalStream(c.stream, device=dev)
    nr, nc, no, k = len(s["rays"]), len(s["casts"]), len(s["regions"]), 16
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rays, casts, regions, lens = T(s["rays"]), T(s["casts"]), T(s["regions"]), T(s["cast_len"])
    ro = dict(leaf=torch.empty(nr, dtype=torch.int32, device=dev), toi=torch.empty(nr, device=dev),
              normal=torch.empty((nr, 3), device=dev), point=torch.empty((nr, 3), device=dev),
              sub=torch.empty(nr, dtype=torch.int32, device=dev))
    co = dict(leaf=torch.empty(nc, dtype=torch.int32, device=dev), toi=torch.empty(nc, device=dev),
              normal=torch.empty((nc, 3), device=dev), point=torch.empty((nc, 3), device=dev),
              sub=torch.empty(nc, dtype=torch.int32, device=dev))
    rcount = torch.empty(no, dtype=torch.int32, device=dev)
    rleaves = torch.empty((no, k), dtype=torch.int32, device=dev)
    steps = T(s["frame_steps"])

    def mixed():
        g.mixed_d(rays=rays, n_rays=nr, ray_max_toi=s["max_toi"], ray_out=ro, casts=casts, n_casts=nc,
                  cast_max_toi=0.0, cast_max_toi_per_query=lens, cast_out=co, regions=regions, n_regions=no,
                  region_k=k, region_count=rcount, region_leaves=rleaves)

    def check(oscene):
        torch.cuda.synchronize()
        rn, cn = oscene.nearest(s["rays"], s["max_toi"]), oscene.shapecast_nearest(s["casts"], s["cast_len"])
        assert np.array_equal(ro["leaf"].cpu().numpy().view(np.uint32), rn.leaf)
        hit = rn.leaf != O.NO_HIT
        assert np.array_equal(ro["toi"].cpu().numpy()[hit].view(np.uint32), rn.toi[hit].view(np.uint32))
        assert np.array_equal(ro["sub"].cpu().numpy().view(np.uint32)[hit], rn.sub[hit])
        assert np.array_equal(co["leaf"].cpu().numpy().view(np.uint32), cn.leaf)
        off, lv = oscene.overlap(s["regions"])
        cnt = np.diff(off).astype(np.uint32)
        assert np.array_equal(rcount.cpu().numpy().view(np.uint32), cnt)
        got = rleaves.cpu().numpy().view(np.uint32)
        for q in range(no):
            m = min(int(cnt[q]), k)
            assert list(got[q, :m]) == list(lv[int(off[q]):int(off[q]) + m])

    mixed()
    check(o)
    # A frame: add this frame's N(0,1) steps to every translation, refit, query.
    # The graph reads the steps from one device buffer; before each replay the
    # frame's own steps are copied into it on the context's stream, so every
    # replay moves the instances by a different amount and the translations
    # accumulate across replays, as the benchmark's 100 frames do.
    delta = torch.empty_like(steps[0])
    trans = s["trans"].copy()
    with torch.cuda.stream(stream):
        delta.copy_(steps[0])
        c.graph_begin()
        g.refit_d(d_delta=delta)
        mixed()
        graph = c.graph_end()
    n_frames = s["frame_steps"].shape[0]
    assert n_frames >= 10
    for f in range(n_frames):
        with torch.cuda.stream(stream):
            delta.copy_(steps[f])
        graph.launch()
        trans = trans + s["frame_steps"][f]
        o.refit(trans)
        check(o)
        nb, wa = g.read_bounds()
        ot = o.tree()
        assert np.array_equal(nb, ot["bounds"]), f"frame {f}: node bounds differ from the oracle's refit"
        assert np.array_equal(wa, ot["world_aabbs"]), f"frame {f}: instance world AABBs differ"
    graph.close()


def test_instanced_full_nearest():
    """The full two-level workload: 4,096 instances of 16 meshes
    (10k..200k triangles), 1,000,000 rays, 262,144 casts, 262,144 regions."""
    s = scenes.instanced_scene(seed=2, n_frames=1)
    oblas, o, blas, g = mesh_pair(s)
    ref = o.nearest(s["rays"], s["max_toi"])
    assert_same_nearest(ref, g.raycast_nearest(s["rays"], s["max_toi"]), label="instanced nearest")
    assert_same_nearest(o.shapecast_nearest(s["casts"], s["cast_len"]),
                        g.shapecast_nearest(s["casts"], s["cast_len"]), label="instanced casts")
    assert_same_csr(o.overlap(s["regions"]), g.overlap(s["regions"]), label="instanced overlaps")


# -- crates/viewport-lib-query/src/lib.rs:338-431 on the device ----------------

def _cube_pair(trans, scale=None):
    from refscenes import cube_mesh, mesh_instances
    cube = cube_mesh(2.0)
    rot, t, sc, bid = mesh_instances(trans, scale)
    oblas = O.BlasSet(np.array([0, cube.shape[0]], np.uint64), cube)
    o = O.TlasScene("mesh", 3, rot, t, sc, blas_id=bid, blas=oblas)
    blas = sq.BlasSet(ctx(), [cube])
    g = sq.DeviceTlas(ctx(), "mesh", 3, rot, t, sc, blas_id=bid, blas=blas)
    return oblas, o, blas, g


@pytest.mark.parametrize("case", ["face_and_id", "nearest_wins", "away_misses", "scaled_world_toi"])
def test_viewport_mesh_known_answers(case, order):
    """The four mesh-instance tests of viewport-lib-query (lib.rs:338-431)
    through the device's mesh instances: the reference's answers hold, and
    every field equals the oracle's bit for bit."""
    ray = lambda d: ray_new(np.zeros(3, np.float32), np.asarray(d, np.float32))[None]
    if case == "face_and_id":
        keep = _cube_pair([[5.0, 0.0, 0.0]])
        r = ray([1, 0, 0])
    elif case == "nearest_wins":
        keep = _cube_pair([[10.0, 0.0, 0.0], [5.0, 0.0, 0.0]])
        r = ray([1, 0, 0])
    elif case == "away_misses":
        keep = _cube_pair([[5.0, 0.0, 0.0]])
        r = ray([-1, 0, 0])
    else:
        keep = _cube_pair([[20.0, 0.0, 0.0]], scale=[3.0])
        r = ray([1, 0, 0])
    _, o, _, g = keep
    ref = o.nearest(r, 100.0)
    got = g.raycast_nearest(r, 100.0)
    assert_same_nearest(ref, got, label=case)
    if case == "face_and_id":
        assert got.leaf[0] == 0 and abs(float(got.toi[0]) - 4.0) < 1e-3 and abs(float(got.normal[0, 0])) > 0.9
        assert got.sub_object[0] < 12
    elif case == "nearest_wins":
        assert [100, 200][got.leaf[0]] == 200
    elif case == "away_misses":
        assert got.leaf[0] == O.NO_HIT
    else:
        assert got.leaf[0] == 0 and abs(float(got.toi[0]) - 17.0) < 1e-2
