"""The learned guide on the GPU, through the C ABI (include/sq_guide.h).

* The tcgen05 GEMM it trains with == an f32 product of the same bf16
  operands (torch), relative error <= 1e-4 of the row scale.
* Forward/backward gradients == the CPU restatement (tests/guide_ref.py,
  float64 with the GPU's bf16 rounding points): relative Frobenius error
  <= 2e-2 per tensor (bf16 rounding of activations and dZ can land on the
  other side of a tie between the f32 and f64 sums); loss within 1e-4.
* The fused inference kernel's top-1 bucket == the CPU argmax wherever the
  CPU's top-2 margin exceeds 1e-3, and its logit is within 1e-3 of the CPU
  maximum everywhere (bf16 rounding of an activation and the f32 sums move a
  logit by about 1e-4 at most here).
* Whatever bucket seeds a query (trained, untrained, random, out of range),
  the learned-seeded nearest hits are bit-identical to the plain query's and
  to the CPU oracle's.
* Seeded with the true bucket of every ray, the walk tests no more boxes
  than the plain walk; trained on rays labelled by the plain traversal, the
  guide predicts the hit's bucket far better than untrained and its seeds
  cost fewer box tests than the untrained network's.
"""
import numpy as np
import pytest

import guide_ref as R
import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_nearest
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def ctx():
    c = sq.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (256, 384, 128), (200, 136, 72), (8192, 128, 4096),
                                   (4096, 128, 8192), (1024, 4096, 128)])
def test_gemm_matches_f32_product(ctx, m, n, k):
    g = torch.Generator(device="cpu").manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16).to(DEV)
    b = torch.randn(n, k, generator=g).to(torch.bfloat16).to(DEV)
    c = torch.full((m, n), float("nan"), device=DEV)
    torch.cuda.synchronize()
    sq.gemm_bf16_tn_d(ctx, a, b, c, m, n, k, k, k, n)
    ctx.synchronize()
    want = a.double() @ b.double().T
    scale = (a.double().abs() @ b.double().abs().T)
    err = ((c.double() - want).abs() / scale.clamp_min(1e-30)).max().item()
    assert not torch.isnan(c).any()
    assert err <= 1e-4, err


def small_terrain():
    s = scenes.terrain_scene(seed=5, nx=128, ny=64, n_coherent=8192, n_incoherent=8192)
    geom = sq.Geometry("tris", 3, s["prims"])
    return s, geom, sq.HostBvh.build(geom)


def test_gradients_match_cpu(ctx):
    s, geom, tree = small_terrain()
    scene = sq.DeviceBvh(ctx, tree, geom)
    guide = sq.Guide(scene, depth=12, batch=256, seed=3)
    info = guide.info()
    assert info["n_buckets"] == 4096 and info["n_out"] == 4096
    rays = s["rays"][::64][:256].copy()
    d_rays = torch.from_numpy(rays).to(DEV)
    d_lab = torch.empty(256, dtype=torch.int32, device=DEV)
    torch.cuda.synchronize()
    guide.label_d(d_rays, 256, s["max_toi"], d_lab)
    ctx.synchronize()
    labels = d_lab.cpu().numpy()
    assert (labels >= 0).mean() > 0.3
    loss = guide.forward_backward_d(d_rays, d_lab)
    g_gpu = R.unpack(guide.get_grads(), info["n_out"])
    p = R.unpack(guide.get_params(), info["n_out"])
    root = scene.read_bounds()[0]
    x = R.features(rays, root[:3], root[3:])
    loss_ref, g_ref = R.loss_and_grads(p, x, labels, info["n_buckets"])
    assert abs(loss - loss_ref) <= 1e-4 * max(1.0, abs(loss_ref)), (loss, loss_ref)
    for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        ref = g_ref[k]
        err = np.linalg.norm(g_gpu[k] - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err <= 2e-2, (k, err)


@pytest.mark.parametrize("grid", ["full", "ragged"])
def test_inference_matches_cpu_argmax(ctx, grid):
    if grid == "full":  # 4,096 buckets, fewer tiles than CTAs
        s, geom, tree = small_terrain()
    else:  # a few hundred buckets (a partial output chunk), several tiles per CTA
        s = scenes.terrain_scene(seed=6, nx=20, ny=18, n_coherent=20000, n_incoherent=20000)
        geom = sq.Geometry("tris", 3, s["prims"])
        tree = sq.HostBvh.build(geom)
    scene = sq.DeviceBvh(ctx, tree, geom)
    guide = sq.Guide(scene, depth=12, batch=256, seed=9)
    info = guide.info()
    assert info["n_out"] % 128 == 0 and info["n_buckets"] <= info["n_out"] < info["n_buckets"] + 128
    rays = s["rays"]
    n = rays.shape[0] - 37  # a ragged last tile
    d_rays = torch.from_numpy(rays[:n].copy()).to(DEV)
    d_b = torch.full((n,), -7, dtype=torch.int32, device=DEV)
    torch.cuda.synchronize()
    guide.predict_d(d_rays, n, d_b)
    ctx.synchronize()
    got = d_b.cpu().numpy()
    p = R.unpack(guide.get_params(), info["n_out"])
    root = scene.read_bounds()[0]
    _, logits = R.forward(p, R.features(rays[:n], root[:3], root[3:]))
    assert ((got >= 0) & (got < info["n_buckets"])).all()
    top2 = np.sort(logits, axis=1)[:, -2:]
    clear = (top2[:, 1] - top2[:, 0]) > 1e-3
    want = logits.argmax(axis=1)
    assert clear.mean() > 0.5
    assert np.array_equal(got[clear], want[clear])
    assert (logits[np.arange(n), got] >= top2[:, 1] - 1e-3).all()


@pytest.fixture(scope="module")
def terrain(ctx):
    s = scenes.terrain_scene(seed=1)
    geom = sq.Geometry("tris", 3, s["prims"])
    tree = sq.HostBvh.build(geom)
    scene = sq.DeviceBvh(ctx, tree, geom)
    return s, geom, tree, scene


def _nearest_d(scene, d_rays, n, max_toi):
    leaf = torch.empty(n, dtype=torch.int32, device=DEV)
    toi = torch.empty(n, dtype=torch.float32, device=DEV)
    nrm = torch.empty((n, 3), dtype=torch.float32, device=DEV)
    torch.cuda.synchronize()
    st = scene.raycast_nearest_d(d_rays, n, max_toi, leaf, toi, nrm, stats=True)
    scene.ctx.synchronize()
    return leaf, toi, nrm, st


def test_seeded_hits_identical_whatever_the_seed(ctx, terrain):
    s, geom, tree, scene = terrain
    n = s["rays"].shape[0]
    d_rays = torch.from_numpy(s["rays"]).to(DEV)
    leaf0, toi0, nrm0, _ = _nearest_d(scene, d_rays, n, s["max_toi"])
    guide = sq.Guide(scene, seed=1)
    info = guide.info()
    gen = torch.Generator(device="cpu").manual_seed(0)
    seeds = {
        "untrained": None,
        "random": torch.randint(0, info["n_buckets"], (n,), generator=gen, dtype=torch.int32).to(DEV),
        "out_of_range": torch.randint(-5, info["n_buckets"] + 5, (n,), generator=gen, dtype=torch.int32).to(DEV),
    }
    # after the seed the walk follows the context's order: near-first, or the crate's far-first child order
    for order in (sq.ORDER_NEAR_FIRST, sq.ORDER_REFERENCE):
        ctx.set_order(order)
        for name, d_b in seeds.items():
            leaf = torch.empty(n, dtype=torch.int32, device=DEV)
            toi = torch.empty(n, dtype=torch.float32, device=DEV)
            nrm = torch.empty((n, 3), dtype=torch.float32, device=DEV)
            torch.cuda.synchronize()
            guide.raycast_nearest_guided_d(d_rays, n, s["max_toi"], leaf, toi, nrm, d_bucket=d_b)
            ctx.synchronize()
            assert torch.equal(leaf, leaf0), (order, name)
            assert torch.equal(toi.view(torch.int32), toi0.view(torch.int32)), (order, name)
            assert torch.equal(nrm.view(torch.int32), nrm0.view(torch.int32)), (order, name)
    ctx.set_order(sq.ORDER_NEAR_FIRST)
    # and the host-buffer entry point against the CPU oracle on a slice
    o = O.Scene("tris", 3, s["prims"])
    sl = s["rays"][:65536]
    assert_same_nearest(o.nearest(sl, s["max_toi"]), guide.raycast_nearest_guided(sl, s["max_toi"]),
                        label="guided vs oracle")


def test_trained_guide_gains_over_untrained(ctx, terrain):
    """What training buys, in the walk's own work. Box tests per ray (the
    QueryStats nodes_visited counter): seeded with the TRUE bucket of every
    ray (the upper bound of any guide) never exceed the plain near-first
    walk's, and seeded with the trained network they fall below seeding with
    the untrained one; top-1 accuracy rises far above the untrained
    network's; every seeded answer stays bit-identical to the plain one."""
    s, geom, tree, scene = terrain
    nx, ny = s["grid"]
    zmin, zmax = s["zrange"]
    n_train = 1 << 21
    train = scenes.terrain_rays(scenes.Rng(4), nx, ny, zmin, zmax, n_train // 2, n_train // 2)
    d_train = torch.from_numpy(train).to(DEV)
    d_lab = torch.empty(n_train, dtype=torch.int32, device=DEV)
    guide = sq.Guide(scene, seed=2)
    n = s["rays"].shape[0]
    d_rays = torch.from_numpy(s["rays"]).to(DEV)
    torch.cuda.synchronize()
    guide.label_d(d_train, n_train, s["max_toi"], d_lab)
    d_lt = torch.empty(n, dtype=torch.int32, device=DEV)
    guide.label_d(d_rays, n, s["max_toi"], d_lt)
    ctx.synchronize()
    hit = d_lt >= 0
    leaf0, toi0, _, st0 = _nearest_d(scene, d_rays, n, s["max_toi"])
    plain = st0["nodes_visited"] / n

    def seeded(d_b):
        leaf = torch.empty(n, dtype=torch.int32, device=DEV)
        toi = torch.empty(n, dtype=torch.float32, device=DEV)
        st = guide.raycast_nearest_guided_d(d_rays, n, s["max_toi"], leaf, toi, d_bucket=d_b, stats=True)
        ctx.synchronize()
        assert torch.equal(leaf, leaf0) and torch.equal(toi.view(torch.int32), toi0.view(torch.int32))
        return st["nodes_visited"] / n

    def measure():
        d_b = torch.empty(n, dtype=torch.int32, device=DEV)
        guide.predict_d(d_rays, n, d_b)
        ctx.synchronize()
        acc = (d_b[hit] == d_lt[hit]).float().mean().item()
        return acc, seeded(d_b)

    perfect = seeded(d_lt)  # misses carry -1: a plain walk
    acc0, nodes0 = measure()
    losses = guide.train_d(d_train, d_lab, n_train, 6)
    assert losses[-1] < losses[0] and np.isfinite(losses).all()
    acc1, nodes1 = measure()
    print(f"top-1 untrained {acc0:.4f} trained {acc1:.4f}; box tests per ray: plain near-first {plain:.2f}, "
          f"seeded untrained {nodes0:.2f}, trained {nodes1:.2f}, true bucket {perfect:.2f}")
    assert perfect <= plain
    assert nodes1 < nodes0
    assert acc1 > 0.1 and acc1 > 20 * acc0
    blob = guide.save()
    g2 = sq.Guide(scene, seed=99)
    g2.load(blob)
    assert np.array_equal(g2.get_params(), guide.get_params())
