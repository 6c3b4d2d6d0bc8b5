"""Marched implicit-surface leaves as a consumer narrow phase (the field
leaves of tests/field.rs:45-150, written as CUDA and compiled with NVRTC
into the traversal kernels), with every crossing listed by
raycast_crossings through the optional sq_narrow_crossings hook.

The checks are the reference's own for field leaves: the tree agrees with
the naive scan bit for bit, nearest and crossings, so broad phase never
prunes a leaf the march would hit (tests/field.rs:165-210; the naive scan
here is the same kernels over a one-leaf tree holding every blob), in both
traversal orders; the march converges to a sphere's analytic entry and
exit, 17 and 23, with the near-face normal along -x (field.rs:212-251);
misses and the empty scene return nothing (field.rs:253-275).

The march spans [0, 500] whatever limit the traversal passes, and returns
only roots within it, so a leaf's roots never depend on the visiting order.
"""
import numpy as np
import pytest

import spatial_query_b200 as sq
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu

FIELD = """// Implicit blobs (tests/field.rs:45-150): prim = centre[3], r0, amp, freq.
// field(p) = |p - c|^2 - r0^2 + amp (sin(f dx) + sin(f dy) + sin(f dz)).
constexpr float kStep = 0.05f;
constexpr float kHorizon = 500.f;  // the march always spans [0, 500]: the roots never depend on the limit

__device__ float blob_field(const float* b, const float* p) {
  float d[3];
  for (int i = 0; i < 3; ++i) d[i] = fsub(p[i], b[i]);
  const float base = fsub(pdot<3>(d, d), fmul(b[3], b[3]));
  const float bump = fmul(b[4], fadd(fadd(sinf(fmul(b[5], d[0])), sinf(fmul(b[5], d[1]))), sinf(fmul(b[5], d[2]))));
  return fadd(base, bump);
}

__device__ void blob_gradient(const float* b, const float* p, float* g) {
  const float k = fmul(b[4], b[5]);
  for (int i = 0; i < 3; ++i) {
    const float d = fsub(p[i], b[i]);
    g[i] = fadd(fmul(2.f, d), fmul(k, cosf(fmul(b[5], d))));
  }
}

template <class Emit>
__device__ void sq_narrow_crossings(const float* b, uint32_t leaf, const float* ro, const float* rd, float max_toi,
                                    Emit& emit) {
  float p[3];
  float t = 0.f;
  ray_at<3>(ro, rd, t, p);
  float f_prev = blob_field(b, p);
  while (t < kHorizon) {
    const float t_next = fminf(fadd(t, kStep), kHorizon);
    ray_at<3>(ro, rd, t_next, p);
    const float f_next = blob_field(b, p);
    if (f_prev != 0.f && ((f_prev < 0.f) != (f_next < 0.f))) {
      float a = t, c = t_next, fa = f_prev;
      for (int i = 0; i < 40; ++i) {
        const float m = fmul(0.5f, fadd(a, c));
        ray_at<3>(ro, rd, m, p);
        const float fm = blob_field(b, p);
        if ((fa < 0.f) != (fm < 0.f)) {
          c = m;
        } else {
          a = m;
          fa = fm;
        }
      }
      const float root = fmul(0.5f, fadd(a, c));
      if (root > max_toi) return;
      float n[3];
      ray_at<3>(ro, rd, root, p);
      blob_gradient(b, p, n);
      normalize_or_zero<3>(n);
      emit(root, n);
    }
    if (t_next >= kHorizon) break;
    t = t_next;
    f_prev = f_next;
  }
}

__device__ bool sq_narrow(const float* b, uint32_t leaf, const float* ro, const float* rd, float max_toi, float* toi,
                          float* normal) {
  bool found = false;
  auto first = [&](float t, const float* n) {
    if (!found) {
      found = true;
      *toi = t;
      for (int i = 0; i < 3; ++i) normal[i] = n[i];
    }
  };
  sq_narrow_crossings(b, leaf, ro, rd, max_toi, first);
  return found;
}
"""


@pytest.fixture(scope="module")
def ctx():
    c = sq.Context(0)
    yield c
    c.set_order(sq.ORDER_NEAR_FIRST)
    c.close()


def blob_aabbs(prims):
    h = (prims[:, 3] + prims[:, 4] + 1.0)[:, None]  # Blob::half_extent
    return np.ascontiguousarray(np.concatenate([prims[:, :3] - h, prims[:, :3] + h], axis=1), dtype=np.float32)


def random_blobs(rng, n):
    c = rng.range(-40.0, 40.0, (n, 3))
    r0 = rng.range(2.0, 5.0, (n, 1))
    amp = rng.range(0.0, 2.0, (n, 1))
    freq = rng.range(0.5, 1.5, (n, 1))
    return np.ascontiguousarray(np.concatenate([c, r0, amp, freq], axis=1), dtype=np.float32)


def flat_tree(aabbs):
    n = aabbs.shape[0]
    b = np.concatenate([aabbs[:, :3].min(axis=0), aabbs[:, 3:].max(axis=0)])[None, :].astype(np.float32)
    z = np.zeros(1, np.uint32)
    return sq.HostBvh(3, b, z, z.copy(), np.array([n], np.uint32), np.arange(n, dtype=np.uint32))


def same_lists(a, b, label):
    assert np.array_equal(a.count, b.count), f"{label}: counts differ"
    k = a.leaf.shape[1]
    mask = np.arange(k)[None, :] < np.minimum(a.count, k)[:, None]
    assert np.array_equal(a.leaf[mask], b.leaf[mask]), f"{label}: leaves differ"
    assert np.array_equal(a.toi[mask].view(np.uint32), b.toi[mask].view(np.uint32)), f"{label}: toi differ"


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_field_tree_matches_naive(ctx, seed):
    rng = scenes.Rng(0xF1E1D000 + seed)
    prims = random_blobs(rng, 40)
    aabbs = blob_aabbs(prims)
    n = 8192
    org = rng.range(-60.0, 60.0, (n, 3))
    d = scenes.normalize_rows(rng.range(-1.0, 1.0, (n, 3)).astype(np.float32))
    rays = np.ascontiguousarray(np.concatenate([org, d], axis=1), dtype=np.float32)
    tree = sq.DeviceBvh.custom(ctx, sq.HostBvh.build_from_aabbs(3, aabbs), prims, aabbs, FIELD)
    naive = sq.DeviceBvh.custom(ctx, flat_tree(aabbs), prims, aabbs, FIELD)
    ctx.set_order(sq.ORDER_REFERENCE)
    ref = naive.raycast_nearest(rays, 500.0)
    assert (ref.leaf != sq.NO_HIT).mean() > 0.03  # 40 sparse blobs: a few hundred rays hit
    for order in (sq.ORDER_REFERENCE, sq.ORDER_NEAR_FIRST):
        ctx.set_order(order)
        got = tree.raycast_nearest(rays, 500.0)
        assert np.array_equal(ref.leaf, got.leaf), f"order {order}: nearest leaf"
        assert np.array_equal(ref.toi.view(np.uint32), got.toi.view(np.uint32)), f"order {order}: nearest toi"
    ctx.set_order(sq.ORDER_NEAR_FIRST)
    c_ref = naive.raycast_crossings(rays, 500.0, k=16)
    c_got = tree.raycast_crossings(rays, 500.0, k=16)
    assert (c_ref.count >= 2).sum() > 100  # entries and exits
    same_lists(c_ref, c_got, "crossings")
    tree.close()
    naive.close()


def test_field_march_converges(ctx):
    prims = np.array([[20.0, 0.0, 0.0, 3.0, 0.0, 1.0]], np.float32)  # a pure sphere, radius 3
    aabbs = blob_aabbs(prims)
    g = sq.DeviceBvh.custom(ctx, sq.HostBvh.build_from_aabbs(3, aabbs), prims, aabbs, FIELD)
    ray = np.array([[0, 0, 0, 1, 0, 0]], np.float32)
    h = g.raycast_nearest(ray, 100.0, outputs=("normal",))
    assert h.leaf[0] == 0 and abs(float(h.toi[0]) - 17.0) < 1e-2
    assert float(h.normal[0] @ ray[0, 3:]) < 0.0 and abs(float(h.normal[0, 0]) + 1.0) < 1e-2
    c = g.raycast_crossings(ray, 100.0, k=4)
    assert c.count[0] == 2
    assert abs(float(c.toi[0, 0]) - 17.0) < 1e-2 and abs(float(c.toi[0, 1]) - 23.0) < 1e-2
    g.close()


def test_field_misses_and_empty(ctx):
    prims = np.array([[0.0, 0.0, 0.0, 2.0, 0.5, 1.0]], np.float32)
    aabbs = blob_aabbs(prims)
    g = sq.DeviceBvh.custom(ctx, sq.HostBvh.build_from_aabbs(3, aabbs), prims, aabbs, FIELD)
    miss = np.array([[-10, 0, 50, 1, 0, 0]], np.float32)
    assert g.raycast_nearest(miss, 100.0).leaf[0] == sq.NO_HIT
    g.close()
    empty = np.zeros((0, 6), np.float32)
    e = sq.DeviceBvh.custom(ctx, sq.HostBvh.build_from_aabbs(3, empty), empty, empty, FIELD)
    ray = np.array([[0, 0, 0, 1, 0, 0]], np.float32)
    assert e.raycast_nearest(ray, 100.0).leaf[0] == sq.NO_HIT
    assert e.raycast_crossings(ray, 100.0, k=4).count[0] == 0
    e.close()
