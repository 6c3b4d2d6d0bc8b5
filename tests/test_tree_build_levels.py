"""The device tree build's method (sq_tree_build_d, tree_build_gpu.cu),
restated level by level in numpy on the CPU, gives the host build's arrays
(sq_tree_build, the crate's recursive tree::build, accel/tree.rs:112-163):

* per level, each segment's node box and centroid box, leaf or split by the
  first longest centroid axis (split at start + count / 2);
* one stable sort of the WHOLE primitive order per level on the keys
  (segment start << 32 | total_cmp key of the split axis), every position
  outside a split segment keyed (position << 32), is each node's own stable
  sort, with ties kept in the order the parent's sort left them;
* nodes numbered in level order, then renumbered in preorder from subtree
  sizes and left-subtree offsets.

This pins the composite-key argument on the CPU (ties, coincident
centroids, signed zeros, several dimensions); the GPU tests compare the
device build itself with the host build."""
import numpy as np
import pytest

import spatial_query_b200 as sq
from spatial_query_b200 import scenes

EPS = np.float32(1.1920928955078125e-7)


def total_ukey(x: np.ndarray) -> np.ndarray:
    b = x.astype(np.float32).view(np.uint32)
    return np.where(b & 0x80000000, ~b, b | 0x80000000).astype(np.uint32)


def level_build(dim: int, aabbs: np.ndarray):
    n = aabbs.shape[0]
    lo, hi = aabbs[:, :dim], aabbs[:, dim:]
    cen = ((lo + hi) * np.float32(0.5)).astype(np.float32)
    keys = [total_ukey(cen[:, k]).astype(np.uint64) for k in range(dim)]
    idx = np.arange(n, dtype=np.int64)
    nodes = [None]  # level-order id -> (s, e, a, b, bounds)
    segs = [(0, n, 0)]
    while segs:
        ck = np.arange(n, dtype=np.uint64) << np.uint64(32)
        nxt = []
        for s, e, nid in segs:
            sub = idx[s:e]
            box = np.concatenate([lo[sub].min(axis=0), hi[sub].max(axis=0)]).astype(np.float32)
            clo, chi = cen[sub].min(axis=0), cen[sub].max(axis=0)
            a = b = None
            if e - s > 4:
                ext = (chi - clo).astype(np.float32)
                ax = 0
                for k in range(1, dim):
                    if ext[k] > ext[ax]:
                        ax = k
                if ext[ax] > EPS:
                    mid = s + (e - s) // 2
                    a, b = len(nodes), len(nodes) + 1
                    nodes += [None, None]
                    nxt += [(s, mid, a), (mid, e, b)]
                    ck[s:e] = (np.uint64(s) << np.uint64(32)) | keys[ax][sub]
            nodes[nid] = (s, e, a, b, box)
        idx = idx[np.argsort(ck, kind="stable")]
        segs = nxt
    # level order -> preorder
    m = len(nodes)
    size = np.ones(m, np.int64)
    for i in range(m - 1, -1, -1):  # children have larger level-order ids
        s, e, a, b, _ = nodes[i]
        if a is not None:
            size[i] = 1 + size[a] + size[b]
    pre = np.zeros(m, np.int64)
    for i in range(m):
        s, e, a, b, _ = nodes[i]
        if a is not None:
            pre[a] = pre[i] + 1
            pre[b] = pre[i] + 1 + size[a]
    bounds = np.zeros((m, 2 * dim), np.float32)
    ca, cb, pc = np.zeros(m, np.uint32), np.zeros(m, np.uint32), np.zeros(m, np.uint32)
    for i in range(m):
        s, e, a, b, box = nodes[i]
        j = pre[i]
        bounds[j] = box
        if a is None:
            ca[j], cb[j], pc[j] = s, 0, e - s
        else:
            ca[j], cb[j], pc[j] = pre[a], pre[b], 0
    return bounds, ca, cb, pc, idx.astype(np.uint32)


def check(dim, aabbs):
    aabbs = np.ascontiguousarray(aabbs, dtype=np.float32)
    h = sq.HostBvh.build_from_aabbs(dim, aabbs)
    bounds, ca, cb, pc, pi = level_build(dim, aabbs)
    assert h.node_count == len(ca)
    assert np.array_equal(h.child_a, ca) and np.array_equal(h.child_b, cb) and np.array_equal(h.prim_count, pc)
    assert np.array_equal(h.prim_indices, pi)
    assert np.array_equal(h.bounds, bounds)  # as numbers: a zero bound may differ in sign
    return h


def boxes(rng, n, dim):
    c = rng.range(-100.0, 100.0, (n, dim))
    e = rng.range(0.25, 2.0, (n, dim))
    return np.concatenate([c - e, c + e], axis=1)


@pytest.mark.parametrize("n", [1, 4, 5, 9, 33, 1000, 6000])
def test_counts(n):
    check(3, boxes(scenes.Rng(300 + n), n, 3))


@pytest.mark.parametrize("dim", [2, 4, 6])
def test_dimensions(dim):
    check(dim, boxes(scenes.Rng(310 + dim), 4000, dim))


def test_ties_keep_parent_order():
    rng = scenes.Rng(320)
    c = np.floor(rng.range(0.0, 6.0, (3000, 3))).astype(np.float32)
    e = rng.range(0.1, 0.4, (3000, 3)).astype(np.float32)
    check(3, np.concatenate([c - e, c + e], axis=1))


def test_coincident_and_signed_zero_centroids():
    same = np.tile(np.array([[1.0, 2.0, 3.0, 2.0, 3.0, 4.0]], np.float32), (50, 1))
    h = check(3, np.concatenate([same, boxes(scenes.Rng(321), 40, 3), same[:13]]))
    assert (h.prim_count > 4).any()
    z = np.zeros((64, 6), np.float32)
    z[:, 0] = np.where(np.arange(64) % 2 == 0, -0.0, 0.0)
    z[:, 3] = z[:, 0]
    z[:, 2] = (np.arange(64) % 3) * np.float32(0.1)
    z[:, 5] = z[:, 2] + np.float32(0.1)
    z[::5, 0] = -1.0
    check(3, z)


def test_terrain_patch():
    s = scenes.terrain_scene(seed=5, nx=64, ny=32, n_coherent=1, n_incoherent=1)
    check(3, sq.Geometry("tris", 3, s["prims"]).world_aabbs())
