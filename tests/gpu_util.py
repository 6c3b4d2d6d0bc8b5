"""Helpers for the GPU parity tests: build a scene once for both the oracle and
the CUDA path, and compare their results field by field (bit-exact)."""
from __future__ import annotations

import numpy as np

import oracle as O
import spatial_query_b200 as sq

_CTX = None


def ctx() -> sq.Context:
    global _CTX
    if _CTX is None:
        _CTX = sq.Context(0)
    return _CTX


def pair(kind: str, dim: int, prims, layers=None, sub=None):
    """(oracle scene, device scene) over the same leaves and the same tree."""
    o = O.Scene(kind, dim, prims, layers=layers, sub=sub)
    g = sq.Geometry(kind, dim, prims, layers=layers, sub_objects=sub)
    t = sq.HostBvh.build(g)
    return o, sq.DeviceBvh(ctx(), t, g)


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def assert_same_nearest(o: O.Hits, h: sq.Hits, normals=True, points=True, sub=True, label=""):
    bad = np.nonzero(o.leaf != h.leaf)[0]
    assert bad.size == 0, f"{label}: leaf differs on {bad.size} queries, first {bad[:5]} " \
                          f"oracle {o.leaf[bad[:5]]} gpu {h.leaf[bad[:5]]}"
    hit = o.leaf != O.NO_HIT
    tb = np.nonzero(bits(o.toi[hit]) != bits(h.toi[hit]))[0]
    assert tb.size == 0, f"{label}: toi differs on {tb.size} hits"
    if normals and h.normal is not None:
        assert np.array_equal(bits(o.normal[hit]), bits(h.normal[hit])), f"{label}: normals differ"
    if points and h.point is not None:
        assert np.array_equal(bits(o.point[hit]), bits(h.point[hit])), f"{label}: points differ"
    if sub and h.sub_object is not None:
        assert np.array_equal(o.sub[hit], h.sub_object[hit]), f"{label}: sub-objects differ"


def assert_same_lists(o: O.HitLists, h: sq.HitLists, normals=True, sub=True, label=""):
    assert np.array_equal(o.count, h.count), f"{label}: counts differ on {(o.count != h.count).sum()} queries"
    k = o.leaf.shape[1]
    m = np.minimum(o.count, k)
    mask = np.arange(k)[None, :] < m[:, None]
    assert np.array_equal(o.leaf[mask], h.leaf[mask]), f"{label}: list leaves differ"
    assert np.array_equal(bits(o.toi[mask]), bits(h.toi[mask])), f"{label}: list toi differ"
    if normals and h.normal is not None:
        assert np.array_equal(bits(o.normal[mask]), bits(h.normal[mask])), f"{label}: list normals differ"
    if sub and h.sub_object is not None:
        assert np.array_equal(o.sub[mask], h.sub_object[mask]), f"{label}: list sub-objects differ"


def assert_same_csr(a, b, label=""):
    assert np.array_equal(a[0], b[0]), f"{label}: overlap offsets differ"
    assert np.array_equal(a[1], b[1]), f"{label}: overlap leaves differ"
