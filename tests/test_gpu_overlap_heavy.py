"""Overlap regions heavier than the per-thread visit budget, and regions
with more results than the count pass keeps, are finished by the
block-per-region kernel (its count pass stores the leaves it finds, its fill
pass copies them or walks again); the CSR result (offsets, and each
region's leaves ascending) must equal the oracle's whatever mix of light
and heavy regions a batch holds: regions covering most of a box scene among
small ones, with a layer filter, in 3 and 6 dimensions, and through the
host-buffer and device-pointer calls."""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_csr
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sq.Context(0)
    yield c
    c.close()


def regions_mix(rng, dim, n_small, n_big, lo, hi):
    c = rng.range(lo, hi, (n_small, dim))
    h = rng.range(0.5, 3.0, (n_small, dim))
    small = np.concatenate([c - h, c + h], axis=1)
    cb = rng.range(lo / 2, hi / 2, (n_big, dim))
    hb = rng.range((hi - lo) / 4, (hi - lo) / 2, (n_big, dim))
    big = np.concatenate([cb - hb, cb + hb], axis=1)
    r = np.concatenate([small, big])
    return np.ascontiguousarray(r[np.random.default_rng(7).permutation(len(r))], dtype=np.float32)


def test_heavy_regions_3d(ctx):
    rng = scenes.Rng(300)
    s = scenes.boxes_scene(seed=301, n_boxes=40000, n_rays=1)
    n = s["prims"].shape[0]
    layers = (np.arange(n) % 5 + 1).astype(np.uint64)
    geom = sq.Geometry("boxes", 3, s["prims"], layers=layers)
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    regions = regions_mix(rng, 3, 20000, 24, -100.0, 100.0)
    o = O.Scene("boxes", 3, s["prims"], layers=layers)
    ref = o.overlap(regions)
    counts = np.diff(ref[0].astype(np.int64))
    assert counts.max() > 5000  # some regions are far over the visit budget
    assert_same_csr(ref, scene.overlap(regions), label="heavy 3d")
    assert_same_csr(o.overlap(regions, mask=0b10110, exclude=77), scene.overlap(regions, mask=0b10110, exclude=77),
                    label="heavy 3d filtered")
    scene.close()


def test_heavy_regions_6d_device_call(ctx):
    import torch
    s = scenes.mixture_scene(seed=302, n_boxes=200000, n_rays=1, n_regions=50000)
    geom = sq.Geometry("boxes", 6, s["prims"])
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    regions = np.ascontiguousarray(np.concatenate([s["regions"], np.tile([[0.2] * 6 + [0.8] * 6], (8, 1))]),
                                   dtype=np.float32)
    ref = O.Scene("boxes", 6, s["prims"]).overlap(regions)
    n = regions.shape[0]
    dev = torch.device("cuda", 0)
    d_reg = torch.from_numpy(regions).to(dev)
    offs = torch.empty(n + 1, dtype=torch.int64, device=dev)
    total = scene.overlap_d(d_reg, n, offs, None, 0)
    leaves = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
    assert scene.overlap_d(d_reg, n, offs, leaves, total) == total
    got = (offs.cpu().numpy().view(np.uint64), leaves[:total].cpu().numpy().view(np.uint32))
    assert_same_csr(ref, got, label="heavy 6d")
    assert np.diff(ref[0].astype(np.int64)).max() > 1000
    scene.close()
