"""The CUDA path against the committed golden fixtures (tests/golden/*.npz,
the oracle's answers on small seeded cases of every workload): nearest leaf,
toi and normal bit for bit, bounded all-hits lists, CSR overlaps, and the
two-level scene's rays, casts and regions. No oracle runs here: the answers
come from the fixtures."""
import os
import sys

import numpy as np
import pytest

import spatial_query_b200 as sq

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import cases  # noqa: E402

pytestmark = pytest.mark.gpu
NO_HIT = 0xFFFFFFFF
CASES = cases.all_cases()


@pytest.fixture(scope="module")
def ctx():
    c = sq.Context(0)
    yield c
    c.close()


def f32bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", sorted(n for n in CASES if n != "tlas_mesh"))
def test_one_level_case(ctx, name):
    c = CASES[name]
    z = np.load(cases.fixture_path(name))
    assert str(z["inputs_digest"]) == cases.inputs_digest(name, c)
    geom = sq.Geometry(c["kind"], c["dim"], c["prims"])
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    h = scene.raycast_nearest(c["rays"], c["max_toi"], outputs=("normal",))
    assert np.array_equal(h.leaf, z["leaf"])
    hit = z["leaf"] != NO_HIT
    assert np.array_equal(f32bits(h.toi)[hit], z["toi"][hit])
    assert np.array_equal(f32bits(h.normal)[hit], z["normal"][hit])
    if "all_k" in c:
        k = c["all_k"]
        a = scene.raycast_all(c["rays"][:1024], c["max_toi"], k=k, outputs=())
        assert np.array_equal(a.count, z["all_count"])
        m = np.arange(k)[None, :] < np.minimum(z["all_count"], k)[:, None]
        assert np.array_equal(a.leaf[m], z["all_leaf"][m])
        assert np.array_equal(f32bits(a.toi)[m], z["all_toi"][m])
    if "regions" in c:
        off, lv = scene.overlap(c["regions"])
        assert np.array_equal(off, z["overlap_offsets"])
        assert np.array_equal(lv, z["overlap_leaves"])
    scene.close()


def test_two_level_case(ctx):
    c = CASES["tlas_mesh"]
    z = np.load(cases.fixture_path("tlas_mesh"))
    assert str(z["inputs_digest"]) == cases.inputs_digest("tlas_mesh", c)
    blas = sq.BlasSet(ctx, c["meshes"])
    g = sq.DeviceTlas(ctx, "mesh", 3, c["rot"], c["trans"], c["scale"], blas_id=c["blas_id"], blas=blas)
    h = g.raycast_nearest(c["rays"], c["max_toi"])
    assert np.array_equal(h.leaf, z["ray_leaf"])
    hit = z["ray_leaf"] != NO_HIT
    assert np.array_equal(f32bits(h.toi)[hit], z["ray_toi"][hit])
    assert np.array_equal(f32bits(h.normal)[hit], z["ray_normal"][hit])
    h = g.shapecast_nearest(c["casts"], c["cast_len"])
    assert np.array_equal(h.leaf, z["cast_leaf"])
    hit = z["cast_leaf"] != NO_HIT
    assert np.array_equal(f32bits(h.toi)[hit], z["cast_toi"][hit])
    off, lv = g.overlap(c["regions"])
    assert np.array_equal(off, z["overlap_offsets"])
    assert np.array_equal(lv, z["overlap_leaves"])
