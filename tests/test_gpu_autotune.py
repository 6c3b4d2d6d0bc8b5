"""The nearest-ray autotuner (sq_autotune_nearest_d): it times every order x
node-layout x blocks-per-SM candidate, keeps the fastest in the context, and the tuned
context still returns the oracle's hits bit for bit."""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_nearest
from spatial_query_b200 import scenes

pytestmark = pytest.mark.gpu


def test_autotune_keeps_hits_exact():
    import torch
    s = scenes.terrain_scene(seed=5, nx=256, ny=128, n_coherent=32768, n_incoherent=32768)
    ctx = sq.Context(0)
    geom = sq.Geometry("tris", 3, s["prims"])
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    n = s["rays"].shape[0]
    d_rays = torch.from_numpy(s["rays"]).to(torch.device("cuda", 0))
    torch.cuda.synchronize()
    res = scene.autotune_nearest_d(d_rays, n, s["max_toi"], reps=2)
    # near-first over child-pair, four-wide and quantised four-wide records, the reference order: 8 grids each
    assert len(res["table"]) == 48
    assert {(e["order"], e["layout"]) for e in res["table"]} == {(0, 0), (0, 1), (0, 2), (0, 3), (0, 4), (1, 0)}
    assert all(e["ms"] > 0 for e in res["table"])
    assert res["best"]["ms"] == min(e["ms"] for e in res["table"])
    ref = O.Scene("tris", 3, s["prims"]).nearest(s["rays"], s["max_toi"])
    assert_same_nearest(ref, scene.raycast_nearest(s["rays"], s["max_toi"]), label="tuned nearest")
    scene.close()
    ctx.close()
