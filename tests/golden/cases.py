"""Golden cases: small seeded instances of each workload's scenes and
queries, shared by the fixture generator (make_golden.py) and the tests.

Inputs are regenerated from their seeds (spatial_query_b200.scenes); a
fixture stores the oracle's answers plus a digest of the inputs, so a test
can tell a changed answer from a changed scene generator."""
from __future__ import annotations

import hashlib
import os

import numpy as np

from spatial_query_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def balls_scene(kind: str) -> dict:
    rng = scenes.Rng(91)
    n = 3000
    prims = np.concatenate([rng.range(-80.0, 80.0, (n, 3)), rng.range(0.2, 2.5, (n, 1))], axis=1).astype(np.float32)
    o = rng.range(-120.0, 120.0, (4096, 3))
    d = scenes.normalize_rows(rng.range(-60.0, 60.0, (4096, 3)) - o)
    rays = np.ascontiguousarray(np.concatenate([o, d], axis=1), dtype=np.float32)
    return dict(kind=kind, dim=3, prims=prims, rays=rays, max_toi=500.0)


def one_level_cases() -> dict:
    """name -> scene dict with kind, dim, prims, rays, max_toi (+ regions, all_k)."""
    c = {}
    s = scenes.boxes_scene(seed=0, n_rays=4096)
    c["boxes3"] = dict(kind="boxes", dim=3, prims=s["prims"], rays=s["rays"], max_toi=s["max_toi"])
    s = scenes.terrain_scene(seed=1, nx=64, ny=32, n_coherent=2048, n_incoherent=2048)
    c["terrain"] = dict(kind="tris", dim=3, prims=s["prims"], rays=s["rays"], max_toi=s["max_toi"], all_k=8)
    c["balls"] = balls_scene("balls")
    c["balls_near"] = balls_scene("balls_near")
    # D = 6: the boxes scene with its boxes widened 6x about their centres
    # (rays in six dimensions rarely meet the narrow ones), and regions of
    # half-extent U[5, 25] about centres U[-100, 100]^6
    s = scenes.boxes_scene(seed=66, n_boxes=10000, n_rays=4096, dim=6)
    p = s["prims"]
    ctr, half = (p[:, :6] + p[:, 6:]) * np.float32(0.5), (p[:, 6:] - p[:, :6]) * np.float32(0.5)
    wide = np.ascontiguousarray(np.concatenate([ctr - 6 * half, ctr + 6 * half], axis=1), dtype=np.float32)
    rng = scenes.Rng(67)
    rc, rh = rng.range(-100.0, 100.0, (512, 6)), rng.range(5.0, 25.0, (512, 6))
    regions = np.ascontiguousarray(np.concatenate([rc - rh, rc + rh], axis=1), dtype=np.float32)
    c["boxes6"] = dict(kind="boxes", dim=6, prims=wide, rays=s["rays"], max_toi=s["max_toi"], regions=regions)
    return c


def instanced_case() -> dict:
    return scenes.instanced_scene(seed=7, n_instances=64, n_blas=2, n_rays=4096, n_casts=256, n_regions=256,
                                  n_frames=1, blas_lo=500, blas_hi=2000)


def inputs_digest(name: str, c: dict) -> str:
    if name == "tlas_mesh":
        return digest(c["blas_tris"], c["blas_offsets"], c["rot"], c["trans"], c["scale"], c["blas_id"], c["rays"],
                      c["casts"], c["cast_len"], c["regions"])
    return digest(c["prims"], c["rays"], c.get("regions", np.zeros(0)))


def oracle_answers(O, name: str, c: dict) -> dict:
    """The oracle's answers for case `name` as flat arrays (floats as bits)."""
    bits = lambda a: np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    out = {}
    if name == "tlas_mesh":
        sc = O.TlasScene("mesh", 3, c["rot"], c["trans"], c["scale"], blas_id=c["blas_id"],
                         blas=O.BlasSet(c["blas_offsets"], c["blas_tris"]))
        h = sc.nearest(c["rays"], c["max_toi"])
        out.update(ray_leaf=h.leaf, ray_toi=bits(h.toi), ray_normal=bits(h.normal))
        h = sc.shapecast_nearest(c["casts"], c["cast_len"])
        out.update(cast_leaf=h.leaf, cast_toi=bits(h.toi))
        off, lv = sc.overlap(c["regions"])
        out.update(overlap_offsets=off, overlap_leaves=lv)
        return out
    sc = O.Scene(c["kind"], c["dim"], c["prims"])
    h = sc.nearest(c["rays"], c["max_toi"])
    out.update(leaf=h.leaf, toi=bits(h.toi), normal=bits(h.normal))
    if "all_k" in c:
        a = sc.all(c["rays"][:1024], c["max_toi"], k=c["all_k"])
        out.update(all_count=a.count, all_leaf=a.leaf, all_toi=bits(a.toi))
    if "regions" in c:
        off, lv = sc.overlap(c["regions"])
        out.update(overlap_offsets=off, overlap_leaves=lv)
    return out


def all_cases() -> dict:
    c = one_level_cases()
    c["tlas_mesh"] = instanced_case()
    return c


def fixture_path(name: str) -> str:
    return os.path.join(HERE, f"{name}.npz")
