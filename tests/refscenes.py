"""Scenes of the spatial-query test-suite, regenerated draw-for-draw.

Each function replays the SplitMix64 draw order of one reference test file so
the oracle and the CUDA path see the same balls, boxes and rays the crate's
own tests use (file:line cited per function).
"""
from __future__ import annotations

import numpy as np

from spatial_query_b200.scenes import Rng, normalize_rows

TAU32 = np.float32(6.2831855)


def point(rng: Rng, dim: int, lo: float, hi: float) -> np.ndarray:
    return rng.range(lo, hi, dim)


def ray_new(origin: np.ndarray, d: np.ndarray) -> np.ndarray:
    """Ray::new: origin, normalize_or_zero(dir)."""
    return np.concatenate([origin.astype(np.float32), normalize_rows(d[None, :].astype(np.float32))[0]])


def balls_prims(centers: np.ndarray, radii: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.concatenate([centers, radii[:, None]], axis=1), dtype=np.float32)


def random_balls(rng: Rng, n: int, dim: int, lo=-50.0, hi=50.0, rlo=0.5, rhi=4.0) -> np.ndarray:
    """tests/differential.rs:85-89: n centres, then n radii."""
    centers = np.stack([point(rng, dim, lo, hi) for _ in range(n)]) if n else np.zeros((0, dim), np.float32)
    radii = rng.range(rlo, rhi, n) if n else np.zeros(0, np.float32)
    return balls_prims(centers, radii)


def differential_cases(dim: int, seed: int, n_balls: int, lo: float, hi: float, count: int = 200):
    """tests/differential.rs:120-162: (prims, ray) per iteration, zero-dir skipped."""
    rng = Rng(seed)
    for _ in range(count):
        prims = random_balls(rng, n_balls, dim)
        o = point(rng, dim, lo, hi)
        d = point(rng, dim, -1.0, 1.0)
        ray = ray_new(o, d)
        if not np.any(ray[dim:]):
            continue
        yield prims, ray


def conformance_balls(n: int, seed: int) -> np.ndarray:
    """tests/conformance.rs:246-259: per ball x, y, z in [-20, 20), radius [0.3, 1.4)."""
    rng = Rng(seed)
    raw = rng.take(4 * n).reshape(n, 4) if n else np.zeros((0, 4), np.uint64)
    from spatial_query_b200.scenes import f32_range
    c = f32_range(raw[:, :3], -20.0, 20.0)
    r = f32_range(raw[:, 3], 0.3, 1.4)
    return balls_prims(c, r)


def conformance_rays(n: int, seed: int, lo=-30.0, hi=30.0, tlo=-8.0, thi=8.0) -> np.ndarray:
    """tests/conformance.rs:296-313: origin in [-30,30)^3, toward a target in [-8,8)^3."""
    rng = Rng(seed)
    out = []
    for _ in range(n):
        o = rng.range(lo, hi, 3)
        t = rng.range(tlo, thi, 3)
        out.append(ray_new(o, t - o))
    return np.stack(out) if out else np.zeros((0, 6), np.float32)


def plane_rotation(dim: int, a: int, b: int, angle: np.float32) -> np.ndarray:
    r = np.eye(dim, dtype=np.float32)
    s = np.float32(np.sin(np.float32(angle)))
    c = np.float32(np.cos(np.float32(angle)))
    r[a, a] = c
    r[a, b] = -s
    r[b, a] = s
    r[b, b] = c
    return r


def random_oriented_boxes(rng: Rng, n: int, dim: int):
    """tests/two_level.rs:115-131: per instance t, plane (a, b), angle, halves."""
    rots, trans, halves = [], [], []
    for _ in range(n):
        t = point(rng, dim, -40.0, 40.0)
        a = rng.next_u64() % dim
        b = rng.next_u64() % dim
        if b == a:
            b = (b + 1) % dim
        ang = rng.range(0.0, float(TAU32), 1)[0]
        rots.append(plane_rotation(dim, a, b, ang))
        trans.append(t)
        halves.append(np.maximum(point(rng, dim, 0.5, 2.5), np.float32(0.5)))
    return np.stack(rots), np.stack(trans), np.stack(halves)


def line_balls(n: int, radius: float) -> np.ndarray:
    """tests/stats.rs:14-21, result_identity.rs:60-66: centres (2(i+1), 0, 0)."""
    c = np.zeros((n, 3), np.float32)
    c[:, 0] = 2.0 * (np.arange(n, dtype=np.float32) + np.float32(1.0))
    return balls_prims(c, np.full(n, radius, np.float32))


def axis_ray() -> np.ndarray:
    return np.array([0, 0, 0, 1, 0, 0], np.float32)


def cube_mesh(size: float) -> np.ndarray:
    """A cube of edge `size` centred on the origin, two triangles per face
    (tris[12, 9]): the mesh of viewport-lib's primitives::cube(size) that the
    known-answer tests of crates/viewport-lib-query/src/lib.rs:338-431 put
    under their instances (that crate is absent, so its triangulation is
    restated here; the tests' answers depend only on the cube's faces)."""
    h = np.float32(size) * np.float32(0.5)
    tris = []
    for axis in range(3):
        u, v = (axis + 1) % 3, (axis + 2) % 3
        for side in (-h, h):
            quad = []
            for a, b in ((-h, -h), (h, -h), (h, h), (-h, h)):
                p = [np.float32(0)] * 3
                p[axis], p[u], p[v] = side, a, b
                quad.append(p)
            tris.append(quad[0] + quad[1] + quad[2])
            tris.append(quad[0] + quad[2] + quad[3])
    return np.asarray(tris, dtype=np.float32)


def mesh_instances(trans, scale=None):
    """(rot, trans, scale, blas_id) of identity-rotation instances of one mesh
    (Mat4::from_translation / from_scale_rotation_translation with an identity
    quaternion, lib.rs:357, 381-382, 396, 410-418)."""
    trans = np.asarray(trans, dtype=np.float32).reshape(-1, 3)
    n = trans.shape[0]
    rot = np.repeat(np.eye(3, dtype=np.float32)[None], n, axis=0)
    s = np.ones(n, np.float32) if scale is None else np.asarray(scale, dtype=np.float32).reshape(n)
    return rot, trans, s, np.zeros(n, np.uint32)
