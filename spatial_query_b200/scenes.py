"""Seeded synthetic workloads for the batched-query path.

Every value comes from SplitMix64, the generator the spatial-query test-suite
uses (crates/spatial-query/tests/differential.rs:8-33): ``next_u64`` advances
the state by 0x9E3779B97F4A7C15 and mixes it; a float in ``[lo, hi)`` is
``lo + ((x >> 11) as f32 / 2^53) * (hi - lo)`` in f32 arithmetic. Because the
n-th output depends only on ``seed + n * golden``, a whole stream is produced
at once with numpy's wrapping uint64 arithmetic.

Normal deviates use Box-Muller in f64 on the same stream; trigonometry is
evaluated on the host in f64 and only the f32-rounded results are handed on.
Ray directions are normalised with the crate's exact f32 rule
(maths/point.rs:82-89, maths/ray.rs:18-23).

The scenes are the benchmark configurations of the path:

* ``boxes_scene``: D-dim axis-aligned boxes with rays from a sphere shell
  (10,000 boxes / 65,536 rays at D = 3).
* ``terrain_scene``: a 1024 x 512 height-field triangle soup (1,048,576
  triangles) with half coherent, half incoherent rays.
* ``instanced_scene``: 16 height-field meshes under 4,096 scaled, rotated
  instances, with rays, box casts and overlap regions.
* ``mixture_scene``: D = 6 boxes from a 64-component Gaussian mixture with
  rays and overlap regions.
"""
from __future__ import annotations

import math

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
F32_EPS = np.float32(1.1920928955078125e-7)


class Rng:
    """SplitMix64 stream; ``take(n)`` returns the next n outputs in order."""

    def __init__(self, seed: int):
        self.state = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)

    def take(self, n: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            steps = np.arange(1, n + 1, dtype=np.uint64)
            z = self.state + steps * GOLDEN
            self.state = self.state + np.uint64(n) * GOLDEN
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
            return z ^ (z >> np.uint64(31))

    def next_u64(self) -> int:
        return int(self.take(1)[0])

    def range(self, lo: float, hi: float, n: int | tuple = 1) -> np.ndarray:
        """f32 uniform in [lo, hi), the reference tests' ``Rng::range``."""
        shape = (n,) if isinstance(n, int) else tuple(n)
        cnt = int(np.prod(shape))
        return f32_range(self.take(cnt), lo, hi).reshape(shape)

    def unit64(self, n: int | tuple) -> np.ndarray:
        """f64 uniform in [0, 1) (53 random bits)."""
        shape = (n,) if isinstance(n, int) else tuple(n)
        cnt = int(np.prod(shape))
        return ((self.take(cnt) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)).reshape(shape)

    def normal64(self, n: int | tuple) -> np.ndarray:
        """f64 standard normal deviates (Box-Muller, cosine branch)."""
        shape = (n,) if isinstance(n, int) else tuple(n)
        cnt = int(np.prod(shape))
        u = self.unit64((cnt, 2))
        r = np.sqrt(-2.0 * np.log1p(-u[:, 0]))
        return (r * np.cos(2.0 * math.pi * u[:, 1])).reshape(shape)


def f32_range(raw: np.ndarray, lo: float, hi: float) -> np.ndarray:
    u = (raw >> np.uint64(11)).astype(np.float32) / np.float32(9007199254740992.0)
    lo32 = np.float32(lo)
    return lo32 + u * (np.float32(hi) - lo32)


def normalize_rows(v: np.ndarray) -> np.ndarray:
    """Point::normalize_or_zero on each row, in the crate's f32 op order."""
    v = np.ascontiguousarray(v, dtype=np.float32)
    acc = np.zeros(v.shape[0], dtype=np.float32)
    for i in range(v.shape[1]):
        acc = acc + v[:, i] * v[:, i]
    ln = np.sqrt(acc)
    ok = ln > F32_EPS
    inv = np.ones_like(ln)
    inv[ok] = np.float32(1.0) / ln[ok]
    out = v * inv[:, None]
    out[~ok] = 0.0
    return out


def rays_from(origins: np.ndarray, dirs: np.ndarray) -> np.ndarray:
    """Pack rays as origin[D], unit dir[D] (``Ray::new``)."""
    d = normalize_rows(dirs)
    return np.ascontiguousarray(np.concatenate([origins.astype(np.float32), d], axis=1))


def isotropic(rng: Rng, n: int, dim: int) -> np.ndarray:
    return rng.normal64((n, dim)).astype(np.float32)


# ---------------------------------------------------------------------------
# Axis-aligned boxes viewed from a sphere shell (D-generic).
# ---------------------------------------------------------------------------

def boxes_scene(seed: int = 0, n_boxes: int = 10_000, n_rays: int = 65_536, dim: int = 3) -> dict:
    """Boxes with centres U[-100,100]^D and half-extents U[0.25,2]^D; rays from
    a radius-200 sphere toward points U[-50,50]^D; t_max 1000."""
    rng = Rng(seed)
    raw = rng.take(n_boxes * 2 * dim).reshape(n_boxes, 2 * dim)
    c = f32_range(raw[:, :dim], -100.0, 100.0)
    h = f32_range(raw[:, dim:], 0.25, 2.0)
    prims = np.ascontiguousarray(np.concatenate([c - h, c + h], axis=1), dtype=np.float32)
    rays = sphere_rays(rng, n_rays, dim)
    return dict(name=f"boxes{dim}d", dim=dim, kind="boxes", prims=prims, rays=rays, max_toi=1000.0)


def sphere_rays(rng: Rng, n_rays: int, dim: int = 3) -> np.ndarray:
    """The boxes scene's rays: origins uniform on the radius-200 sphere,
    directions normalised toward points U[-50,50]^D."""
    sph = rng.normal64((n_rays, dim))
    sph /= np.linalg.norm(sph, axis=1, keepdims=True)
    origins = (200.0 * sph).astype(np.float32)
    targets = rng.range(-50.0, 50.0, (n_rays, dim))
    return rays_from(origins, targets - origins)


# ---------------------------------------------------------------------------
# Height-field triangle soups.
# ---------------------------------------------------------------------------

def heightfield(rng: Rng, nx: int, ny: int, cell: float, amp_lo: float, amp_hi: float, noise: float,
                lam_lo: float, lam_hi: float):
    """Vertices of an (nx+1) x (ny+1) grid, z = sum of 6 random-phase
    sinusoids plus N(0, noise). Returns (verts[ny+1, nx+1, 3] f32, waves)."""
    amp = amp_lo + (amp_hi - amp_lo) * rng.unit64(6)
    phase = 2.0 * math.pi * rng.unit64(6)
    lam = lam_lo * (lam_hi / lam_lo) ** rng.unit64(6)
    ang = 2.0 * math.pi * rng.unit64(6)
    kx = 2.0 * math.pi / lam * np.cos(ang)
    ky = 2.0 * math.pi / lam * np.sin(ang)
    xs = np.arange(nx + 1, dtype=np.float64) * cell
    ys = np.arange(ny + 1, dtype=np.float64) * cell
    X, Y = np.meshgrid(xs, ys)
    Z = np.zeros_like(X)
    for i in range(6):
        Z += amp[i] * np.sin(kx[i] * X + ky[i] * Y + phase[i])
    Z += noise * rng.normal64(X.shape)
    verts = np.stack([X, Y, Z], axis=-1).astype(np.float32)
    waves = dict(amp=amp, phase=phase, lam=lam, ang=ang)
    return verts, waves


def grid_triangles(verts: np.ndarray) -> np.ndarray:
    """Two triangles per cell, cell-major (row j outer, column i inner):
    (v00, v10, v11) and (v00, v11, v01). Returns tris[n, 9] f32."""
    v00 = verts[:-1, :-1]
    v10 = verts[:-1, 1:]
    v11 = verts[1:, 1:]
    v01 = verts[1:, :-1]
    t0 = np.concatenate([v00, v10, v11], axis=-1)
    t1 = np.concatenate([v00, v11, v01], axis=-1)
    tris = np.stack([t0, t1], axis=2).reshape(-1, 9)
    return np.ascontiguousarray(tris, dtype=np.float32)


def terrain_scene(seed: int = 1, nx: int = 1024, ny: int = 512, n_coherent: int | None = None,
                  n_incoherent: int | None = None) -> dict:
    """A 1024 x 512 height field over [0,1024] x [0,512] (2 triangles per cell,
    1,048,576 triangles at full size) with coherent rays from a camera grid at
    z = 200 jittered within 2 degrees of -z, then incoherent rays from uniform
    origins in the scene box with isotropic directions; t_max 2000."""
    rng = Rng(seed)
    verts, waves = heightfield(rng, nx, ny, 1.0, 1.0, 20.0, 0.5, 16.0, 512.0)
    tris = grid_triangles(verts)
    n_coh = nx * ny if n_coherent is None else n_coherent
    n_inc = nx * ny if n_incoherent is None else n_incoherent
    zmin, zmax = float(verts[..., 2].min()), float(verts[..., 2].max())
    rays = terrain_rays(rng, nx, ny, zmin, zmax, n_coh, n_inc)
    return dict(name="terrain", dim=3, kind="tris", prims=tris, rays=rays, max_toi=2000.0,
                n_coherent=n_coh, waves=waves, all_hits_k=16, zrange=(zmin, zmax), grid=(nx, ny))


def terrain_rays(rng: "Rng", nx: int, ny: int, zmin: float, zmax: float, n_coh: int, n_inc: int) -> np.ndarray:
    """The terrain workload's two ray kinds: coherent rays from the nx x ny
    camera grid at z = 200 jittered within 2 degrees of -z (cells sampled
    evenly, repeating when n_coh exceeds the grid), then incoherent rays from
    uniform origins in the scene box with isotropic directions."""
    cam = np.arange(n_coh, dtype=np.int64) * (nx * ny) // max(n_coh, 1)
    cx = (cam % nx).astype(np.float64) + 0.5
    cy = (cam // nx).astype(np.float64) + 0.5
    u = rng.unit64((n_coh, 2))
    theta = math.radians(2.0) * np.sqrt(u[:, 0])
    phi = 2.0 * math.pi * u[:, 1]
    d_coh = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), -np.cos(theta)], axis=1)
    o_coh = np.stack([cx, cy, np.full(n_coh, 200.0)], axis=1)
    lo = np.array([0.0, 0.0, zmin])
    hi = np.array([float(nx), float(ny), zmax])
    o_inc = lo + (hi - lo) * rng.unit64((n_inc, 3))
    d_inc = rng.normal64((n_inc, 3))
    origins = np.concatenate([o_coh, o_inc]).astype(np.float32)
    dirs = np.concatenate([d_coh, d_inc]).astype(np.float32)
    return rays_from(origins, dirs)


# ---------------------------------------------------------------------------
# Instanced two-level scene.
# ---------------------------------------------------------------------------

def quat_to_rot(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    r = np.empty((q.shape[0], 3, 3))
    r[:, 0, 0] = 1 - 2 * (y * y + z * z)
    r[:, 0, 1] = 2 * (x * y - w * z)
    r[:, 0, 2] = 2 * (x * z + w * y)
    r[:, 1, 0] = 2 * (x * y + w * z)
    r[:, 1, 1] = 1 - 2 * (x * x + z * z)
    r[:, 1, 2] = 2 * (y * z - w * x)
    r[:, 2, 0] = 2 * (x * z - w * y)
    r[:, 2, 1] = 2 * (y * z + w * x)
    r[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return r


def uniform_rotations(rng: Rng, n: int) -> np.ndarray:
    """Uniform random rotations (Shoemake's uniform quaternion), f32 row-major."""
    u = rng.unit64((n, 3))
    a = np.sqrt(1 - u[:, 0])
    b = np.sqrt(u[:, 0])
    q = np.stack([a * np.sin(2 * math.pi * u[:, 1]), a * np.cos(2 * math.pi * u[:, 1]),
                  b * np.sin(2 * math.pi * u[:, 2]), b * np.cos(2 * math.pi * u[:, 2])], axis=1)
    return quat_to_rot(q).astype(np.float32)


def blas_sizes(n_blas: int = 16, lo: int = 10_000, hi: int = 200_000) -> list[int]:
    """Triangle counts evenly spaced from lo to hi, each an even grid."""
    out = []
    for target in np.linspace(lo, hi, n_blas):
        cells = int(round(target / 2))
        ny = max(1, int(round(math.sqrt(cells / 2))))
        nx = max(1, cells // ny)
        out.append((nx, ny))
    return out


def instanced_scene(seed: int = 2, n_instances: int = 4096, n_blas: int = 16, n_rays: int = 1_000_000,
                    n_casts: int = 262_144, n_regions: int = 262_144, n_frames: int = 100,
                    blas_lo: int = 10_000, blas_hi: int = 200_000) -> dict:
    """16 height-field meshes of 10k..200k triangles spanning about 100 units,
    under n_instances instances (uniform rotation, scale U[0.5,2], translation
    U[-2000,2000]^3). Rays: half aimed at random instances, half isotropic,
    t_max 8000. Box casts: half-extent U[0.5,5], length U[0,200]. Regions:
    half-extent U[1,50]. Frames: per-instance N(0,1) translation steps."""
    rng = Rng(seed)
    meshes = []
    for (nx, ny) in blas_sizes(n_blas, blas_lo, blas_hi):
        cell = 100.0 / max(nx, ny)
        verts, _ = heightfield(rng, nx, ny, cell, 0.5, 6.0, 0.05, 8.0, 60.0)
        verts[..., 0] -= np.float32(nx * cell / 2)
        verts[..., 1] -= np.float32(ny * cell / 2)
        meshes.append(grid_triangles(verts))
    offsets = np.zeros(n_blas + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum([m.shape[0] for m in meshes])
    rot = uniform_rotations(rng, n_instances)
    scale = rng.range(0.5, 2.0, n_instances)
    trans = rng.range(-2000.0, 2000.0, (n_instances, 3))
    blas_id = (rng.take(n_instances) % np.uint64(n_blas)).astype(np.uint32)

    half = n_rays // 2
    o = rng.range(-2200.0, 2200.0, (n_rays, 3))
    pick = (rng.take(half) % np.uint64(n_instances)).astype(np.int64)
    aim = trans[pick] + rng.range(-30.0, 30.0, (half, 3))
    d = np.concatenate([aim - o[:half], isotropic(rng, n_rays - half, 3)])
    rays = rays_from(o, d)

    pick = (rng.take(n_casts) % np.uint64(n_instances)).astype(np.int64)
    co = trans[pick] + rng.range(-300.0, 300.0, (n_casts, 3))
    cd = normalize_rows(isotropic(rng, n_casts, 3))
    ch = rng.range(0.5, 5.0, (n_casts, 3))
    casts = np.ascontiguousarray(np.concatenate([co, cd, -ch, ch], axis=1), dtype=np.float32)
    cast_len = rng.range(0.0, 200.0, n_casts)

    pick = (rng.take(n_regions) % np.uint64(n_instances)).astype(np.int64)
    rc = trans[pick] + rng.range(-200.0, 200.0, (n_regions, 3))
    rh = rng.range(1.0, 50.0, (n_regions, 3))
    regions = np.ascontiguousarray(np.concatenate([rc - rh, rc + rh], axis=1), dtype=np.float32)

    steps = rng.normal64((n_frames, n_instances, 3)).astype(np.float32)
    return dict(name="instanced", dim=3, meshes=meshes, blas_offsets=offsets,
                blas_tris=np.ascontiguousarray(np.concatenate(meshes)), rot=rot, scale=scale, trans=trans,
                blas_id=blas_id, rays=rays, max_toi=8000.0, casts=casts, cast_len=cast_len, regions=regions,
                frame_steps=steps)


# ---------------------------------------------------------------------------
# High-dimensional Gaussian-mixture boxes.
# ---------------------------------------------------------------------------

def mixture_scene(seed: int = 3, n_boxes: int = 2_097_152, n_rays: int = 1_048_576, n_regions: int = 262_144,
                  dim: int = 6, n_comp: int = 64) -> dict:
    """Boxes with centres from a 64-component Gaussian mixture in [0,1]^D
    (sigma U[0.02,0.1], clamped to the unit cube) and half-extents
    log-uniform in [1e-4, 1e-2]; rays from U[0,1]^D with isotropic unit
    directions, t_max 2; regions with half-extent U[0.01,0.05]."""
    rng = Rng(seed)
    means = rng.unit64((n_comp, dim))
    sig = 0.02 + 0.08 * rng.unit64(n_comp)
    comp = (rng.take(n_boxes) % np.uint64(n_comp)).astype(np.int64)
    c = np.clip(means[comp] + sig[comp, None] * rng.normal64((n_boxes, dim)), 0.0, 1.0).astype(np.float32)
    h = np.exp(math.log(1e-4) + (math.log(1e-2) - math.log(1e-4)) * rng.unit64((n_boxes, dim))).astype(np.float32)
    prims = np.ascontiguousarray(np.concatenate([c - h, c + h], axis=1), dtype=np.float32)
    o = rng.range(0.0, 1.0, (n_rays, dim))
    rays = rays_from(o, isotropic(rng, n_rays, dim))
    rc = rng.range(0.0, 1.0, (n_regions, dim))
    rh = rng.range(0.01, 0.05, (n_regions, dim))
    regions = np.ascontiguousarray(np.concatenate([rc - rh, rc + rh], axis=1), dtype=np.float32)
    return dict(name=f"mixture{dim}d", dim=dim, kind="boxes", prims=prims, rays=rays, max_toi=2.0, regions=regions)
