// Exact device maths for the batched-query kernels.
//
// Every function restates the spatial-query CPU expression it replaces, in the
// same order of IEEE f32 operations, so a hit's toi and identity are
// bit-identical to the reference CPU path. All arithmetic goes through the
// _rn intrinsics, which the compiler never contracts into an FMA (the files are
// additionally compiled with --fmad=false), and division / sqrt are the
// correctly rounded IEEE forms.
#pragma once

#ifdef __CUDACC_RTC__
// Runtime compilation (NVRTC, for consumer narrow phases) has no <cstdint>.
typedef unsigned int uint32_t;
typedef int int32_t;
typedef unsigned long long uint64_t;
typedef long long int64_t;
#else
#include <cstdint>
#endif

namespace sq {

constexpr float kEps = 1.1920928955078125e-7f;  // f32::EPSILON
constexpr uint32_t kNoHit = 0xFFFFFFFFu;
constexpr uint32_t kLeafBit = 0x80000000u;

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }

// Rust's f32::total_cmp as a signed key.
__device__ __forceinline__ int32_t total_key(float x) {
  int32_t b = __float_as_int(x);
  return b ^ int32_t(uint32_t(b >> 31) >> 1);
}

// hit_ordering (query/hit.rs:77-84): is (ta, la) strictly before (tb, lb)?
__device__ __forceinline__ bool hit_before(float ta, uint32_t la, float tb, uint32_t lb) {
  int32_t ka = total_key(ta), kb = total_key(tb);
  return ka < kb || (ka == kb && la < lb);
}

// A ray or sweep with its per-axis reciprocals: inv[i] = 1 / d[i] is the value
// Aabb::ray_intersect recomputes at every node (aabb.rs:130); bit i of `par`
// marks an axis with |d| < EPSILON (the parallel-slab branch, aabb.rs:124-128).
template <int D> struct RayPre {
  float o[D];
  float d[D];
  float inv[D];
  uint32_t par;
};

template <int D> __device__ __forceinline__ void ray_prep(RayPre<D>& r) {
  r.par = 0;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    if (fabsf(r.d[i]) < kEps) {
      r.par |= 1u << i;
      r.inv[i] = 0.f;
    } else {
      r.inv[i] = fdiv(1.0f, r.d[i]);
    }
  }
}

// Aabb::ray_intersect (aabb.rs:118-148). The reference returns early once
// t_min > t_max; t_min only grows and t_max only shrinks along the axes, so
// testing once at the end gives the same outcome. Returns pass and the entry
// parameter; `axis` is the last axis that raised t_min (-1: none).
template <int D>
__device__ __forceinline__ bool slab(const RayPre<D>& r, const float* lo, const float* hi, float max_toi,
                                     float& t_enter, int& axis) {
  float tmin = 0.f, tmax = max_toi;
  bool ok = true;
  axis = -1;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    if (r.par & (1u << i)) {
      ok = ok && !(r.o[i] < lo[i] || r.o[i] > hi[i]);
    } else {
      float t1 = fmul(fsub(lo[i], r.o[i]), r.inv[i]);
      float t2 = fmul(fsub(hi[i], r.o[i]), r.inv[i]);
      if (t1 > t2) { float t = t1; t1 = t2; t2 = t; }
      if (t1 > tmin) { tmin = t1; axis = i; }
      if (t2 < tmax) tmax = t2;
    }
  }
  t_enter = tmin;
  return ok && !(tmin > tmax);
}

// The slab for a finite ray against a finite box. With no NaN possible, the
// compare-and-swap of the reference equals a min/max pair and its
// `if t > t_min` update equals a max, except that a max may return -0 where
// the reference keeps +0: only the returned entry can show that sign, so it is
// normalised with + 0. Callers use this form only for rays with no parallel
// axis and finite origin, direction, probe and limit, against a scene whose
// bounds are all finite; other rays take `slab`.
template <int D>
__device__ __forceinline__ bool slab_fast(const RayPre<D>& r, const float* lo, const float* hi, float max_toi,
                                          float& t_enter) {
  float tmin = 0.f, tmax = max_toi;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const float t1 = fmul(fsub(lo[i], r.o[i]), r.inv[i]);
    const float t2 = fmul(fsub(hi[i], r.o[i]), r.inv[i]);
    tmin = fmaxf(tmin, fminf(t1, t2));
    tmax = fminf(tmax, fmaxf(t1, t2));
  }
  t_enter = fadd(tmin, 0.0f);
  return !(tmin > tmax);
}

// The same slab against a box grown by a probe: ShapeCast::broadphase
// (query/shapecast.rs:70-73): grown = [lo - probe.max, hi - probe.min].
template <int D>
__device__ __forceinline__ bool slab_grown(const RayPre<D>& r, const float* lo, const float* hi, const float* pmin,
                                           const float* pmax, float max_toi, float& t_enter, int& axis) {
  float glo[D], ghi[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    glo[i] = fsub(lo[i], pmax[i]);
    ghi[i] = fsub(hi[i], pmin[i]);
  }
  return slab<D>(r, glo, ghi, max_toi, t_enter, axis);
}

template <int D>
__device__ __forceinline__ bool slab_grown_fast(const RayPre<D>& r, const float* lo, const float* hi,
                                                const float* pmin, const float* pmax, float max_toi,
                                                float& t_enter) {
  float glo[D], ghi[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    glo[i] = fsub(lo[i], pmax[i]);
    ghi[i] = fsub(hi[i], pmin[i]);
  }
  return slab_fast<D>(r, glo, ghi, max_toi, t_enter);
}

// Aabb::intersects (aabb.rs:101-108): touching faces count.
template <int D> __device__ __forceinline__ bool box_overlap(const float* lo, const float* hi, const float* qlo,
                                                             const float* qhi) {
  bool ok = true;
#pragma unroll
  for (int i = 0; i < D; ++i) ok = ok && !(lo[i] > qhi[i] || hi[i] < qlo[i]);
  return ok;
}

// Point::dot (point.rs:60-66): accumulate from 0.0 in index order.
template <int D> __device__ __forceinline__ float pdot(const float* a, const float* b) {
  float acc = 0.f;
#pragma unroll
  for (int i = 0; i < D; ++i) acc = fadd(acc, fmul(a[i], b[i]));
  return acc;
}

// Point::normalize_or_zero (point.rs:82-89), in place.
template <int D> __device__ __forceinline__ void normalize_or_zero(float* v) {
  float len = fsqrt(pdot<D>(v, v));
  if (len > kEps) {
    float s = fdiv(1.0f, len);
#pragma unroll
    for (int i = 0; i < D; ++i) v[i] = fmul(v[i], s);
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) v[i] = 0.f;
  }
}

// Ray::at (ray.rs:33-35): origin + dir * t.
template <int D> __device__ __forceinline__ void ray_at(const float* o, const float* d, float t, float* out) {
#pragma unroll
  for (int i = 0; i < D; ++i) out[i] = fadd(o[i], fmul(d[i], t));
}

// Entry-face normal: -sign(d[axis]) on `axis`, zero when axis < 0.
template <int D> __device__ __forceinline__ void entry_normal(const float* d, int axis, float* n) {
#pragma unroll
  for (int i = 0; i < D; ++i) n[i] = (i == axis) ? ((d[i] > 0.f) ? -1.f : 1.f) : 0.f;
}

// Ray against a ball (tests/differential.rs:61-82; near-root-only variant
// tests/gpu.rs:92-106): the near root, or the far root when the origin is
// inside (FAR). Writes toi and the outward normal.
template <int D, bool FAR>
__device__ __forceinline__ bool ray_ball(const float* o, const float* d, const float* c, float r, float max_toi,
                                         float& t_out, float* n_out) {
  float oc[D];
#pragma unroll
  for (int i = 0; i < D; ++i) oc[i] = fsub(o[i], c[i]);
  float b = pdot<D>(oc, d);
  float cc = fsub(pdot<D>(oc, oc), fmul(r, r));
  float disc = fsub(fmul(b, b), cc);
  if (disc < 0.f) return false;
  float sq = fsqrt(disc);
  float nb = -b;
  float t = fsub(nb, sq);
  if (FAR && t < 0.f) t = fadd(nb, sq);
  if (t < 0.f || t > max_toi) return false;
  t_out = t;
  float p[D];
  ray_at<D>(o, d, t, p);
#pragma unroll
  for (int i = 0; i < D; ++i) n_out[i] = fsub(p[i], c[i]);
  normalize_or_zero<D>(n_out);
  return true;
}

// glam Vec3 dot / cross, the operations of the reference triangle test
// (crates/viewport-lib-query/src/lib.rs:295-320).
__device__ __forceinline__ float gdot(const float* a, const float* b) {
  return fadd(fadd(fmul(a[0], b[0]), fmul(a[1], b[1])), fmul(a[2], b[2]));
}
__device__ __forceinline__ void gcross(const float* a, const float* b, float* o) {
  o[0] = fsub(fmul(a[1], b[2]), fmul(b[1], a[2]));
  o[1] = fsub(fmul(a[2], b[0]), fmul(b[2], a[0]));
  o[2] = fsub(fmul(a[0], b[1]), fmul(b[0], a[1]));
}

// Moeller-Trumbore, double-sided: |det| < 1e-8 rejects, u in [0, 1], v >= 0,
// u + v <= 1, t > 1e-6; the caller bounds t by max_toi.
__device__ __forceinline__ bool ray_triangle(const float* o, const float* d, const float* v0, const float* v1,
                                             const float* v2, float& t_out) {
  float e1[3], e2[3], p[3], tv[3], q[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) { e1[i] = fsub(v1[i], v0[i]); e2[i] = fsub(v2[i], v0[i]); }
  gcross(d, e2, p);
  float det = gdot(e1, p);
  if (fabsf(det) < 1e-8f) return false;
  float inv = fdiv(1.0f, det);
#pragma unroll
  for (int i = 0; i < 3; ++i) tv[i] = fsub(o[i], v0[i]);
  float u = fmul(gdot(tv, p), inv);
  if (!(0.f <= u && u <= 1.f)) return false;
  gcross(tv, e1, q);
  float v = fmul(gdot(d, q), inv);
  if (v < 0.f || fadd(u, v) > 1.f) return false;
  float t = fmul(gdot(e2, q), inv);
  if (!(t > 1e-6f)) return false;
  t_out = t;
  return true;
}

// Face normal: normalize_or_zero(cross(v1 - v0, v2 - v0)).
__device__ __forceinline__ void tri_normal(const float* v0, const float* v1, const float* v2, float* n) {
  float e1[3], e2[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) { e1[i] = fsub(v1[i], v0[i]); e2[i] = fsub(v2[i], v0[i]); }
  gcross(e1, e2, n);
  normalize_or_zero<3>(n);
}

// Aabb::EMPTY grown by the three vertices (min/max with Rust's NaN rule:
// fminf/fmaxf return the non-NaN operand).
__device__ __forceinline__ void tri_aabb(const float* v0, const float* v1, const float* v2, float* lo, float* hi) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lo[i] = fminf(fminf(fminf(__int_as_float(0x7f800000), v0[i]), v1[i]), v2[i]);
    hi[i] = fmaxf(fmaxf(fmaxf(__int_as_float(0xff800000), v0[i]), v1[i]), v2[i]);
  }
}

}  // namespace sq
