// Exact device maths for the batched-query kernels.
//
// Every function restates the spatial-query CPU expression it replaces, in the
// same order of IEEE operations, so a hit's toi and identity are bit-identical
// to the reference CPU path. All arithmetic goes through the _rn intrinsics,
// which the compiler never contracts into an FMA (the files are additionally
// compiled with --fmad=false), and division / sqrt are the correctly rounded
// IEEE forms. The scalar type S is float (the crate's default) or double (its
// `f64` feature, maths/point.rs:14-18); float is the default everywhere.
#pragma once

#ifdef __CUDACC_RTC__
// Runtime compilation (NVRTC, for consumer narrow phases) has no <cstdint>.
typedef unsigned char uint8_t;
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

// Per-scalar constants: EPSILON (f32 / f64) and the triangle test's two
// literals (viewport-lib-query/src/lib.rs:281-306), in the scalar's precision.
template <class S> struct Lim;
template <> struct Lim<float> {
  static constexpr float eps = 1.1920928955078125e-7f;  // f32::EPSILON
  static constexpr float tri_det = 1e-8f;
  static constexpr float tri_t = 1e-6f;
};
template <> struct Lim<double> {
  static constexpr double eps = 2.220446049250313080847e-16;  // f64::EPSILON
  static constexpr double tri_det = 1e-8;
  static constexpr double tri_t = 1e-6;
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float sabs(float a) { return fabsf(a); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double fsqrt(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ double sabs(double a) { return fabs(a); }

// Rust's f32::total_cmp / f64::total_cmp as signed keys.
__device__ __forceinline__ int32_t total_key(float x) {
  int32_t b = __float_as_int(x);
  return b ^ int32_t(uint32_t(b >> 31) >> 1);
}
__device__ __forceinline__ int64_t total_key(double x) {
  int64_t b = __double_as_longlong(x);
  return b ^ int64_t(uint64_t(b >> 63) >> 1);
}

// hit_ordering (query/hit.rs:77-84): is (ta, la) strictly before (tb, lb)?
template <class S>
__device__ __forceinline__ bool hit_before(S ta, uint32_t la, S tb, uint32_t lb) {
  const auto ka = total_key(ta), kb = total_key(tb);
  return ka < kb || (ka == kb && la < lb);
}

// A ray or sweep with its per-axis reciprocals: inv[i] = 1 / d[i] is the value
// Aabb::ray_intersect recomputes at every node (aabb.rs:130); bit i of `par`
// marks an axis with |d| < EPSILON (the parallel-slab branch, aabb.rs:124-128).
template <int D, class S = float> struct RayPre {
  S o[D];
  S d[D];
  S inv[D];
  uint32_t par;
};

template <int D, class S> __device__ __forceinline__ void ray_prep(RayPre<D, S>& r) {
  r.par = 0;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    if (sabs(r.d[i]) < Lim<S>::eps) {
      r.par |= 1u << i;
      r.inv[i] = S(0);
    } else {
      r.inv[i] = fdiv(S(1), r.d[i]);
    }
  }
}

// Aabb::ray_intersect (aabb.rs:118-148). The reference returns early once
// t_min > t_max; t_min only grows and t_max only shrinks along the axes, so
// testing once at the end gives the same outcome. Returns pass and the entry
// parameter; `axis` is the last axis that raised t_min (-1: none).
template <int D, class S>
__device__ __forceinline__ bool slab(const RayPre<D, S>& r, const S* lo, const S* hi, S max_toi, S& t_enter,
                                     int& axis) {
  S tmin = S(0), tmax = max_toi;
  bool ok = true;
  axis = -1;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    if (r.par & (1u << i)) {
      ok = ok && !(r.o[i] < lo[i] || r.o[i] > hi[i]);
    } else {
      S t1 = fmul(fsub(lo[i], r.o[i]), r.inv[i]);
      S t2 = fmul(fsub(hi[i], r.o[i]), r.inv[i]);
      if (t1 > t2) { S t = t1; t1 = t2; t2 = t; }
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
template <int D, class S>
__device__ __forceinline__ bool slab_grown(const RayPre<D, S>& r, const S* lo, const S* hi, const S* pmin,
                                           const S* pmax, S max_toi, S& t_enter, int& axis) {
  S glo[D], ghi[D];
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
template <int D, class S> __device__ __forceinline__ bool box_overlap(const S* lo, const S* hi, const S* qlo,
                                                                      const S* qhi) {
  bool ok = true;
#pragma unroll
  for (int i = 0; i < D; ++i) ok = ok && !(lo[i] > qhi[i] || hi[i] < qlo[i]);
  return ok;
}

// Point::dot (point.rs:60-66): accumulate from 0.0 in index order.
template <int D, class S> __device__ __forceinline__ S pdot(const S* a, const S* b) {
  S acc = S(0);
#pragma unroll
  for (int i = 0; i < D; ++i) acc = fadd(acc, fmul(a[i], b[i]));
  return acc;
}

// Point::normalize_or_zero (point.rs:82-89), in place.
template <int D, class S> __device__ __forceinline__ void normalize_or_zero(S* v) {
  S len = fsqrt(pdot<D>(v, v));
  if (len > Lim<S>::eps) {
    S s = fdiv(S(1), len);
#pragma unroll
    for (int i = 0; i < D; ++i) v[i] = fmul(v[i], s);
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) v[i] = S(0);
  }
}

// Ray::at (ray.rs:33-35): origin + dir * t.
template <int D, class S> __device__ __forceinline__ void ray_at(const S* o, const S* d, S t, S* out) {
#pragma unroll
  for (int i = 0; i < D; ++i) out[i] = fadd(o[i], fmul(d[i], t));
}

// Entry-face normal: -sign(d[axis]) on `axis`, zero when axis < 0.
template <int D, class S> __device__ __forceinline__ void entry_normal(const S* d, int axis, S* n) {
#pragma unroll
  for (int i = 0; i < D; ++i) n[i] = (i == axis) ? ((d[i] > S(0)) ? S(-1) : S(1)) : S(0);
}

// Ray against a ball (tests/differential.rs:61-82; near-root-only variant
// tests/gpu.rs:92-106): the near root, or the far root when the origin is
// inside (FAR). Writes toi and the outward normal.
template <int D, bool FAR, class S>
__device__ __forceinline__ bool ray_ball(const S* o, const S* d, const S* c, S r, S max_toi, S& t_out, S* n_out) {
  S oc[D];
#pragma unroll
  for (int i = 0; i < D; ++i) oc[i] = fsub(o[i], c[i]);
  S b = pdot<D>(oc, d);
  S cc = fsub(pdot<D>(oc, oc), fmul(r, r));
  S disc = fsub(fmul(b, b), cc);
  if (disc < S(0)) return false;
  S sq = fsqrt(disc);
  S nb = -b;
  S t = fsub(nb, sq);
  if (FAR && t < S(0)) t = fadd(nb, sq);
  if (t < S(0) || t > max_toi) return false;
  t_out = t;
  S p[D];
  ray_at<D>(o, d, t, p);
#pragma unroll
  for (int i = 0; i < D; ++i) n_out[i] = fsub(p[i], c[i]);
  normalize_or_zero<D>(n_out);
  return true;
}

// glam Vec3 dot / cross, the operations of the reference triangle test
// (crates/viewport-lib-query/src/lib.rs:281-306).
template <class S> __device__ __forceinline__ S gdot(const S* a, const S* b) {
  return fadd(fadd(fmul(a[0], b[0]), fmul(a[1], b[1])), fmul(a[2], b[2]));
}
template <class S> __device__ __forceinline__ void gcross(const S* a, const S* b, S* o) {
  o[0] = fsub(fmul(a[1], b[2]), fmul(b[1], a[2]));
  o[1] = fsub(fmul(a[2], b[0]), fmul(b[2], a[0]));
  o[2] = fsub(fmul(a[0], b[1]), fmul(b[0], a[1]));
}

// Moeller-Trumbore, double-sided: |det| < 1e-8 rejects, u in [0, 1], v >= 0,
// u + v <= 1, t > 1e-6; the caller bounds t by max_toi.
template <class S>
__device__ __forceinline__ bool ray_triangle(const S* o, const S* d, const S* v0, const S* v1, const S* v2, S& t_out) {
  S e1[3], e2[3], p[3], tv[3], q[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) { e1[i] = fsub(v1[i], v0[i]); e2[i] = fsub(v2[i], v0[i]); }
  gcross(d, e2, p);
  S det = gdot(e1, p);
  if (sabs(det) < Lim<S>::tri_det) return false;
  S inv = fdiv(S(1), det);
#pragma unroll
  for (int i = 0; i < 3; ++i) tv[i] = fsub(o[i], v0[i]);
  S u = fmul(gdot(tv, p), inv);
  if (!(S(0) <= u && u <= S(1))) return false;
  gcross(tv, e1, q);
  S v = fmul(gdot(d, q), inv);
  if (v < S(0) || fadd(u, v) > S(1)) return false;
  S t = fmul(gdot(e2, q), inv);
  if (!(t > Lim<S>::tri_t)) return false;
  t_out = t;
  return true;
}

// Face normal: normalize_or_zero(cross(v1 - v0, v2 - v0)).
template <class S> __device__ __forceinline__ void tri_normal(const S* v0, const S* v1, const S* v2, S* n) {
  S e1[3], e2[3];
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
__device__ __forceinline__ void tri_aabb(const double* v0, const double* v1, const double* v2, double* lo,
                                         double* hi) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lo[i] = fmin(fmin(fmin(__longlong_as_double(0x7ff0000000000000ll), v0[i]), v1[i]), v2[i]);
    hi[i] = fmax(fmax(fmax(__longlong_as_double(0xfff0000000000000ll), v0[i]), v1[i]), v2[i]);
  }
}

}  // namespace sq
