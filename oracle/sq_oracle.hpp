// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the batched-query path.
//
// A C++ restatement of the spatial-query crate's CPU query path
// (crates/spatial-query/src/{maths,accel,query}), used by the test-suite, by
// `__graft_entry__.smoke()` and by the CPU-baseline leg of `bench.py` as the
// checker. Nothing in the product library links or calls this code.
//
// Exactness rules followed everywhere (the reference is Rust, which never
// contracts a*b+c into an FMA): compile with -ffp-contract=off, no fast-math,
// every expression evaluated in the reference's order, IEEE `/` and `sqrt`.
// `Scalar` is a template parameter so an f64 build (the crate's `f64` feature,
// maths/point.rs:14-18) can be instantiated beside the f32 one.
//
// Parity pinning: the reference cannot be compiled in this image (no Rust
// toolchain). This restatement is pinned by the reference's own known-answer
// tests and its BVH==naive randomised parity seeds, ported under tests/.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <optional>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// L0 maths: Point<D> (maths/point.rs), Aabb<D> (maths/aabb.rs),
// Ray<D> (maths/ray.rs), Isometry<D> (maths/isometry.rs).
// ---------------------------------------------------------------------------

template <class S> struct Lim;
template <> struct Lim<float> {
  static constexpr float eps = 1.1920928955078125e-7f;  // f32::EPSILON
};
template <> struct Lim<double> {
  static constexpr double eps = 2.220446049250313080847e-16;  // f64::EPSILON
};

// Rust's f32::min / f32::max: a NaN operand yields the other operand.
template <class S> inline S rmin(S a, S b) { return std::fmin(a, b); }
template <class S> inline S rmax(S a, S b) { return std::fmax(a, b); }

template <int D, class S> struct Point {
  S v[D];
  static Point zero() { Point p; for (int i = 0; i < D; ++i) p.v[i] = S(0); return p; }
  static Point splat(S x) { Point p; for (int i = 0; i < D; ++i) p.v[i] = x; return p; }
  S operator[](int i) const { return v[i]; }
  S& operator[](int i) { return v[i]; }
  // point.rs:40-56
  Point min(const Point& o) const { Point r = *this; for (int i = 0; i < D; ++i) r.v[i] = rmin(r.v[i], o.v[i]); return r; }
  Point max(const Point& o) const { Point r = *this; for (int i = 0; i < D; ++i) r.v[i] = rmax(r.v[i], o.v[i]); return r; }
  // point.rs:60-66: accumulate from 0.0 in index order.
  S dot(const Point& o) const { S acc = S(0); for (int i = 0; i < D; ++i) acc += v[i] * o.v[i]; return acc; }
  S length_squared() const { return dot(*this); }
  S length() const { return std::sqrt(length_squared()); }
  // point.rs:82-89: multiply by the reciprocal, zero below EPSILON.
  Point normalize_or_zero() const {
    S len = length();
    if (len > Lim<S>::eps) return (*this) * (S(1) / len);
    return zero();
  }
  Point operator+(const Point& o) const { Point r = *this; for (int i = 0; i < D; ++i) r.v[i] += o.v[i]; return r; }
  Point operator-(const Point& o) const { Point r = *this; for (int i = 0; i < D; ++i) r.v[i] -= o.v[i]; return r; }
  Point operator*(S s) const { Point r = *this; for (int i = 0; i < D; ++i) r.v[i] *= s; return r; }
  Point operator-() const { return (*this) * S(-1); }  // point.rs:136-142
  bool is_zero() const { for (int i = 0; i < D; ++i) if (v[i] != S(0)) return false; return true; }
};

template <int D, class S> struct Ray {
  Point<D, S> origin, dir;
  // ray.rs:18-23
  static Ray make(const Point<D, S>& o, const Point<D, S>& d) { return Ray{o, d.normalize_or_zero()}; }
  Point<D, S> at(S t) const { return origin + dir * t; }  // ray.rs:33-35
};

template <int D, class S> struct Aabb {
  Point<D, S> min, max;
  static Aabb empty() {
    return Aabb{Point<D, S>::splat(std::numeric_limits<S>::infinity()),
                Point<D, S>::splat(-std::numeric_limits<S>::infinity())};
  }
  Aabb unite(const Aabb& o) const { return Aabb{min.min(o.min), max.max(o.max)}; }       // aabb.rs:38-43
  Aabb union_point(const Point<D, S>& p) const { return Aabb{min.min(p), max.max(p)}; }  // aabb.rs:47-52
  Point<D, S> center() const { return (min + max) * S(0.5); }                             // aabb.rs:56-58
  Point<D, S> extents() const { return max - min; }                                       // aabb.rs:62-64
  int longest_axis() const {                                                              // aabb.rs:68-77
    Point<D, S> e = extents();
    int best = 0;
    for (int i = 1; i < D; ++i) if (e[i] > e[best]) best = i;
    return best;
  }
  S half_surface() const {  // aabb.rs:84-97
    Point<D, S> e = extents();
    S sum = S(0);
    for (int i = 0; i < D; ++i) {
      S prod = S(1);
      for (int j = 0; j < D; ++j) if (j != i) prod *= e[j];
      sum += prod;
    }
    return sum;
  }
  bool intersects(const Aabb& o) const {  // aabb.rs:101-108
    for (int i = 0; i < D; ++i)
      if (min[i] > o.max[i] || max[i] < o.min[i]) return false;
    return true;
  }
  // aabb.rs:118-148. `axis_out` (an addition of this restatement) reports the
  // last axis whose entry raised t_min, or -1 when t_min stayed at zero; the
  // built-in box narrow phase uses it for the entry-face normal.
  bool ray_intersect(const Ray<D, S>& ray, S max_toi, S* tmin_out, S* tmax_out, int* axis_out = nullptr) const {
    S t_min = S(0);
    S t_max = max_toi;
    int axis = -1;
    for (int i = 0; i < D; ++i) {
      S o = ray.origin[i];
      S d = ray.dir[i];
      if (std::fabs(d) < Lim<S>::eps) {
        if (o < min[i] || o > max[i]) return false;
      } else {
        S inv = S(1) / d;
        S t1 = (min[i] - o) * inv;
        S t2 = (max[i] - o) * inv;
        if (t1 > t2) std::swap(t1, t2);
        if (t1 > t_min) { t_min = t1; axis = i; }
        if (t2 < t_max) t_max = t2;
        if (t_min > t_max) return false;
      }
    }
    *tmin_out = t_min;
    *tmax_out = t_max;
    if (axis_out) *axis_out = axis;
    return true;
  }
};

template <int D, class S> struct Isometry {
  S rot[D][D];  // row-major, isometry.rs:21-22
  Point<D, S> translation;
  static Isometry identity() {
    Isometry r;
    for (int i = 0; i < D; ++i) for (int j = 0; j < D; ++j) r.rot[i][j] = (i == j) ? S(1) : S(0);
    r.translation = Point<D, S>::zero();
    return r;
  }
  Point<D, S> rotate(const Point<D, S>& v) const {  // isometry.rs:100-110
    Point<D, S> out;
    for (int i = 0; i < D; ++i) { S acc = S(0); for (int j = 0; j < D; ++j) acc += rot[i][j] * v[j]; out[i] = acc; }
    return out;
  }
  Point<D, S> rotate_transpose(const Point<D, S>& v) const {  // isometry.rs:113-123
    Point<D, S> out;
    for (int i = 0; i < D; ++i) { S acc = S(0); for (int j = 0; j < D; ++j) acc += rot[j][i] * v[j]; out[i] = acc; }
    return out;
  }
  Point<D, S> transform_point(const Point<D, S>& p) const { return rotate(p) + translation; }        // :58-60
  Point<D, S> transform_vector(const Point<D, S>& v) const { return rotate(v); }                     // :64-66
  Point<D, S> inverse_transform_point(const Point<D, S>& p) const { return rotate_transpose(p - translation); }  // :70-72
  Point<D, S> inverse_transform_vector(const Point<D, S>& v) const { return rotate_transpose(v); }   // :76-78
  Aabb<D, S> transform_aabb(const Aabb<D, S>& local) const {  // isometry.rs:84-97
    Point<D, S> c = transform_point(local.center());
    Point<D, S> h = local.extents() * S(0.5);
    Point<D, S> wh;
    for (int i = 0; i < D; ++i) { S acc = S(0); for (int j = 0; j < D; ++j) acc += std::fabs(rot[i][j]) * h[j]; wh[i] = acc; }
    return Aabb<D, S>{c - wh, c + wh};
  }
};

// Rust's f32::total_cmp as a signed integer key (-0 < +0, NaNs at the ends).
inline int32_t total_key(float x) {
  int32_t b; std::memcpy(&b, &x, 4);
  return b ^ int32_t(uint32_t(b >> 31) >> 1);
}
inline int64_t total_key(double x) {
  int64_t b; std::memcpy(&b, &x, 8);
  return b ^ int64_t(uint64_t(b >> 63) >> 1);
}

// ---------------------------------------------------------------------------
// L1 query vocabulary: LeafHit/Hit + hit_ordering (query/hit.rs),
// QueryFilter (query/filter.rs), ShapeCast (query/shapecast.rs).
// ---------------------------------------------------------------------------

constexpr uint32_t kNoSub = 0xFFFFFFFFu;  // `sub_object: None`

template <int D, class S> struct LeafHit {
  S toi;
  Point<D, S> normal;
  uint32_t sub = kNoSub;
};

template <int D, class S> struct Hit {
  uint32_t leaf;
  S toi;
  Point<D, S> point, normal;
  uint32_t sub;
};

// hit.rs:77-84: toi by total_cmp, then leaf. Returns <0, 0, >0.
template <int D, class S> inline int hit_cmp(const Hit<D, S>& a, const Hit<D, S>& b) {
  auto ka = total_key(a.toi), kb = total_key(b.toi);
  if (ka != kb) return ka < kb ? -1 : 1;
  if (a.leaf != b.leaf) return a.leaf < b.leaf ? -1 : 1;
  return 0;
}

struct Filter {  // filter.rs:12-29
  uint64_t layer_mask = ~0ull;
  bool has_exclude = false;
  uint64_t exclude = 0;
};

template <int D, class S> struct ShapeCast {
  Point<D, S> origin, dir;
  Aabb<D, S> aabb;
  Point<D, S> at(S t) const { return origin + dir * t; }  // shapecast.rs:61-63
  // shapecast.rs:70-73: slab test against the target grown by the probe box.
  bool broadphase(const Aabb<D, S>& target, S max_toi, S* t0, S* t1, int* axis = nullptr) const {
    Aabb<D, S> grown{target.min - aabb.max, target.max - aabb.min};
    Ray<D, S> r{origin, dir};
    return grown.ray_intersect(r, max_toi, t0, t1, axis);
  }
};

struct QueryStats {  // accel/stats.rs:41-50
  uint64_t nodes_visited = 0, aabb_tests = 0, narrow_tests = 0, hits = 0;
};

// ---------------------------------------------------------------------------
// L2a tree storage, median-split build and refit (accel/tree.rs).
// ---------------------------------------------------------------------------

constexpr uint32_t kLeafSize = 4;  // tree.rs:12

template <int D, class S> struct Node {  // tree.rs:21-26
  Aabb<D, S> bounds;
  uint32_t child_a, child_b, prim_count;
  bool is_leaf() const { return prim_count > 0; }
};

template <int D, class S>
uint32_t build_recursive(std::vector<Node<D, S>>& nodes, uint32_t* indices, const Aabb<D, S>* bounds,
                         const Point<D, S>* centroids, uint32_t start, uint32_t end) {
  // tree.rs:112-163
  Aabb<D, S> nb = Aabb<D, S>::empty();
  for (uint32_t k = start; k < end; ++k) nb = nb.unite(bounds[indices[k]]);
  uint32_t node_index = uint32_t(nodes.size());
  uint32_t count = end - start;
  nodes.push_back(Node<D, S>{nb, start, 0, count});
  if (count <= kLeafSize) return node_index;
  Aabb<D, S> cb = Aabb<D, S>::empty();
  for (uint32_t k = start; k < end; ++k) cb = cb.union_point(centroids[indices[k]]);
  int axis = cb.longest_axis();
  if (cb.extents()[axis] <= Lim<S>::eps) return node_index;
  // Stable sort by total_cmp on the chosen centroid axis (tree.rs:152-153).
  std::stable_sort(indices + start, indices + end, [&](uint32_t a, uint32_t b) {
    return total_key(centroids[a][axis]) < total_key(centroids[b][axis]);
  });
  uint32_t mid = start + count / 2;
  uint32_t ca = build_recursive(nodes, indices, bounds, centroids, start, mid);
  uint32_t cbi = build_recursive(nodes, indices, bounds, centroids, mid, end);
  Node<D, S>& n = nodes[node_index];
  n.child_a = ca;
  n.child_b = cbi;
  n.prim_count = 0;
  return node_index;
}

template <int D, class S>
void tree_build(const std::vector<Aabb<D, S>>& bounds, std::vector<Node<D, S>>& nodes, std::vector<uint32_t>& indices) {
  // tree.rs:39-49
  uint32_t n = uint32_t(bounds.size());
  indices.resize(n);
  for (uint32_t i = 0; i < n; ++i) indices[i] = i;
  nodes.clear();
  if (n == 0) return;
  std::vector<Point<D, S>> centroids(n);
  for (uint32_t i = 0; i < n; ++i) centroids[i] = bounds[i].center();
  nodes.reserve(2 * n);
  build_recursive(nodes, indices.data(), bounds.data(), centroids.data(), 0, n);
}

template <int D, class S>
void tree_refit(std::vector<Node<D, S>>& nodes, const std::vector<uint32_t>& indices, const std::vector<Aabb<D, S>>& pb) {
  // tree.rs:54-75
  for (size_t ni = nodes.size(); ni-- > 0;) {
    Node<D, S> node = nodes[ni];
    if (node.is_leaf()) {
      Aabb<D, S> b = Aabb<D, S>::empty();
      for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) b = b.unite(pb[indices[k]]);
      nodes[ni].bounds = b;
    } else {
      nodes[ni].bounds = nodes[node.child_a].bounds.unite(nodes[node.child_b].bounds);
    }
  }
}

template <int D, class S>
void tree_structural(const std::vector<Node<D, S>>& nodes, size_t* leaves, size_t* prims, size_t* depth) {
  // tree.rs:81-99
  *leaves = *prims = *depth = 0;
  if (nodes.empty()) return;
  std::vector<size_t> dep(nodes.size(), 0);
  for (size_t ni = nodes.size(); ni-- > 0;) {
    const Node<D, S>& n = nodes[ni];
    if (n.is_leaf()) { ++*leaves; *prims += n.prim_count; dep[ni] = 1; }
    else dep[ni] = 1 + std::max(dep[n.child_a], dep[n.child_b]);
  }
  *depth = dep[0];
}

template <int D, class S> S interior_surface_sum(const std::vector<Node<D, S>>& nodes) {
  // tree.rs:104-110 (an iterator sum: sequential from 0.0 in node order)
  S sum = S(0);
  for (const auto& n : nodes) if (!n.is_leaf()) sum += n.bounds.half_surface();
  return sum;
}

// ---------------------------------------------------------------------------
// Providers: the QueryGeometry implementations the reference's tests and the
// benchmark scenes use (query/geometry.rs:19-98 is the trait).
// ---------------------------------------------------------------------------

// Shared accept hook: with no per-leaf layers the provider accepts every leaf
// (the trait default, geometry.rs:95-97); with layers it accepts a leaf whose
// layer bits meet the mask and that is not the excluded leaf
// (tests/result_identity.rs:102-104 uses layers 1 << (leaf % 2)).
struct LayerAccept {
  const uint64_t* layers = nullptr;
  bool accepts(size_t leaf, const Filter& f) const {
    if (!layers) return true;
    if (f.has_exclude && f.exclude == leaf) return false;
    return (layers[leaf] & f.layer_mask) != 0;
  }
};

// Ray against a ball (tests/differential.rs:61-82, shape_overlap.rs:120-138):
// near root, or the far root when the origin is inside (`far_root`); the
// near-root-only form is tests/gpu.rs:92-106 and conformance.rs:277-291.
template <int D, class S>
inline bool ray_ball(const Ray<D, S>& ray, const Point<D, S>& c, S r, S max_toi, bool far_root, S* t_out,
                     Point<D, S>* n_out) {
  Point<D, S> oc = ray.origin - c;
  S b = oc.dot(ray.dir);
  S cc = oc.length_squared() - r * r;
  S disc = b * b - cc;
  if (disc < S(0)) return false;
  S sq = std::sqrt(disc);
  S t = -b - sq;
  if (far_root && t < S(0)) t = -b + sq;
  if (t < S(0) || t > max_toi) return false;
  *t_out = t;
  *n_out = (ray.at(t) - c).normalize_or_zero();
  return true;
}

// The two roots of an unbounded ray against a sphere (tests/crossings.rs:52-66).
template <int D, class S>
inline bool sphere_roots(const Ray<D, S>& ray, const Point<D, S>& c, S r, S* t0, S* t1) {
  Point<D, S> oc = ray.origin - c;
  S b = oc.dot(ray.dir);
  S disc = b * b - (oc.length_squared() - r * r);
  if (disc < S(0)) return false;
  S sq = std::sqrt(disc);
  *t0 = -b - sq;
  *t1 = -b + sq;
  return true;
}

// Distance from a point to a box, zero inside (tests/shape_overlap.rs:59-72).
template <int D, class S> inline S point_to_aabb(const Point<D, S>& p, const Aabb<D, S>& b) {
  S d2 = S(0);
  for (int i = 0; i < D; ++i) {
    S v = (p[i] < b.min[i]) ? (b.min[i] - p[i]) : ((p[i] > b.max[i]) ? (p[i] - b.max[i]) : S(0));
    d2 += v * v;
  }
  return std::sqrt(d2);
}

// Outward normal of the face a ray enters through: -sign(d[axis]) on `axis`
// (the convention of tests/two_level.rs:108-112); zero when axis < 0.
template <int D, class S> inline Point<D, S> entry_normal(const Point<D, S>& dir, int axis) {
  Point<D, S> n = Point<D, S>::zero();
  if (axis >= 0) n[axis] = (dir[axis] > S(0)) ? S(-1) : S(1);
  return n;
}

// Moeller-Trumbore, double-sided (crates/viewport-lib-query/src/lib.rs:281-306),
// with glam Vec3's dot = (x*x' + y*y') + z*z' and cross component order.
template <class S> struct V3 { S x, y, z; };
template <class S> inline V3<S> v3sub(V3<S> a, V3<S> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S> inline S v3dot(V3<S> a, V3<S> b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
template <class S> inline V3<S> v3cross(V3<S> a, V3<S> b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class S> inline bool ray_triangle(V3<S> o, V3<S> d, V3<S> v0, V3<S> v1, V3<S> v2, S* t_out) {
  V3<S> e1 = v3sub(v1, v0), e2 = v3sub(v2, v0);
  V3<S> p = v3cross(d, e2);
  S det = v3dot(e1, p);
  if (std::fabs(det) < S(1e-8)) return false;
  S inv = S(1) / det;
  V3<S> tv = v3sub(o, v0);
  S u = v3dot(tv, p) * inv;
  if (!(S(0) <= u && u <= S(1))) return false;
  V3<S> q = v3cross(tv, e1);
  S v = v3dot(d, q) * inv;
  if (v < S(0) || u + v > S(1)) return false;
  S t = v3dot(e2, q) * inv;
  if (t > S(1e-6)) { *t_out = t; return true; }
  return false;
}

// Triangle face normal: normalize_or_zero(cross(v1 - v0, v2 - v0)) with the
// crate's Point normalisation (point.rs:82-89).
template <class S> inline Point<3, S> tri_normal(V3<S> v0, V3<S> v1, V3<S> v2) {
  V3<S> n = v3cross(v3sub(v1, v0), v3sub(v2, v0));
  Point<3, S> p; p[0] = n.x; p[1] = n.y; p[2] = n.z;
  return p.normalize_or_zero();
}

// Provider kinds shared with the C API.
enum Kind : int {
  kBoxes = 0,      // leaf = an axis-aligned box; hit = slab entry (aabb.rs:118-148)
  kBalls = 1,      // leaf = a ball; near root, far root when inside
  kBallsNear = 2,  // leaf = a ball; near root only
  kTris = 3,       // leaf = a triangle (D = 3); Moeller-Trumbore
};

template <int D, class S> struct Scene {
  int kind = kBoxes;
  uint32_t n = 0;
  std::vector<S> data;  // per-leaf parameters, leaf-major
  LayerAccept acc;
  std::vector<uint64_t> layers;
  std::vector<uint32_t> sub;  // per-leaf sub-object ids (empty: none)

  uint32_t stride() const {
    switch (kind) {
      case kBoxes: return 2 * D;
      case kBalls: case kBallsNear: return D + 1;
      default: return 9;
    }
  }
  size_t leaf_count() const { return n; }
  uint32_t sub_of(size_t leaf) const { return sub.empty() ? kNoSub : sub[leaf]; }
  bool accepts(size_t leaf, const Filter& f) const { return acc.accepts(leaf, f); }

  Aabb<D, S> world_aabb(size_t leaf) const {
    const S* p = &data[leaf * stride()];
    Aabb<D, S> a;
    if (kind == kBoxes) {
      for (int i = 0; i < D; ++i) { a.min[i] = p[i]; a.max[i] = p[D + i]; }
    } else if (kind == kBalls || kind == kBallsNear) {
      Point<D, S> c; for (int i = 0; i < D; ++i) c[i] = p[i];
      S r = p[D];
      a.min = c - Point<D, S>::splat(r);
      a.max = c + Point<D, S>::splat(r);
    } else {
      // aabb_of (viewport-lib-query/src/lib.rs:323-329): EMPTY grown by each vertex.
      a = Aabb<D, S>::empty();
      for (int k = 0; k < 3; ++k) {
        Point<D, S> q = Point<D, S>::zero();
        for (int i = 0; i < 3 && i < D; ++i) q[i] = p[3 * k + i];
        a = a.union_point(q);
      }
    }
    return a;
  }

  bool test_ray(size_t leaf, const Ray<D, S>& ray, S max_toi, LeafHit<D, S>* out) const {
    const S* p = &data[leaf * stride()];
    if (kind == kBoxes) {
      S t0, t1; int axis;
      if (!world_aabb(leaf).ray_intersect(ray, max_toi, &t0, &t1, &axis)) return false;
      out->toi = t0;
      out->normal = entry_normal(ray.dir, axis);
      out->sub = sub_of(leaf);
      return true;
    }
    if (kind == kBalls || kind == kBallsNear) {
      Point<D, S> c; for (int i = 0; i < D; ++i) c[i] = p[i];
      S t; Point<D, S> nrm;
      if (!ray_ball(ray, c, p[D], max_toi, kind == kBalls, &t, &nrm)) return false;
      out->toi = t; out->normal = nrm; out->sub = sub_of(leaf);
      return true;
    }
    if constexpr (D == 3) {
      V3<S> o{ray.origin[0], ray.origin[1], ray.origin[2]}, d{ray.dir[0], ray.dir[1], ray.dir[2]};
      V3<S> v0{p[0], p[1], p[2]}, v1{p[3], p[4], p[5]}, v2{p[6], p[7], p[8]};
      S t;
      if (!ray_triangle(o, d, v0, v1, v2, &t)) return false;
      if (t > max_toi) return false;
      out->toi = t; out->normal = tri_normal(v0, v1, v2); out->sub = sub_of(leaf);
      return true;
    }
    return false;
  }

  // geometry.rs:56-66 default, overridden for balls with both roots
  // (tests/crossings.rs:505-521).
  template <class F> void test_ray_crossings(size_t leaf, const Ray<D, S>& ray, S max_toi, F&& out) const {
    if (kind == kBalls) {
      const S* p = &data[leaf * stride()];
      Point<D, S> c; for (int i = 0; i < D; ++i) c[i] = p[i];
      S t0, t1;
      if (!sphere_roots(ray, c, p[D], &t0, &t1)) return;
      for (S t : {t0, t1}) {
        if (t >= S(0) && t <= max_toi) {
          LeafHit<D, S> lh; lh.toi = t; lh.normal = (ray.at(t) - c).normalize_or_zero(); lh.sub = sub_of(leaf);
          out(lh);
        }
      }
      return;
    }
    LeafHit<D, S> lh;
    if (test_ray(leaf, ray, max_toi, &lh)) out(lh);
  }

  // Shape casts. Balls: a ball probe of radius cast.aabb.max[0] reduces to a ray
  // against the summed radius (tests/shape_overlap.rs:96-110,
  // result_identity.rs:88-99). Boxes: the exact swept-box TOI is the
  // broad-phase entry against the grown box. Triangles: the reference defines
  // no swept-box narrow phase; this one is swept box vs the triangle's AABB.
  bool test_shape_cast(size_t leaf, const ShapeCast<D, S>& cast, S max_toi, LeafHit<D, S>* out) const {
    if (kind == kBalls || kind == kBallsNear) {
      const S* p = &data[leaf * stride()];
      Point<D, S> c; for (int i = 0; i < D; ++i) c[i] = p[i];
      S sum = p[D] + cast.aabb.max[0];
      Ray<D, S> r{cast.origin, cast.dir};
      S t; Point<D, S> nrm;
      if (!ray_ball(r, c, sum, max_toi, kind == kBalls, &t, &nrm)) return false;
      out->toi = t;
      out->normal = (cast.at(t) - c).normalize_or_zero();
      out->sub = sub_of(leaf);
      return true;
    }
    S t0, t1; int axis;
    if (!cast.broadphase(world_aabb(leaf), max_toi, &t0, &t1, &axis)) return false;
    out->toi = t0;
    out->normal = entry_normal(cast.dir, axis);
    out->sub = sub_of(leaf);
    return true;
  }

  bool test_overlap(size_t leaf, const Aabb<D, S>& region) const {
    if (kind == kBalls || kind == kBallsNear) {
      const S* p = &data[leaf * stride()];
      Point<D, S> c; for (int i = 0; i < D; ++i) c[i] = p[i];
      return point_to_aabb(c, region) <= p[D];  // shape_overlap.rs:113-115
    }
    // Boxes and triangles answer at the level of their own AABB. (The trait
    // default, geometry.rs:89-91, returns true, which Bvh::overlap would turn
    // into whole-leaf-node answers; these providers override it.)
    return world_aabb(leaf).intersects(region);
  }
};

// ---------------------------------------------------------------------------
// Single-level BVH queries (accel/bvh.rs) and the naive scans (query/naive.rs).
// ---------------------------------------------------------------------------

template <int D, class S> struct Bvh {
  std::vector<Node<D, S>> nodes;
  std::vector<uint32_t> prim_indices;

  template <class G> void build(const G& g) {  // bvh.rs:31-38
    std::vector<Aabb<D, S>> b(g.leaf_count());
    for (size_t i = 0; i < b.size(); ++i) b[i] = g.world_aabb(i);
    tree_build(b, nodes, prim_indices);
  }
  template <class G> void refit(const G& g) {  // bvh.rs:45-48
    std::vector<Aabb<D, S>> b(g.leaf_count());
    for (size_t i = 0; i < b.size(); ++i) b[i] = g.world_aabb(i);
    tree_refit(nodes, prim_indices, b);
  }

  // bvh.rs:73-124
  template <class G>
  std::optional<Hit<D, S>> nearest(const G& g, const Ray<D, S>& ray, S max_toi, const Filter& f, QueryStats* st) const {
    if (nodes.empty()) return std::nullopt;
    std::optional<Hit<D, S>> best;
    S limit = max_toi;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      if (st) { st->nodes_visited++; st->aabb_tests++; }
      S te, tx;
      if (!node.bounds.ray_intersect(ray, limit, &te, &tx) || !(te <= limit)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t leaf = prim_indices[k];
          if (!g.accepts(leaf, f)) continue;
          if (st) st->narrow_tests++;
          LeafHit<D, S> lh;
          if (g.test_ray(leaf, ray, limit, &lh)) {
            if (st) st->hits++;
            Hit<D, S> h{leaf, lh.toi, ray.at(lh.toi), lh.normal, lh.sub};  // naive.rs:17-31
            if (!best || hit_cmp(*best, h) > 0) { limit = h.toi; best = h; }
          }
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    return best;
  }

  // bvh.rs:218-259 (all hits) and bvh.rs:286-328 (crossings).
  template <class G>
  void all(const G& g, const Ray<D, S>& ray, S max_toi, const Filter& f, bool crossings,
           std::vector<Hit<D, S>>& hits, QueryStats* st) const {
    hits.clear();
    if (nodes.empty()) return;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      if (st) { st->nodes_visited++; st->aabb_tests++; }
      S te, tx;
      if (!node.bounds.ray_intersect(ray, max_toi, &te, &tx)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t leaf = prim_indices[k];
          if (!g.accepts(leaf, f)) continue;
          if (st) st->narrow_tests++;
          auto push = [&](const LeafHit<D, S>& lh) {
            if (st) st->hits++;
            hits.push_back(Hit<D, S>{leaf, lh.toi, ray.at(lh.toi), lh.normal, lh.sub});
          };
          if (crossings) {
            g.test_ray_crossings(leaf, ray, max_toi, push);
          } else {
            LeafHit<D, S> lh;
            if (g.test_ray(leaf, ray, max_toi, &lh)) push(lh);
          }
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    std::stable_sort(hits.begin(), hits.end(), [](const Hit<D, S>& a, const Hit<D, S>& b) { return hit_cmp(a, b) < 0; });
  }

  // bvh.rs:331-375
  template <class G>
  std::optional<Hit<D, S>> shapecast_nearest(const G& g, const ShapeCast<D, S>& cast, S max_toi, const Filter& f) const {
    if (nodes.empty()) return std::nullopt;
    std::optional<Hit<D, S>> best;
    S limit = max_toi;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      S te, tx;
      if (!cast.broadphase(node.bounds, limit, &te, &tx) || !(te <= limit)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t leaf = prim_indices[k];
          if (!g.accepts(leaf, f)) continue;
          LeafHit<D, S> lh;
          if (g.test_shape_cast(leaf, cast, limit, &lh)) {
            Hit<D, S> h{leaf, lh.toi, cast.at(lh.toi), lh.normal, lh.sub};  // naive.rs:114-128
            if (!best || hit_cmp(*best, h) > 0) { limit = h.toi; best = h; }
          }
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    return best;
  }

  // bvh.rs:378-414
  template <class G>
  void shapecast_all(const G& g, const ShapeCast<D, S>& cast, S max_toi, const Filter& f, std::vector<Hit<D, S>>& hits) const {
    hits.clear();
    if (nodes.empty()) return;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      S te, tx;
      if (!cast.broadphase(node.bounds, max_toi, &te, &tx)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t leaf = prim_indices[k];
          if (!g.accepts(leaf, f)) continue;
          LeafHit<D, S> lh;
          if (g.test_shape_cast(leaf, cast, max_toi, &lh))
            hits.push_back(Hit<D, S>{leaf, lh.toi, cast.at(lh.toi), lh.normal, lh.sub});
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    std::stable_sort(hits.begin(), hits.end(), [](const Hit<D, S>& a, const Hit<D, S>& b) { return hit_cmp(a, b) < 0; });
  }

  // bvh.rs:418-456
  template <class G>
  void overlap(const G& g, const Aabb<D, S>& region, const Filter& f, std::vector<uint32_t>& out) const {
    out.clear();
    if (nodes.empty()) return;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      if (!node.bounds.intersects(region)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t leaf = prim_indices[k];
          if (!g.accepts(leaf, f)) continue;
          if (g.test_overlap(leaf, region)) out.push_back(leaf);
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    std::sort(out.begin(), out.end());
  }
};

// query/naive.rs: the O(N) scans the reference checks its BVH against.
namespace naive {
template <int D, class S, class G>
std::optional<Hit<D, S>> nearest(const G& g, const Ray<D, S>& ray, S max_toi, const Filter& f) {  // :34-62
  std::optional<Hit<D, S>> best;
  S limit = max_toi;
  for (size_t leaf = 0; leaf < g.leaf_count(); ++leaf) {
    if (!g.accepts(leaf, f)) continue;
    S te, tx;
    if (!g.world_aabb(leaf).ray_intersect(ray, limit, &te, &tx)) continue;
    LeafHit<D, S> lh;
    if (g.test_ray(leaf, ray, limit, &lh)) {
      Hit<D, S> h{uint32_t(leaf), lh.toi, ray.at(lh.toi), lh.normal, lh.sub};
      if (!best || hit_cmp(*best, h) > 0) { limit = h.toi; best = h; }
    }
  }
  return best;
}
template <int D, class S, class G>
void all(const G& g, const Ray<D, S>& ray, S max_toi, const Filter& f, bool crossings, std::vector<Hit<D, S>>& hits) {  // :65-109
  hits.clear();
  for (size_t leaf = 0; leaf < g.leaf_count(); ++leaf) {
    if (!g.accepts(leaf, f)) continue;
    S te, tx;
    if (!g.world_aabb(leaf).ray_intersect(ray, max_toi, &te, &tx)) continue;
    auto push = [&](const LeafHit<D, S>& lh) { hits.push_back(Hit<D, S>{uint32_t(leaf), lh.toi, ray.at(lh.toi), lh.normal, lh.sub}); };
    if (crossings) g.test_ray_crossings(leaf, ray, max_toi, push);
    else { LeafHit<D, S> lh; if (g.test_ray(leaf, ray, max_toi, &lh)) push(lh); }
  }
  std::stable_sort(hits.begin(), hits.end(), [](const Hit<D, S>& a, const Hit<D, S>& b) { return hit_cmp(a, b) < 0; });
}
template <int D, class S, class G>
std::optional<Hit<D, S>> shapecast_nearest(const G& g, const ShapeCast<D, S>& cast, S max_toi, const Filter& f) {  // :131-158
  std::optional<Hit<D, S>> best;
  S limit = max_toi;
  for (size_t leaf = 0; leaf < g.leaf_count(); ++leaf) {
    if (!g.accepts(leaf, f)) continue;
    S te, tx;
    if (!cast.broadphase(g.world_aabb(leaf), limit, &te, &tx)) continue;
    LeafHit<D, S> lh;
    if (g.test_shape_cast(leaf, cast, limit, &lh)) {
      Hit<D, S> h{uint32_t(leaf), lh.toi, cast.at(lh.toi), lh.normal, lh.sub};
      if (!best || hit_cmp(*best, h) > 0) { limit = h.toi; best = h; }
    }
  }
  return best;
}
template <int D, class S, class G>
void shapecast_all(const G& g, const ShapeCast<D, S>& cast, S max_toi, const Filter& f, std::vector<Hit<D, S>>& hits) {  // :161-181
  hits.clear();
  for (size_t leaf = 0; leaf < g.leaf_count(); ++leaf) {
    if (!g.accepts(leaf, f)) continue;
    S te, tx;
    if (!cast.broadphase(g.world_aabb(leaf), max_toi, &te, &tx)) continue;
    LeafHit<D, S> lh;
    if (g.test_shape_cast(leaf, cast, max_toi, &lh))
      hits.push_back(Hit<D, S>{uint32_t(leaf), lh.toi, cast.at(lh.toi), lh.normal, lh.sub});
  }
  std::stable_sort(hits.begin(), hits.end(), [](const Hit<D, S>& a, const Hit<D, S>& b) { return hit_cmp(a, b) < 0; });
}
template <int D, class S, class G>
void overlap(const G& g, const Aabb<D, S>& region, const Filter& f, std::vector<uint32_t>& out) {  // :184-205
  out.clear();
  for (size_t leaf = 0; leaf < g.leaf_count(); ++leaf) {
    if (!g.accepts(leaf, f)) continue;
    if (!g.world_aabb(leaf).intersects(region)) continue;
    if (g.test_overlap(leaf, region)) out.push_back(uint32_t(leaf));
  }
}
}  // namespace naive

// ---------------------------------------------------------------------------
// Two-level tree (accel/tlas.rs) over instance providers
// (query/instance.rs:19-106).
// ---------------------------------------------------------------------------

enum InstKind : int {
  kInstMesh = 0,   // a scaled, rotated triangle-mesh BLAS (D = 3)
  kInstBox = 1,    // an oriented box [-h, h] (tests/two_level.rs:42-113)
  kInstBall = 2,   // a ball at the local origin (tests/shape_overlap.rs:289-342)
};

// Ray against the local box [-half, half] (tests/two_level.rs:70-113).
template <int D, class S>
inline bool ray_local_box(const Ray<D, S>& ray, const Point<D, S>& half, S max_toi, LeafHit<D, S>* out) {
  S t_min = S(0), t_max = max_toi;
  int axis = -1;
  for (int i = 0; i < D; ++i) {
    S o = ray.origin[i], d = ray.dir[i];
    if (std::fabs(d) < S(1.0e-9)) {
      if (o < -half[i] || o > half[i]) return false;
    } else {
      S inv = S(1) / d;
      S t1 = (-half[i] - o) * inv;
      S t2 = (half[i] - o) * inv;
      if (t1 > t2) std::swap(t1, t2);
      if (t1 > t_min) { t_min = t1; axis = i; }
      if (t2 < t_max) t_max = t2;
      if (t_min > t_max) return false;
    }
  }
  if (!(axis >= 0 && t_min > S(1.0e-6) && t_min <= max_toi)) return false;
  out->toi = t_min;
  out->normal = entry_normal(ray.dir, axis);
  out->sub = kNoSub;
  return true;
}

// A BLAS: one triangle soup with its own Bvh.
template <class S> struct Blas {
  Scene<3, S> soup;
  Bvh<3, S> bvh;
  Aabb<3, S> aabb;  // the root bounds (EMPTY for an empty mesh)
};

template <int D, class S> struct InstScene {
  int kind = kInstBall;
  std::vector<Isometry<D, S>> iso;
  std::vector<S> param;          // per instance: scale (mesh), half-extents (box, D), radius (ball)
  std::vector<uint32_t> blas_id;  // mesh instances
  const std::vector<Blas<S>>* blas = nullptr;
  std::vector<uint64_t> layers;
  std::vector<uint32_t> sub;  // per-instance sub-object for box/ball kinds (empty: none)
  LayerAccept acc;

  size_t instance_count() const { return iso.size(); }
  bool accepts(size_t i, const Filter& f) const { return acc.accepts(i, f); }
  const Isometry<D, S>& transform(size_t i) const { return iso[i]; }
  uint32_t sub_of(size_t i) const { return sub.empty() ? kNoSub : sub[i]; }

  Aabb<D, S> local_aabb(size_t i) const {
    if (kind == kInstBox) {
      Point<D, S> h; for (int k = 0; k < D; ++k) h[k] = param[i * D + k];
      return Aabb<D, S>{-h, h};  // two_level.rs:60-62
    }
    if (kind == kInstBall) {
      S r = param[i];
      return Aabb<D, S>{Point<D, S>::splat(-r), Point<D, S>::splat(r)};
    }
    // Mesh: the mesh AABB scaled by s (s > 0).
    Aabb<D, S> a;
    if constexpr (D == 3) {
      const Blas<S>& b = (*blas)[blas_id[i]];
      S s = param[i];
      a.min = b.aabb.min * s;
      a.max = b.aabb.max * s;
    }
    return a;
  }

  bool test_ray_local(size_t i, const Ray<D, S>& lr, S max_toi, LeafHit<D, S>* out) const {
    if (kind == kInstBox) {
      Point<D, S> h; for (int k = 0; k < D; ++k) h[k] = param[i * D + k];
      return ray_local_box(lr, h, max_toi, out);
    }
    if (kind == kInstBall) {
      S t; Point<D, S> n;
      if (!ray_ball(lr, Point<D, S>::zero(), param[i], max_toi, true, &t, &n)) return false;
      out->toi = t; out->normal = n; out->sub = sub_of(i);
      return true;
    }
    if constexpr (D == 3) {
      // Scaled mesh: traverse the mesh Bvh in unscaled mesh space with the
      // origin divided by s and max_toi / s, and scale the toi back.
      const Blas<S>& b = (*blas)[blas_id[i]];
      S s = param[i];
      Ray<3, S> ms;
      for (int k = 0; k < 3; ++k) ms.origin[k] = lr.origin[k] / s;
      ms.dir = lr.dir;
      auto h = b.bvh.nearest(b.soup, ms, max_toi / s, Filter{}, nullptr);
      if (!h) return false;
      S toi = h->toi * s;
      if (toi > max_toi) return false;
      out->toi = toi;
      out->normal = h->normal;
      out->sub = h->leaf;  // the face within the mesh
      return true;
    }
    return false;
  }

  template <class F> void test_ray_crossings_local(size_t i, const Ray<D, S>& lr, S max_toi, F&& out) const {
    if (kind == kInstBall) {  // tests/crossings.rs:679-694
      S t0, t1;
      if (!sphere_roots(lr, Point<D, S>::zero(), param[i], &t0, &t1)) return;
      for (S t : {t0, t1}) {
        if (t >= S(0) && t <= max_toi) {
          LeafHit<D, S> lh; lh.toi = t; lh.normal = lr.at(t).normalize_or_zero(); lh.sub = sub_of(i);
          out(lh);
        }
      }
      return;
    }
    LeafHit<D, S> lh;
    if (test_ray_local(i, lr, max_toi, &lh)) out(lh);
  }

  Aabb<D, S> world_aabb(size_t i) const { return iso[i].transform_aabb(local_aabb(i)); }

  bool test_shape_cast(size_t i, const ShapeCast<D, S>& cast, S max_toi, LeafHit<D, S>* out) const {
    if (kind == kInstBall) {  // shape_overlap.rs:326-338
      Point<D, S> c = iso[i].translation;
      S sum = param[i] + cast.aabb.max[0];
      Ray<D, S> r{cast.origin, cast.dir};
      S t; Point<D, S> n;
      if (!ray_ball(r, c, sum, max_toi, true, &t, &n)) return false;
      out->toi = t; out->normal = (cast.at(t) - c).normalize_or_zero(); out->sub = sub_of(i);
      return true;
    }
    if (kind == kInstMesh) {
      // Swept box against the instance's world AABB (the reference defines no
      // swept-box vs mesh test).
      S t0, t1; int axis;
      if (!cast.broadphase(world_aabb(i), max_toi, &t0, &t1, &axis)) return false;
      out->toi = t0; out->normal = entry_normal(cast.dir, axis); out->sub = kNoSub;
      return true;
    }
    return false;  // instance.rs:264-271 default
  }

  bool test_overlap(size_t i, const Aabb<D, S>& region) const {
    if (kind == kInstBall) return point_to_aabb(iso[i].translation, region) <= param[i];  // :339-341
    if (kind == kInstMesh) return world_aabb(i).intersects(region);  // AABB-level answer
    return true;  // instance.rs:280-282 default (tests/two_level.rs boxes keep it)
  }
};

template <int D, class S> struct Tlas {
  std::vector<Node<D, S>> nodes;
  std::vector<uint32_t> indices;
  std::vector<Aabb<D, S>> world;
  S baseline = S(0);

  template <class I> void build(const I& sc) {  // tlas.rs:35-45
    world.resize(sc.instance_count());
    for (size_t i = 0; i < world.size(); ++i) world[i] = sc.transform(i).transform_aabb(sc.local_aabb(i));
    tree_build(world, nodes, indices);
    baseline = interior_surface_sum(nodes);
  }
  template <class I> void refit(const I& sc) {  // tlas.rs:49-54
    for (size_t i = 0; i < world.size(); ++i) world[i] = sc.transform(i).transform_aabb(sc.local_aabb(i));
    tree_refit(nodes, indices, world);
  }
  bool needs_rebuild(S factor) const {  // tlas.rs:58-60
    return baseline > S(0) && interior_surface_sum(nodes) > factor * baseline;
  }

  // tlas.rs:459-481
  template <class I>
  static bool test_instance(const I& sc, size_t i, const Ray<D, S>& ray, S max_toi, Hit<D, S>* out) {
    const Isometry<D, S>& iso = sc.transform(i);
    Ray<D, S> local{iso.inverse_transform_point(ray.origin), iso.inverse_transform_vector(ray.dir)};
    LeafHit<D, S> lh;
    if (!sc.test_ray_local(i, local, max_toi, &lh)) return false;
    *out = Hit<D, S>{uint32_t(i), lh.toi, ray.at(lh.toi), iso.transform_vector(lh.normal), lh.sub};
    return true;
  }

  template <class I>
  std::optional<Hit<D, S>> nearest(const I& sc, const Ray<D, S>& ray, S max_toi, const Filter& f, QueryStats* st) const {
    // tlas.rs:104-154
    if (nodes.empty()) return std::nullopt;
    std::optional<Hit<D, S>> best;
    S limit = max_toi;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      if (st) { st->nodes_visited++; st->aabb_tests++; }
      S te, tx;
      if (!node.bounds.ray_intersect(ray, limit, &te, &tx) || !(te <= limit)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t i = indices[k];
          if (!sc.accepts(i, f)) continue;
          if (st) st->narrow_tests++;
          Hit<D, S> h;
          if (test_instance(sc, i, ray, limit, &h)) {
            if (st) st->hits++;
            if (!best || hit_cmp(*best, h) > 0) { limit = h.toi; best = h; }
          }
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    return best;
  }

  template <class I>
  void all(const I& sc, const Ray<D, S>& ray, S max_toi, const Filter& f, bool crossings, std::vector<Hit<D, S>>& hits,
           QueryStats* st) const {
    // tlas.rs:180-221 and 249-303
    hits.clear();
    if (nodes.empty()) return;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      if (st) { st->nodes_visited++; st->aabb_tests++; }
      S te, tx;
      if (!node.bounds.ray_intersect(ray, max_toi, &te, &tx)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t i = indices[k];
          if (!sc.accepts(i, f)) continue;
          if (st) st->narrow_tests++;
          if (crossings) {
            const Isometry<D, S>& iso = sc.transform(i);
            Ray<D, S> local{iso.inverse_transform_point(ray.origin), iso.inverse_transform_vector(ray.dir)};
            sc.test_ray_crossings_local(i, local, max_toi, [&](const LeafHit<D, S>& lh) {
              if (st) st->hits++;
              hits.push_back(Hit<D, S>{i, lh.toi, ray.at(lh.toi), iso.transform_vector(lh.normal), lh.sub});
            });
          } else {
            Hit<D, S> h;
            if (test_instance(sc, i, ray, max_toi, &h)) { if (st) st->hits++; hits.push_back(h); }
          }
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    std::stable_sort(hits.begin(), hits.end(), [](const Hit<D, S>& a, const Hit<D, S>& b) { return hit_cmp(a, b) < 0; });
  }

  template <class I>
  std::optional<Hit<D, S>> shapecast_nearest(const I& sc, const ShapeCast<D, S>& cast, S max_toi, const Filter& f) const {
    // tlas.rs:306-349 + shapecast_instance :437-452
    if (nodes.empty()) return std::nullopt;
    std::optional<Hit<D, S>> best;
    S limit = max_toi;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      S te, tx;
      if (!cast.broadphase(node.bounds, limit, &te, &tx) || !(te <= limit)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t i = indices[k];
          if (!sc.accepts(i, f)) continue;
          LeafHit<D, S> lh;
          if (sc.test_shape_cast(i, cast, limit, &lh)) {
            Hit<D, S> h{i, lh.toi, cast.at(lh.toi), lh.normal, lh.sub};
            if (!best || hit_cmp(*best, h) > 0) { limit = h.toi; best = h; }
          }
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    return best;
  }

  template <class I>
  void shapecast_all(const I& sc, const ShapeCast<D, S>& cast, S max_toi, const Filter& f, std::vector<Hit<D, S>>& hits) const {
    // tlas.rs:353-389
    hits.clear();
    if (nodes.empty()) return;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      S te, tx;
      if (!cast.broadphase(node.bounds, max_toi, &te, &tx)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t i = indices[k];
          if (!sc.accepts(i, f)) continue;
          LeafHit<D, S> lh;
          if (sc.test_shape_cast(i, cast, max_toi, &lh)) hits.push_back(Hit<D, S>{i, lh.toi, cast.at(lh.toi), lh.normal, lh.sub});
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    std::stable_sort(hits.begin(), hits.end(), [](const Hit<D, S>& a, const Hit<D, S>& b) { return hit_cmp(a, b) < 0; });
  }

  template <class I>
  void overlap(const I& sc, const Aabb<D, S>& region, const Filter& f, std::vector<uint32_t>& out) const {
    // tlas.rs:393-431
    out.clear();
    if (nodes.empty()) return;
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t ni = stack.back(); stack.pop_back();
      const Node<D, S> node = nodes[ni];
      if (!node.bounds.intersects(region)) continue;
      if (node.is_leaf()) {
        for (uint32_t k = node.child_a; k < node.child_a + node.prim_count; ++k) {
          uint32_t i = indices[k];
          if (!sc.accepts(i, f)) continue;
          if (sc.test_overlap(i, region)) out.push_back(i);
        }
      } else {
        stack.push_back(node.child_a);
        stack.push_back(node.child_b);
      }
    }
    std::sort(out.begin(), out.end());
  }
};

// The naive instance scans of tests/two_level.rs:134-174 (no AABB reject).
template <int D, class S, class I>
std::optional<Hit<D, S>> inst_naive_nearest(const I& sc, const Ray<D, S>& ray, S max_toi, const Filter& f) {
  std::optional<Hit<D, S>> best;
  for (size_t i = 0; i < sc.instance_count(); ++i) {
    if (!sc.accepts(i, f)) continue;
    Hit<D, S> h;
    if (Tlas<D, S>::test_instance(sc, i, ray, max_toi, &h))
      if (!best || hit_cmp(*best, h) > 0) best = h;
  }
  return best;
}

// Fixed-order parallel batch (bvh.rs:160-193): contiguous chunks, one per
// worker, each writing only its own slice.
template <class F> void parallel_chunks(size_t n, int threads, F&& body) {
  size_t workers = std::max<size_t>(1, std::min<size_t>(size_t(std::max(threads, 1)), std::max<size_t>(n, 1)));
  if (workers == 1) { body(size_t(0), n); return; }
  size_t chunk = (n + workers - 1) / workers;
  std::vector<std::thread> ts;
  for (size_t s = 0; s < n; s += chunk) ts.emplace_back([&, s] { body(s, std::min(n, s + chunk)); });
  for (auto& t : ts) t.join();
}

}  // namespace orc
