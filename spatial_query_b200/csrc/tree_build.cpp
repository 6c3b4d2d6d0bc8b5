// Host median-split tree build: tree::build (crates/spatial-query/src/accel/
// tree.rs:39-49, 112-163) for callers that do not run the Rust crate.
//
// The output is the crate's tree exactly: preorder node array, root at 0, a
// leaf holds <= 4 primitives unless all its centroids coincide, the split axis
// is the first longest axis of the centroid bounds, primitives are ordered by
// a stable sort on that centroid coordinate under f32::total_cmp and split at
// start + count / 2. Differences from the reference are in how, not what:
// centroid sort keys are computed once per axis as integers, and the two
// halves of the upper levels are built on separate threads into their own
// arrays and spliced back in preorder.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <future>
#include <thread>
#include <vector>

#include "../../include/sq.h"

namespace {

constexpr uint32_t kLeafSize = 4;

// The scalar of the build: float (the crate's default) or double (its f64
// feature): EPSILON and the f32 / f64 total_cmp key.
template <class S> struct Sc;
template <> struct Sc<float> {
  static constexpr float eps = 1.1920928955078125e-7f;
  using Key = int32_t;
  static Key key(float x) {
    int32_t b;
    std::memcpy(&b, &x, 4);
    return b ^ int32_t(uint32_t(b >> 31) >> 1);
  }
};
template <> struct Sc<double> {
  static constexpr double eps = 2.220446049250313080847e-16;
  using Key = int64_t;
  static Key key(double x) {
    int64_t b;
    std::memcpy(&b, &x, 8);
    return b ^ int64_t(uint64_t(b >> 63) >> 1);
  }
};

template <class S> struct BNode {
  S lo[8], hi[8];
  uint32_t a, b, cnt;
};

template <class S> struct Builder {
  using BNode = ::BNode<S>;
  using Key = typename Sc<S>::Key;
  int D;
  uint32_t n;
  const S* aabbs;
  std::vector<S> cent;      // n * D
  std::vector<Key> keys;    // D * n
  std::vector<uint32_t> idx;
  int par_depth;

  void bounds_of(uint32_t s, uint32_t e, S* lo, S* hi) const {
    for (int i = 0; i < D; ++i) { lo[i] = INFINITY; hi[i] = -INFINITY; }
    for (uint32_t k = s; k < e; ++k) {
      const S* b = aabbs + size_t(idx[k]) * 2 * D;
      for (int i = 0; i < D; ++i) {
        lo[i] = std::fmin(lo[i], b[i]);
        hi[i] = std::fmax(hi[i], b[D + i]);
      }
    }
  }

  // Builds the subtree over idx[s, e) appending nodes (indices local to
  // `out`, offset by `base`) and returns nothing; the subtree root is at
  // out[first].
  void build(uint32_t s, uint32_t e, std::vector<BNode>& out, uint32_t base, int depth) {
    BNode nd;
    bounds_of(s, e, nd.lo, nd.hi);
    const uint32_t me = uint32_t(out.size());
    const uint32_t count = e - s;
    nd.a = s;
    nd.b = 0;
    nd.cnt = count;
    out.push_back(nd);
    if (count <= kLeafSize) return;
    S clo[8], chi[8];
    for (int i = 0; i < D; ++i) { clo[i] = INFINITY; chi[i] = -INFINITY; }
    for (uint32_t k = s; k < e; ++k) {
      const S* c = cent.data() + size_t(idx[k]) * D;
      for (int i = 0; i < D; ++i) {
        clo[i] = std::fmin(clo[i], c[i]);
        chi[i] = std::fmax(chi[i], c[i]);
      }
    }
    int axis = 0;
    S ext[8];
    for (int i = 0; i < D; ++i) ext[i] = chi[i] - clo[i];
    for (int i = 1; i < D; ++i) if (ext[i] > ext[axis]) axis = i;
    if (ext[axis] <= Sc<S>::eps) return;
    const Key* key = keys.data() + size_t(axis) * n;
    std::stable_sort(idx.begin() + s, idx.begin() + e, [key](uint32_t x, uint32_t y) { return key[x] < key[y]; });
    const uint32_t mid = s + count / 2;
    uint32_t ca, cb;
    if (depth < par_depth && count > 4096) {
      std::vector<BNode> left, right;
      auto fut = std::async(std::launch::async, [&] { build(s, mid, left, 0, depth + 1); });
      build(mid, e, right, 0, depth + 1);
      fut.get();
      ca = base + me + 1;
      cb = ca + uint32_t(left.size());
      auto splice = [&](std::vector<BNode>& v, uint32_t off) {
        for (BNode& x : v) {
          if (x.cnt == 0) { x.a += off; x.b += off; }
          out.push_back(x);
        }
      };
      splice(left, ca);
      splice(right, cb);
    } else {
      ca = base + uint32_t(out.size());
      build(s, mid, out, base, depth + 1);
      cb = base + uint32_t(out.size());
      build(mid, e, out, base, depth + 1);
    }
    out[me].a = ca;
    out[me].b = cb;
    out[me].cnt = 0;
  }
};

template <class S>
int32_t tree_build_impl(int32_t dim, uint32_t n, const S* prim_aabbs, int32_t threads, uint32_t node_capacity,
                        uint32_t* n_nodes_out, S* node_bounds, uint32_t* child_a, uint32_t* child_b,
                        uint32_t* prim_count, uint32_t* prim_indices) {
  if (dim < 1 || dim > 8 || !n_nodes_out) return SQ_ERR_INVALID;
  *n_nodes_out = 0;
  if (n == 0) return SQ_OK;
  if (!prim_aabbs || !node_bounds || !child_a || !child_b || !prim_count || !prim_indices) return SQ_ERR_INVALID;
  if (uint64_t(node_capacity) < 2ull * n - 1) return SQ_ERR_CAPACITY;
  Builder<S> B;
  B.D = dim;
  B.n = n;
  B.aabbs = prim_aabbs;
  B.cent.resize(size_t(n) * dim);
  B.keys.resize(size_t(n) * dim);
  B.idx.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    B.idx[i] = i;
    const S* b = prim_aabbs + size_t(i) * 2 * dim;
    for (int k = 0; k < dim; ++k) {
      S c = (b[k] + b[dim + k]) * S(0.5);  // Aabb::center (aabb.rs:56-58)
      B.cent[size_t(i) * dim + k] = c;
      B.keys[size_t(k) * n + i] = Sc<S>::key(c);
    }
  }
  int t = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
  int pd = 0;
  while ((1 << pd) < t && pd < 8) ++pd;
  B.par_depth = pd;
  std::vector<BNode<S>> nodes;
  nodes.reserve(size_t(2) * n);
  B.build(0, n, nodes, 0, 0);
  if (nodes.size() > node_capacity) return SQ_ERR_CAPACITY;
  for (size_t i = 0; i < nodes.size(); ++i) {
    for (int k = 0; k < dim; ++k) {
      node_bounds[i * 2 * dim + k] = nodes[i].lo[k];
      node_bounds[i * 2 * dim + dim + k] = nodes[i].hi[k];
    }
    child_a[i] = nodes[i].a;
    child_b[i] = nodes[i].b;
    prim_count[i] = nodes[i].cnt;
  }
  std::memcpy(prim_indices, B.idx.data(), size_t(n) * 4);
  *n_nodes_out = uint32_t(nodes.size());
  return SQ_OK;
}

}  // namespace

extern "C" int32_t sq_tree_build(int32_t dim, uint32_t n, const float* prim_aabbs, int32_t threads,
                                 uint32_t node_capacity, uint32_t* n_nodes_out, float* node_bounds,
                                 uint32_t* child_a, uint32_t* child_b, uint32_t* prim_count,
                                 uint32_t* prim_indices) {
  return tree_build_impl<float>(dim, n, prim_aabbs, threads, node_capacity, n_nodes_out, node_bounds, child_a,
                                child_b, prim_count, prim_indices);
}

extern "C" int32_t sq_tree_build_f64(int32_t dim, uint32_t n, const double* prim_aabbs, int32_t threads,
                                     uint32_t node_capacity, uint32_t* n_nodes_out, double* node_bounds,
                                     uint32_t* child_a, uint32_t* child_b, uint32_t* prim_count,
                                     uint32_t* prim_indices) {
  return tree_build_impl<double>(dim, n, prim_aabbs, threads, node_capacity, n_nodes_out, node_bounds, child_a,
                                 child_b, prim_count, prim_indices);
}

template <class S>
static int32_t prim_aabbs_impl(int32_t dim, int32_t narrow, uint32_t n, const S* prim_data, S* out) {
  if (dim < 1 || dim > 8 || (n && (!prim_data || !out))) return SQ_ERR_INVALID;
  for (uint32_t i = 0; i < n; ++i) {
    S* o = out + size_t(i) * 2 * dim;
    if (narrow == SQ_NARROW_AABB) {
      std::memcpy(o, prim_data + size_t(i) * 2 * dim, sizeof(S) * 2 * dim);
    } else if (narrow == SQ_NARROW_SPHERE || narrow == SQ_NARROW_SPHERE_NEAR) {
      const S* p = prim_data + size_t(i) * (dim + 1);
      for (int k = 0; k < dim; ++k) {  // c - splat(r), c + splat(r)
        o[k] = p[k] - p[dim];
        o[dim + k] = p[k] + p[dim];
      }
    } else if (narrow == SQ_NARROW_TRIANGLE) {
      if (dim != 3) return SQ_ERR_INVALID;
      const S* p = prim_data + size_t(i) * 9;
      for (int k = 0; k < 3; ++k) {  // Aabb::EMPTY grown by each vertex
        S lo = S(INFINITY), hi = S(-INFINITY);
        for (int v = 0; v < 3; ++v) {
          lo = std::fmin(lo, p[3 * v + k]);
          hi = std::fmax(hi, p[3 * v + k]);
        }
        o[k] = lo;
        o[3 + k] = hi;
      }
    } else {
      return SQ_ERR_INVALID;
    }
  }
  return SQ_OK;
}

extern "C" int32_t sq_prim_aabbs(int32_t dim, int32_t narrow, uint32_t n, const float* prim_data, float* out) {
  return prim_aabbs_impl<float>(dim, narrow, n, prim_data, out);
}

extern "C" int32_t sq_prim_aabbs_f64(int32_t dim, int32_t narrow, uint32_t n, const double* prim_data, double* out) {
  return prim_aabbs_impl<double>(dim, narrow, n, prim_data, out);
}
