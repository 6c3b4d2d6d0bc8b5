// The crate's f64 feature on the device (Scalar = f64, maths/point.rs:14-18):
// nearest rays against an f64 scene, for consumers whose coordinates need
// double precision (large worlds) or who compare against an f64 CPU build.
//
// The walk is Bvh::raycast_nearest_impl (accel/bvh.rs:73-124) as written: a
// stack of node indices seeded with the root; a popped node is tested with
// Aabb::ray_intersect against the current limit; a leaf tests its accepted
// primitives in prim_indices order with the limit, keeping the first hit in
// hit_ordering and shrinking the limit to it; an interior node pushes
// child_a then child_b. All arithmetic is the f64 form of the f32 kernels'
// (sq_math.cuh with S = double), so answers and QueryStats counters equal the
// f64 CPU path's bit for bit. One thread per ray; the node boxes and links
// are the host tree's nodes as they are (no child-pair records).
//
// The crate's other queries take the same walk on f64 scenes (walk64_kernel):
// raycast_all and raycast_crossings (bvh.rs:196-328: no limit shrink, hits
// kept in hit_ordering, bounded to k per ray with the full count),
// shapecast_nearest / shapecast_all (bvh.rs:330-414: the node test is
// ShapeCast::broadphase, the slab against the box grown by the probe) and
// overlap (bvh.rs:416-456: Aabb::intersects per node, CSR output with each
// region's leaves ascending).
#include <cub/cub.cuh>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "sq_internal.cuh"

using namespace sq;
using sqi::cuda_fail;
using sqi::fail;

namespace {

constexpr int kStack64 = kMaxStack;  // deepest tree accepted, as for f32 scenes

struct Params64 {
  const double* nb;    // [n_nodes][2D]
  const uint2* nc;     // [n_nodes]
  const double* prims; // [n_prims][stride], leaf order
  const uint32_t* ids; // [n_prims]: leaf id at each position
  const uint64_t* layers;
  uint64_t mask;
  long long exclude;
  uint32_t stride;
  const double* rays;  // [n][2D]
  uint32_t n;
  double max_toi;
  const double* max_toi_arr;
  uint32_t* out_leaf;
  double* out_toi;
  double* out_normal;
  unsigned long long* stats;  // nodes, aabb tests, narrow tests, hits (summed)
  // walk64_kernel: queries (rays o,d; casts o,d,probe.min,probe.max; regions lo,hi)
  uint32_t k;                 // list capacity per query
  int crossings;              // raycast_crossings: both roots of sphere leaves
  uint32_t* out_count;        // lists: full count; overlap count pass: results per region
  const unsigned long long* csr_offsets;  // overlap fill pass
  uint32_t* csr_leaves;
};

template <int D, int N>
__device__ __forceinline__ bool narrow64(const double* rec, const RayPre<D, double>& r, double limit, double& t,
                                         double* n) {
  if constexpr (N == kNarrowAabb) {
    int axis;
    if (!slab<D>(r, rec, rec + D, limit, t, axis)) return false;
    entry_normal<D>(r.d, axis, n);
    return true;
  } else if constexpr (N == kNarrowSphere || N == kNarrowSphereNear) {
    return ray_ball<D, N == kNarrowSphere>(r.o, r.d, rec, rec[D], limit, t, n);
  } else {
    if (!ray_triangle(r.o, r.d, rec, rec + 3, rec + 6, t)) return false;
    if (t > limit) return false;
    tri_normal(rec, rec + 3, rec + 6, n);
    return true;
  }
}

template <int D, int N, bool STATS>
__global__ void __launch_bounds__(128) nearest64_kernel(const Params64 p) {
  unsigned long long c_nodes = 0, c_nar = 0, c_hit = 0;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < p.n; q += gridDim.x * blockDim.x) {
    RayPre<D, double> r;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      r.o[i] = p.rays[size_t(q) * 2 * D + i];
      r.d[i] = p.rays[size_t(q) * 2 * D + D + i];
    }
    ray_prep(r);
    double limit = p.max_toi_arr ? p.max_toi_arr[q] : p.max_toi;
    uint32_t best = kNoHit;
    double best_t = 0.0, best_n[D];
#pragma unroll
    for (int i = 0; i < D; ++i) best_n[i] = 0.0;
    uint32_t stack[kStack64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const uint32_t ni = stack[--sp];
      if (STATS) ++c_nodes;
      double te;
      int ax;
      const double* nb = p.nb + size_t(ni) * 2 * D;
      if (!slab<D>(r, nb, nb + D, limit, te, ax) || !(te <= limit)) continue;
      const uint2 c = p.nc[ni];
      if (c.y & kLeafBit) {
        const uint32_t end = c.x + (c.y & ~kLeafBit);
        for (uint32_t pos = c.x; pos < end; ++pos) {
          const uint32_t id = p.ids[pos];
          if (p.layers && ((p.exclude >= 0 && (unsigned long long)p.exclude == id) || !(p.layers[id] & p.mask)))
            continue;
          if (STATS) ++c_nar;
          double t, nrm[D];
          if (narrow64<D, N>(p.prims + size_t(pos) * p.stride, r, limit, t, nrm)) {
            if (STATS) ++c_hit;
            if (best == kNoHit || hit_before(t, id, best_t, best)) {
              best = id;
              best_t = t;
              limit = t;
#pragma unroll
              for (int i = 0; i < D; ++i) best_n[i] = nrm[i];
            }
          }
        }
      } else if (sp + 2 <= kStack64) {  // the upload bounds the depth, so this always holds
        stack[sp++] = c.x;
        stack[sp++] = c.y;
      }
    }
    p.out_leaf[q] = best;
    if (p.out_toi) p.out_toi[q] = best_t;
    if (p.out_normal) {
#pragma unroll
      for (int i = 0; i < D; ++i) p.out_normal[size_t(q) * D + i] = best_n[i];
    }
  }
  if (STATS && p.stats) {
    atomicAdd(p.stats + 0, c_nodes);
    atomicAdd(p.stats + 1, c_nodes);  // one box test per visited node (bvh.rs:91-92)
    atomicAdd(p.stats + 2, c_nar);
    atomicAdd(p.stats + 3, c_hit);
  }
}

// One primitive's swept-probe test (QueryGeometry::test_shape_cast of the
// built-in providers, as the f32 kernels answer it): boxes the grown slab,
// balls the ray against the ball grown by probe.max[0], triangles the grown
// slab against the triangle's AABB.
template <int D, int N>
__device__ __forceinline__ bool cast64(const double* rec, const RayPre<D, double>& r, const double* pmin,
                                       const double* pmax, double limit, double& t, double* n) {
  if constexpr (N == kNarrowAabb) {
    int axis;
    if (!slab_grown<D>(r, rec, rec + D, pmin, pmax, limit, t, axis)) return false;
    entry_normal<D>(r.d, axis, n);
    return true;
  } else if constexpr (N == kNarrowSphere || N == kNarrowSphereNear) {
    return ray_ball<D, N == kNarrowSphere>(r.o, r.d, rec, sq::fadd(rec[D], pmax[0]), limit, t, n);
  } else {
    double lo[3], hi[3];
    tri_aabb(rec, rec + 3, rec + 6, lo, hi);
    int axis;
    if (!slab_grown<3>(r, lo, hi, pmin, pmax, limit, t, axis)) return false;
    entry_normal<3>(r.d, axis, n);
    return true;
  }
}

// One primitive's overlap test (QueryGeometry::test_overlap).
template <int D, int N>
__device__ __forceinline__ bool overlap64(const double* rec, const double* qlo, const double* qhi) {
  if constexpr (N == kNarrowAabb) {
    return box_overlap<D>(rec, rec + D, qlo, qhi);
  } else if constexpr (N == kNarrowSphere || N == kNarrowSphereNear) {
    double d2 = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const double c = rec[i];
      const double v = (c < qlo[i]) ? sq::fsub(qlo[i], c) : ((c > qhi[i]) ? sq::fsub(c, qhi[i]) : 0.0);
      d2 = sq::fadd(d2, sq::fmul(v, v));
    }
    return sq::fsqrt(d2) <= rec[D];
  } else {
    double lo[3], hi[3];
    tri_aabb(rec, rec + 3, rec + 6, lo, hi);
    return box_overlap<3>(lo, hi, qlo, qhi);
  }
}

// Sorted insertion into query q's bounded list (hit_ordering; an equal key
// goes after the entries already there). `count` is the full number so far.
template <int D>
__device__ __forceinline__ void put64(const Params64& p, uint32_t q, uint32_t& count, double t, uint32_t leaf,
                                      const double* n) {
  uint32_t m = count < p.k ? count : p.k;
  ++count;
  if (p.k == 0) return;
  const size_t base = size_t(q) * p.k;
  uint32_t* ol = p.out_leaf;
  double* ot = p.out_toi;
  double* on = p.out_normal;
  if (m == p.k) {
    if (!hit_before(t, leaf, ot[base + p.k - 1], ol[base + p.k - 1])) return;
    m = p.k - 1;
  }
  uint32_t j = m;
  while (j > 0 && hit_before(t, leaf, ot[base + j - 1], ol[base + j - 1])) {
    ot[base + j] = ot[base + j - 1];
    ol[base + j] = ol[base + j - 1];
    if (on)
#pragma unroll
      for (int i = 0; i < D; ++i) on[(base + j) * D + i] = on[(base + j - 1) * D + i];
    --j;
  }
  ot[base + j] = t;
  ol[base + j] = leaf;
  if (on)
#pragma unroll
    for (int i = 0; i < D; ++i) on[(base + j) * D + i] = n[i];
}

// The crate's walk (push child_a, push child_b; pop, test the node against
// the query, open a leaf) for lists, casts and overlap on an f64 scene.
// K: kRayAll (p.crossings: raycast_crossings), kCastNearest, kCastAll,
// kOverlap (p.csr_leaves null: count pass; else fill in walk order).
template <int D, int N, int K>
__global__ void __launch_bounds__(128) walk64_kernel(const Params64 p) {
  constexpr bool kCast = (K == kCastNearest || K == kCastAll);
  constexpr int QW = kCast ? 4 * D : 2 * D;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < p.n; q += gridDim.x * blockDim.x) {
    const double* src = p.rays + size_t(q) * QW;
    RayPre<D, double> r;
    double pmin[D], pmax[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      r.o[i] = src[i];
      r.d[i] = src[D + i];
      if constexpr (kCast) {
        pmin[i] = src[2 * D + i];
        pmax[i] = src[3 * D + i];
      } else {
        pmin[i] = pmax[i] = 0.0;
      }
    }
    if constexpr (K != kOverlap) ray_prep(r);
    double limit = p.max_toi_arr ? p.max_toi_arr[q] : p.max_toi;
    uint32_t best = kNoHit, count = 0;
    double best_t = 0.0, best_n[D];
#pragma unroll
    for (int i = 0; i < D; ++i) best_n[i] = 0.0;
    const unsigned long long csr_base = (K == kOverlap && p.csr_leaves) ? p.csr_offsets[q] : 0ull;
    uint32_t stack[kStack64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const uint32_t ni = stack[--sp];
      const double* nb = p.nb + size_t(ni) * 2 * D;
      if constexpr (K == kOverlap) {
        if (!box_overlap<D>(nb, nb + D, r.o, r.d)) continue;  // region lo / hi sit in o / d
      } else {
        double te;
        int ax;
        bool geo;
        if constexpr (kCast) geo = slab_grown<D>(r, nb, nb + D, pmin, pmax, limit, te, ax);
        else geo = slab<D>(r, nb, nb + D, limit, te, ax);
        if (!geo || !(te <= limit)) continue;
      }
      const uint2 c = p.nc[ni];
      if (!(c.y & kLeafBit)) {
        if (sp + 2 <= kStack64) {  // the upload bounds the depth, so this always holds
          stack[sp++] = c.x;
          stack[sp++] = c.y;
        }
        continue;
      }
      const uint32_t end = c.x + (c.y & ~kLeafBit);
      for (uint32_t pos = c.x; pos < end; ++pos) {
        const uint32_t id = p.ids[pos];
        if (p.layers && ((p.exclude >= 0 && (unsigned long long)p.exclude == id) || !(p.layers[id] & p.mask)))
          continue;
        const double* rec = p.prims + size_t(pos) * p.stride;
        double t, nrm[D];
        if constexpr (K == kOverlap) {
          if (overlap64<D, N>(rec, r.o, r.d)) {
            if (p.csr_leaves) p.csr_leaves[csr_base + count] = id;
            ++count;
          }
        } else if constexpr (K == kCastNearest) {
          if (cast64<D, N>(rec, r, pmin, pmax, limit, t, nrm) &&
              (best == kNoHit || hit_before(t, id, best_t, best))) {
            best = id;
            best_t = t;
            limit = t;
#pragma unroll
            for (int i = 0; i < D; ++i) best_n[i] = nrm[i];
          }
        } else if constexpr (K == kCastAll) {
          if (cast64<D, N>(rec, r, pmin, pmax, limit, t, nrm)) put64<D>(p, q, count, t, id, nrm);
        } else {  // kRayAll
          bool listed = false;
          // Both roots for the ball whose test reports the far root from
          // inside (tests/crossings.rs:505-521); the near-root-only ball lists
          // one crossing per hit, as the f32 kernels do.
          if constexpr (N == kNarrowSphere) {
            if (p.crossings) {
              // Both roots of the unbounded ray (tests/crossings.rs:505-521).
              listed = true;
              double oc[D];
#pragma unroll
              for (int i = 0; i < D; ++i) oc[i] = sq::fsub(r.o[i], rec[i]);
              const double b = pdot<D>(oc, r.d);
              const double disc = sq::fsub(sq::fmul(b, b), sq::fsub(pdot<D>(oc, oc), sq::fmul(rec[D], rec[D])));
              if (!(disc < 0.0)) {
                const double sq = sq::fsqrt(disc);
                const double roots[2] = {sq::fsub(-b, sq), sq::fadd(-b, sq)};
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                  const double tt = roots[j];
                  if (tt >= 0.0 && tt <= limit) {
                    double pt[D];
                    ray_at<D>(r.o, r.d, tt, pt);
#pragma unroll
                    for (int i = 0; i < D; ++i) nrm[i] = sq::fsub(pt[i], rec[i]);
                    normalize_or_zero<D>(nrm);
                    put64<D>(p, q, count, tt, id, nrm);
                  }
                }
              }
            }
          }
          if (!listed && narrow64<D, N>(rec, r, limit, t, nrm)) put64<D>(p, q, count, t, id, nrm);
        }
      }
    }
    if constexpr (K == kCastNearest) {
      p.out_leaf[q] = best;
      if (p.out_toi) p.out_toi[q] = best_t;
      if (p.out_normal) {
#pragma unroll
        for (int i = 0; i < D; ++i) p.out_normal[size_t(q) * D + i] = best_n[i];
      }
    } else if constexpr (K == kOverlap) {
      if (!p.csr_leaves) p.out_count[q] = count;
    } else {
      p.out_count[q] = count;
    }
  }
}

template <int D, int N>
const void* pick(bool stats) {
  return stats ? reinterpret_cast<const void*>(&nearest64_kernel<D, N, true>)
               : reinterpret_cast<const void*>(&nearest64_kernel<D, N, false>);
}

template <int D>
const void* pick_narrow(int narrow, bool stats) {
  switch (narrow) {
    case SQ_NARROW_AABB: return pick<D, kNarrowAabb>(stats);
    case SQ_NARROW_SPHERE: return pick<D, kNarrowSphere>(stats);
    case SQ_NARROW_SPHERE_NEAR: return pick<D, kNarrowSphereNear>(stats);
    case SQ_NARROW_TRIANGLE:
      if constexpr (D == 3) return pick<3, kNarrowTri>(stats);
      return nullptr;
    default: return nullptr;
  }
}

const void* kernel64(int dim, int narrow, bool stats) {
  switch (dim) {
    case 2: return pick_narrow<2>(narrow, stats);
    case 3: return pick_narrow<3>(narrow, stats);
    case 4: return pick_narrow<4>(narrow, stats);
    case 6: return pick_narrow<6>(narrow, stats);
    default: return nullptr;
  }
}

template <int D, int N>
const void* walk_pick(int kind) {
  switch (kind) {
    case kRayAll: return reinterpret_cast<const void*>(&walk64_kernel<D, N, kRayAll>);
    case kCastNearest: return reinterpret_cast<const void*>(&walk64_kernel<D, N, kCastNearest>);
    case kCastAll: return reinterpret_cast<const void*>(&walk64_kernel<D, N, kCastAll>);
    case kOverlap: return reinterpret_cast<const void*>(&walk64_kernel<D, N, kOverlap>);
    default: return nullptr;
  }
}

template <int D>
const void* walk_narrow(int narrow, int kind) {
  switch (narrow) {
    case SQ_NARROW_AABB: return walk_pick<D, kNarrowAabb>(kind);
    case SQ_NARROW_SPHERE: return walk_pick<D, kNarrowSphere>(kind);
    case SQ_NARROW_SPHERE_NEAR: return walk_pick<D, kNarrowSphereNear>(kind);
    case SQ_NARROW_TRIANGLE:
      if constexpr (D == 3) return walk_pick<3, kNarrowTri>(kind);
      return nullptr;
    default: return nullptr;
  }
}

const void* walk64(int dim, int narrow, int kind) {
  switch (dim) {
    case 2: return walk_narrow<2>(narrow, kind);
    case 3: return walk_narrow<3>(narrow, kind);
    case 4: return walk_narrow<4>(narrow, kind);
    case 6: return walk_narrow<6>(narrow, kind);
    default: return nullptr;
  }
}

Params64 base64(const sq_bvh* b, const sq_filter* filter) {
  Params64 p{};
  p.nb = b->d_nb64;
  p.nc = b->d_nc64;
  p.prims = b->d_prims64;
  p.ids = b->d_prim_ids;
  p.layers = b->d_layers;
  p.mask = filter ? filter->layer_mask : ~0ull;
  p.exclude = filter ? filter->exclude : -1;
  p.stride = b->stride;
  return p;
}

int32_t launch64(sq_ctx* ctx, const void* fn, Params64& p) {
  if (!fn) return fail(ctx, SQ_ERR_UNSUPPORTED, "no f64 kernel for this scene");
  const uint32_t grid = std::min<uint32_t>((p.n + 127) / 128, uint32_t(ctx->sm_count) * 16);
  void* args[] = {&p};
  CK(cudaLaunchKernel(fn, dim3(std::max<uint32_t>(grid, 1)), dim3(128), args, 0, ctx->stream));
  ctx->launches++;
  return SQ_OK;
}

uint32_t stride64(int dim, int narrow) {
  if (narrow == SQ_NARROW_AABB) return 2 * dim;
  if (narrow == SQ_NARROW_TRIANGLE) return 9;
  return dim + 1;
}

int32_t check64(sq_ctx* ctx, const sq_bvh* b) {
  if (!ctx) return SQ_ERR_INVALID;
  if (!b) return fail(ctx, SQ_ERR_INVALID, "null scene");
  if (b->device != ctx->device) return fail(ctx, SQ_ERR_INVALID, "scene and context are on different devices");
  if (b->prec != 64) return fail(ctx, SQ_ERR_UNSUPPORTED, "an f32 scene is queried through the f32 entry points");
  const cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, "cudaSetDevice", e);
  return SQ_OK;
}

}  // namespace

extern "C" int32_t sq_bvh_upload_f64(sq_ctx* ctx, int32_t dim, int32_t narrow, uint32_t n_nodes,
                                     const double* node_bounds, const uint32_t* child_a, const uint32_t* child_b,
                                     const uint32_t* prim_count, uint32_t n_prims, const uint32_t* prim_indices,
                                     const double* prim_data, uint32_t prim_stride, const uint64_t* layers,
                                     sq_bvh** out) {
  if (!ctx || !out) return SQ_ERR_INVALID;
  *out = nullptr;
  if (!kernel64(dim, narrow, false))
    return fail(ctx, SQ_ERR_UNSUPPORTED, "no f64 kernels for dim " + std::to_string(dim) + " narrow " +
                                             std::to_string(narrow));
  if (prim_stride != stride64(dim, narrow)) return fail(ctx, SQ_ERR_INVALID, "prim_stride does not match the narrow phase");
  if (n_prims >= kLeafBit || n_nodes >= kLeafBit) return fail(ctx, SQ_ERR_INVALID, "too many nodes or leaves");
  if ((n_nodes == 0) != (n_prims == 0)) return fail(ctx, SQ_ERR_INVALID, "empty tree with leaves, or leaves without a tree");
  if (n_nodes && (!node_bounds || !child_a || !child_b || !prim_count || !prim_indices || !prim_data))
    return fail(ctx, SQ_ERR_INVALID, "null tree array");
  CK(cudaSetDevice(ctx->device));
  auto b = std::make_unique<sq_bvh>();
  b->device = ctx->device;
  b->dim = dim;
  b->narrow = narrow;
  b->prec = 64;
  b->n_nodes = n_nodes;
  b->n_prims = n_prims;
  b->stride = prim_stride;
  if (n_nodes == 0) {
    *out = b.release();
    return SQ_OK;
  }
  // The same topology rules as the f32 upload: children after their parent,
  // leaves inside and partitioning a permutation; the depth bounds the stack.
  std::vector<uint32_t> depth(n_nodes, 1);
  for (uint32_t i = n_nodes; i-- > 0;) {
    if (prim_count[i] == 0) {
      if (child_a[i] <= i || child_b[i] <= i || child_a[i] >= n_nodes || child_b[i] >= n_nodes)
        return fail(ctx, SQ_ERR_INVALID, "interior node " + std::to_string(i) + " has a child out of order");
      depth[i] = 1 + std::max(depth[child_a[i]], depth[child_b[i]]);
    } else if (uint64_t(child_a[i]) + prim_count[i] > n_prims || prim_count[i] >= kLeafBit) {
      return fail(ctx, SQ_ERR_INVALID, "leaf node " + std::to_string(i) + " indexes past the primitives");
    }
  }
  b->depth = depth[0];
  if (b->depth + 1 > uint32_t(kStack64))
    return fail(ctx, SQ_ERR_DEPTH, "tree depth " + std::to_string(b->depth) + " exceeds the traversal stack");
  {
    std::vector<uint8_t> seen(n_prims, 0), covered(n_prims, 0);
    for (uint32_t k = 0; k < n_prims; ++k) {
      if (prim_indices[k] >= n_prims || seen[prim_indices[k]])
        return fail(ctx, SQ_ERR_INVALID, "prim_indices is not a permutation");
      seen[prim_indices[k]] = 1;
    }
    for (uint32_t i = 0; i < n_nodes; ++i) {
      if (prim_count[i] == 0) continue;
      for (uint32_t k = child_a[i]; k < child_a[i] + prim_count[i]; ++k) {
        if (covered[k]) return fail(ctx, SQ_ERR_INVALID, "leaf ranges overlap");
        covered[k] = 1;
      }
    }
    for (uint32_t k = 0; k < n_prims; ++k)
      if (!covered[k]) return fail(ctx, SQ_ERR_INVALID, "leaf ranges leave a primitive uncovered");
  }
  std::vector<uint2> links(n_nodes);
  for (uint32_t i = 0; i < n_nodes; ++i)
    links[i] = prim_count[i] == 0 ? make_uint2(child_a[i], child_b[i]) : make_uint2(child_a[i], prim_count[i] | kLeafBit);
  std::vector<double> prims(size_t(n_prims) * prim_stride);
  for (uint32_t pos = 0; pos < n_prims; ++pos)
    std::copy_n(prim_data + size_t(prim_indices[pos]) * prim_stride, prim_stride, prims.data() + size_t(pos) * prim_stride);
  auto up = [&](void** dst, const void* src, size_t bytes) -> int32_t {
    CK(cudaMalloc(dst, std::max<size_t>(bytes, 16)));
    if (src && bytes) CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    b->bytes += bytes;
    return SQ_OK;
  };
  int32_t rc;
  auto cleanup = [&](int32_t code) {
    sq_bvh_destroy(b.release());
    return code;
  };
  if ((rc = up((void**)&b->d_nb64, node_bounds, size_t(n_nodes) * 2 * dim * 8))) return cleanup(rc);
  if ((rc = up((void**)&b->d_nc64, links.data(), links.size() * sizeof(uint2)))) return cleanup(rc);
  if ((rc = up((void**)&b->d_prims64, prims.data(), prims.size() * 8))) return cleanup(rc);
  if ((rc = up((void**)&b->d_prim_ids, prim_indices, size_t(n_prims) * 4))) return cleanup(rc);
  if (layers && (rc = up((void**)&b->d_layers, layers, size_t(n_prims) * 8))) return cleanup(rc);
  *out = b.release();
  return SQ_OK;
}

extern "C" int32_t sq_raycast_nearest_f64_d(sq_ctx* ctx, const sq_bvh* b, const double* d_rays, uint32_t n,
                                            double max_toi, const double* d_max_toi_per_query,
                                            const sq_filter* filter, uint32_t* d_leaf, double* d_toi,
                                            double* d_normal, sq_query_stats* stats) {
  int32_t rc = check64(ctx, b);
  if (rc) return rc;
  if (n == 0) return SQ_OK;
  if (!d_rays || !d_leaf) return fail(ctx, SQ_ERR_INVALID, "null rays or leaf output");
  const bool st = stats != nullptr;
  if (st) CK(cudaMemsetAsync(ctx->d_stats, 0, 4 * sizeof(unsigned long long), ctx->stream));
  if (b->n_nodes == 0) {
    CK(cudaMemsetAsync(d_leaf, 0xFF, size_t(n) * 4, ctx->stream));
    if (d_toi) CK(cudaMemsetAsync(d_toi, 0, size_t(n) * 8, ctx->stream));
    if (d_normal) CK(cudaMemsetAsync(d_normal, 0, size_t(n) * b->dim * 8, ctx->stream));
  } else {
    Params64 p{};
    p.nb = b->d_nb64;
    p.nc = b->d_nc64;
    p.prims = b->d_prims64;
    p.ids = b->d_prim_ids;
    p.layers = b->d_layers;
    p.mask = filter ? filter->layer_mask : ~0ull;
    p.exclude = filter ? filter->exclude : -1;
    p.stride = b->stride;
    p.rays = d_rays;
    p.n = n;
    p.max_toi = max_toi;
    p.max_toi_arr = d_max_toi_per_query;
    p.out_leaf = d_leaf;
    p.out_toi = d_toi;
    p.out_normal = d_normal;
    p.stats = st ? ctx->d_stats : nullptr;
    const void* fn = kernel64(b->dim, b->narrow, st);
    const uint32_t grid = std::min<uint32_t>((n + 127) / 128, uint32_t(ctx->sm_count) * 16);
    void* args[] = {&p};
    CK(cudaLaunchKernel(fn, dim3(grid), dim3(128), args, 0, ctx->stream));
    ctx->launches++;
  }
  CK(cudaGetLastError());
  if (st) {
    unsigned long long h[4];
    CK(cudaMemcpyAsync(h, ctx->d_stats, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    stats->nodes_visited = h[0];
    stats->aabb_tests = h[1];
    stats->narrow_tests = h[2];
    stats->hits = h[3];
  }
  return SQ_OK;
}

extern "C" int32_t sq_raycast_nearest_f64(sq_ctx* ctx, const sq_bvh* b, const double* rays, uint32_t n,
                                          double max_toi, const double* max_toi_per_query, const sq_filter* filter,
                                          uint32_t* leaf, double* toi, double* normal, sq_query_stats* stats) {
  int32_t rc = check64(ctx, b);
  if (rc) return rc;
  if (n == 0) return SQ_OK;
  if (!rays || !leaf) return fail(ctx, SQ_ERR_INVALID, "null rays or leaf output");
  const int D = b->dim;
  // One scratch allocation for the batch: rays, per-query limits, outputs.
  const size_t b_rays = size_t(n) * 2 * D * 8, b_mt = max_toi_per_query ? size_t(n) * 8 : 0, b_leaf = size_t(n) * 4,
               b_toi = toi ? size_t(n) * 8 : 0, b_nrm = normal ? size_t(n) * D * 8 : 0;
  sqi::Carve cv;
  const size_t o_rays = cv.take(b_rays), o_mt = cv.take(b_mt), o_leaf = cv.take(b_leaf), o_toi = cv.take(b_toi),
               o_nrm = cv.take(b_nrm);
  if ((rc = sqi::arena_reserve(ctx, cv.off))) return rc;
  char* base = static_cast<char*>(ctx->arena.p);
  CK(cudaMemcpyAsync(base + o_rays, rays, b_rays, cudaMemcpyHostToDevice, ctx->stream));
  if (b_mt) CK(cudaMemcpyAsync(base + o_mt, max_toi_per_query, b_mt, cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = sq_raycast_nearest_f64_d(ctx, b, reinterpret_cast<const double*>(base + o_rays), n, max_toi,
                                     b_mt ? reinterpret_cast<const double*>(base + o_mt) : nullptr, filter,
                                     reinterpret_cast<uint32_t*>(base + o_leaf),
                                     b_toi ? reinterpret_cast<double*>(base + o_toi) : nullptr,
                                     b_nrm ? reinterpret_cast<double*>(base + o_nrm) : nullptr, stats)))
    return rc;
  CK(cudaMemcpyAsync(leaf, base + o_leaf, b_leaf, cudaMemcpyDeviceToHost, ctx->stream));
  if (b_toi) CK(cudaMemcpyAsync(toi, base + o_toi, b_toi, cudaMemcpyDeviceToHost, ctx->stream));
  if (b_nrm) CK(cudaMemcpyAsync(normal, base + o_nrm, b_nrm, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

// ---------------------------------------------------------------------------
// Lists, casts and overlap on f64 scenes.
// ---------------------------------------------------------------------------

namespace {

int32_t list_args(sq_ctx* ctx, uint32_t n, const double* q, const sq_hit_lists_f64* o) {
  if (!o || (n && (!q || !o->count || (o->k && (!o->leaf || !o->toi)))))
    return fail(ctx, SQ_ERR_INVALID, "null queries or list output");
  return SQ_OK;
}

int32_t lists64(sq_ctx* ctx, const sq_bvh* b, int kind, const double* d_q, uint32_t n, double max_toi,
                const double* d_mt, const sq_filter* filter, int32_t crossings, const sq_hit_lists_f64* o) {
  int32_t rc = check64(ctx, b);
  if (rc || (rc = list_args(ctx, n, d_q, o))) return rc;
  if (n == 0) return SQ_OK;
  if (b->n_nodes == 0) {
    CK(cudaMemsetAsync(o->count, 0, size_t(n) * 4, ctx->stream));
    return SQ_OK;
  }
  Params64 p = base64(b, filter);
  p.rays = d_q;
  p.n = n;
  p.max_toi = max_toi;
  p.max_toi_arr = d_mt;
  p.k = o->k;
  p.crossings = crossings;
  p.out_count = o->count;
  p.out_leaf = o->leaf;
  p.out_toi = o->toi;
  p.out_normal = o->normal;
  return launch64(ctx, walk64(b->dim, b->narrow, kind), p);
}

// Host-buffer lists: queries (and per-query limits) in, lists out, through
// the context's arena.
int32_t lists64_host(sq_ctx* ctx, const sq_bvh* b, int kind, uint32_t width, const double* q, uint32_t n,
                     double max_toi, const double* mt, const sq_filter* filter, int32_t crossings,
                     const sq_hit_lists_f64* o) {
  int32_t rc = check64(ctx, b);
  if (rc || (rc = list_args(ctx, n, q, o))) return rc;
  if (n == 0) return SQ_OK;
  const int D = b->dim;
  const size_t k = o->k;
  sqi::Carve cv;
  const size_t o_q = cv.take(size_t(n) * width * D * 8), o_mt = cv.take(mt ? size_t(n) * 8 : 0),
               o_cnt = cv.take(size_t(n) * 4), o_leaf = cv.take(size_t(n) * k * 4), o_toi = cv.take(size_t(n) * k * 8),
               o_nrm = cv.take(o->normal ? size_t(n) * k * D * 8 : 0);
  if ((rc = sqi::arena_reserve(ctx, cv.off))) return rc;
  char* base = static_cast<char*>(ctx->arena.p);
  CK(cudaMemcpyAsync(base + o_q, q, size_t(n) * width * D * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (mt) CK(cudaMemcpyAsync(base + o_mt, mt, size_t(n) * 8, cudaMemcpyHostToDevice, ctx->stream));
  sq_hit_lists_f64 d{};
  d.k = o->k;
  d.count = reinterpret_cast<uint32_t*>(base + o_cnt);
  d.leaf = reinterpret_cast<uint32_t*>(base + o_leaf);
  d.toi = reinterpret_cast<double*>(base + o_toi);
  d.normal = o->normal ? reinterpret_cast<double*>(base + o_nrm) : nullptr;
  if ((rc = lists64(ctx, b, kind, reinterpret_cast<const double*>(base + o_q), n, max_toi,
                    mt ? reinterpret_cast<const double*>(base + o_mt) : nullptr, filter, crossings, &d)))
    return rc;
  // Only the stored entries come back: the first min(count, k) of each query.
  std::vector<uint32_t> cnt(n);
  CK(cudaMemcpyAsync(cnt.data(), d.count, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::memcpy(o->count, cnt.data(), size_t(n) * 4);
  if (k) {
    CK(cudaMemcpyAsync(o->leaf, d.leaf, size_t(n) * k * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(o->toi, d.toi, size_t(n) * k * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (o->normal) CK(cudaMemcpyAsync(o->normal, d.normal, size_t(n) * k * D * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return SQ_OK;
}

}  // namespace

extern "C" int32_t sq_raycast_all_f64_d(sq_ctx* ctx, const sq_bvh* b, const double* d_rays, uint32_t n,
                                        double max_toi, const double* d_max_toi_per_query, const sq_filter* filter,
                                        int32_t crossings, const sq_hit_lists_f64* d_out) {
  return lists64(ctx, b, kRayAll, d_rays, n, max_toi, d_max_toi_per_query, filter, crossings, d_out);
}

extern "C" int32_t sq_raycast_all_f64(sq_ctx* ctx, const sq_bvh* b, const double* rays, uint32_t n, double max_toi,
                                      const double* max_toi_per_query, const sq_filter* filter, int32_t crossings,
                                      const sq_hit_lists_f64* out) {
  return lists64_host(ctx, b, kRayAll, 2, rays, n, max_toi, max_toi_per_query, filter, crossings, out);
}

extern "C" int32_t sq_shapecast_all_f64_d(sq_ctx* ctx, const sq_bvh* b, const double* d_casts, uint32_t n,
                                          double max_toi, const double* d_max_toi_per_query, const sq_filter* filter,
                                          const sq_hit_lists_f64* d_out) {
  return lists64(ctx, b, kCastAll, d_casts, n, max_toi, d_max_toi_per_query, filter, 0, d_out);
}

extern "C" int32_t sq_shapecast_all_f64(sq_ctx* ctx, const sq_bvh* b, const double* casts, uint32_t n,
                                        double max_toi, const double* max_toi_per_query, const sq_filter* filter,
                                        const sq_hit_lists_f64* out) {
  return lists64_host(ctx, b, kCastAll, 4, casts, n, max_toi, max_toi_per_query, filter, 0, out);
}

extern "C" int32_t sq_shapecast_nearest_f64_d(sq_ctx* ctx, const sq_bvh* b, const double* d_casts, uint32_t n,
                                              double max_toi, const double* d_max_toi_per_query,
                                              const sq_filter* filter, uint32_t* d_leaf, double* d_toi,
                                              double* d_normal) {
  int32_t rc = check64(ctx, b);
  if (rc) return rc;
  if (n && (!d_casts || !d_leaf)) return fail(ctx, SQ_ERR_INVALID, "null casts or leaf output");
  if (n == 0) return SQ_OK;
  if (b->n_nodes == 0) {
    CK(cudaMemsetAsync(d_leaf, 0xFF, size_t(n) * 4, ctx->stream));
    if (d_toi) CK(cudaMemsetAsync(d_toi, 0, size_t(n) * 8, ctx->stream));
    if (d_normal) CK(cudaMemsetAsync(d_normal, 0, size_t(n) * b->dim * 8, ctx->stream));
    return SQ_OK;
  }
  Params64 p = base64(b, filter);
  p.rays = d_casts;
  p.n = n;
  p.max_toi = max_toi;
  p.max_toi_arr = d_max_toi_per_query;
  p.out_leaf = d_leaf;
  p.out_toi = d_toi;
  p.out_normal = d_normal;
  return launch64(ctx, walk64(b->dim, b->narrow, kCastNearest), p);
}

extern "C" int32_t sq_shapecast_nearest_f64(sq_ctx* ctx, const sq_bvh* b, const double* casts, uint32_t n,
                                            double max_toi, const double* max_toi_per_query, const sq_filter* filter,
                                            uint32_t* leaf, double* toi, double* normal) {
  int32_t rc = check64(ctx, b);
  if (rc) return rc;
  if (n == 0) return SQ_OK;
  if (!casts || !leaf) return fail(ctx, SQ_ERR_INVALID, "null casts or leaf output");
  const int D = b->dim;
  sqi::Carve cv;
  const size_t o_q = cv.take(size_t(n) * 4 * D * 8), o_mt = cv.take(max_toi_per_query ? size_t(n) * 8 : 0),
               o_leaf = cv.take(size_t(n) * 4), o_toi = cv.take(toi ? size_t(n) * 8 : 0),
               o_nrm = cv.take(normal ? size_t(n) * D * 8 : 0);
  if ((rc = sqi::arena_reserve(ctx, cv.off))) return rc;
  char* base = static_cast<char*>(ctx->arena.p);
  CK(cudaMemcpyAsync(base + o_q, casts, size_t(n) * 4 * D * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (max_toi_per_query)
    CK(cudaMemcpyAsync(base + o_mt, max_toi_per_query, size_t(n) * 8, cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = sq_shapecast_nearest_f64_d(ctx, b, reinterpret_cast<const double*>(base + o_q), n, max_toi,
                                       max_toi_per_query ? reinterpret_cast<const double*>(base + o_mt) : nullptr,
                                       filter, reinterpret_cast<uint32_t*>(base + o_leaf),
                                       toi ? reinterpret_cast<double*>(base + o_toi) : nullptr,
                                       normal ? reinterpret_cast<double*>(base + o_nrm) : nullptr)))
    return rc;
  CK(cudaMemcpyAsync(leaf, base + o_leaf, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (toi) CK(cudaMemcpyAsync(toi, base + o_toi, size_t(n) * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (normal) CK(cudaMemcpyAsync(normal, base + o_nrm, size_t(n) * D * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

extern "C" int32_t sq_overlap_f64_d(sq_ctx* ctx, const sq_bvh* b, const double* d_regions, uint32_t n,
                                    const sq_filter* filter, uint64_t* d_offsets, uint32_t* d_leaves,
                                    uint64_t leaf_capacity, uint64_t* total) {
  int32_t rc = check64(ctx, b);
  if (rc) return rc;
  if (!d_offsets || !total || (n && !d_regions)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  // Counts and the scan's scratch from the context's arena.
  size_t scan_bytes = 0;
  CK(cub::DeviceScan::ExclusiveScan(nullptr, scan_bytes, static_cast<const uint32_t*>(nullptr),
                                    static_cast<unsigned long long*>(nullptr), cuda::std::plus<>{}, 0ull, int(n) + 1,
                                    ctx->stream));
  sqi::Carve cv;
  const size_t o_cnt = cv.take((size_t(n) + 1) * 4), o_tmp = cv.take(scan_bytes);
  if ((rc = sqi::arena_reserve(ctx, cv.off))) return rc;
  char* base = static_cast<char*>(ctx->arena.p);
  uint32_t* d_counts = reinterpret_cast<uint32_t*>(base + o_cnt);
  CK(cudaMemsetAsync(d_counts, 0, (size_t(n) + 1) * 4, ctx->stream));
  Params64 p = base64(b, filter);
  p.rays = d_regions;
  p.n = n;
  p.out_count = d_counts;
  const void* fn = walk64(b->dim, b->narrow, kOverlap);
  if (b->n_nodes != 0 && n != 0 && (rc = launch64(ctx, fn, p))) return rc;
  CK(cub::DeviceScan::ExclusiveScan(base + o_tmp, scan_bytes, d_counts, reinterpret_cast<unsigned long long*>(d_offsets),
                                    cuda::std::plus<>{}, 0ull, int(n) + 1, ctx->stream));
  ctx->launches++;
  unsigned long long tot = 0;
  CK(cudaMemcpyAsync(&tot, d_offsets + n, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *total = tot;
  if (tot > leaf_capacity) return fail(ctx, SQ_ERR_CAPACITY, "overlap results exceed leaf_capacity");
  if (tot && b->n_nodes != 0) {
    if (!d_leaves) return fail(ctx, SQ_ERR_INVALID, "null leaf output");
    p.csr_offsets = reinterpret_cast<const unsigned long long*>(d_offsets);
    p.csr_leaves = d_leaves;
    if ((rc = launch64(ctx, fn, p))) return rc;
    if ((rc = sqi::sort_csr_segments(ctx, d_leaves, tot, d_offsets, n))) return rc;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

extern "C" int32_t sq_overlap_f64(sq_ctx* ctx, const sq_bvh* b, const double* regions, uint32_t n,
                                  const sq_filter* filter, uint64_t* offsets, uint32_t* leaves, uint64_t leaf_capacity,
                                  uint64_t* total) {
  int32_t rc = check64(ctx, b);
  if (rc) return rc;
  if (!offsets || !total || (n && !regions)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  const int D = b->dim;
  // Regions and offsets in a scratch block of their own: the device call
  // takes the arena for its counts.
  char* dq = nullptr;
  const size_t qb = (size_t(n) * 2 * D * 8 + 255) & ~size_t(255);
  CK(sqi::scratch_alloc(ctx, reinterpret_cast<void**>(&dq), qb + (size_t(n) + 1) * 8 + size_t(leaf_capacity) * 4 + 16));
  uint64_t* d_off = reinterpret_cast<uint64_t*>(dq + qb);
  uint32_t* d_lv = reinterpret_cast<uint32_t*>(dq + qb + (size_t(n) + 1) * 8);
  cudaError_t e = n ? cudaMemcpyAsync(dq, regions, size_t(n) * 2 * D * 8, cudaMemcpyHostToDevice, ctx->stream)
                    : cudaSuccess;
  if (e == cudaSuccess) {
    rc = sq_overlap_f64_d(ctx, b, reinterpret_cast<const double*>(dq), n, filter, d_off, d_lv, leaf_capacity, total);
    if (rc == SQ_OK || rc == SQ_ERR_CAPACITY)
      e = cudaMemcpyAsync(offsets, d_off, (size_t(n) + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (rc == SQ_OK && e == cudaSuccess && *total && leaves)
      e = cudaMemcpyAsync(leaves, d_lv, size_t(*total) * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  }
  cudaFreeAsync(dq, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, "overlap f64 copies", e);
  return rc;
}
