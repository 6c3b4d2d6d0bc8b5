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
