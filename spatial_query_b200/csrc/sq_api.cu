// C ABI of the batched-query library: contexts, scene upload, refit and the
// query entry points declared in include/sq.h.
//
// The host part of GpuRaycaster (crates/spatial-query/src/gpu/mod.rs:229-535)
// re-designed for CUDA: a context owns a stream, a ring of work counters for
// the persistent kernels and a growable staging arena (host-buffer calls
// reuse it, so a steady stream of same-sized batches allocates nothing);
// an uploaded scene owns its node and primitive records in HBM.
#include <cuda_runtime.h>

#include <cub/device/device_segmented_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda/std/functional>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "sq_internal.cuh"

using namespace sq;

namespace {

using namespace sqi;

void base_params(const sq_bvh* b, const sq_filter* f, QueryParams& p) {
  std::memset(&p, 0, sizeof(p));
  p.nodes = b->d_nodes;
  p.prims = b->d_prims;
  p.layers = b->d_layers;
  p.sub = b->d_sub;
  p.root_box = b->d_root;
  p.nonfinite = b->d_nonfinite;
  p.root_code = b->root_code;
  p.wnodes = b->d_wnodes;
  p.qnodes = b->d_qnodes;
  p.wroot = b->wroot;
  p.mask = f ? f->layer_mask : ~0ull;
  p.exclude = f ? f->exclude : -1;
}

int32_t check_scene(sq_ctx* ctx, const sq_bvh* b) {
  if (!ctx) return SQ_ERR_INVALID;
  if (!b) return fail(ctx, SQ_ERR_INVALID, "null scene");
  if (b->device != ctx->device) return fail(ctx, SQ_ERR_INVALID, "scene and context are on different devices");
  if (b->prec != 32) return fail(ctx, SQ_ERR_UNSUPPORTED, "an f64 scene is queried through the _f64 entry points");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, "cudaSetDevice", e);
  return SQ_OK;
}

// ---- the query cores (device pointers, enqueue only) -----------------------

int32_t nearest_core(sq_ctx* ctx, const sq_bvh* b, bool cast, const float* d_q, uint32_t n, float max_toi,
                     const float* d_mt, const sq_filter* f, const sq_hits& o, bool stats) {
  if (n == 0) return SQ_OK;
  if (!o.leaf) return fail(ctx, SQ_ERR_INVALID, "null leaf output");
  if (b->n_nodes == 0) {
    // Empty tree (gpu/mod.rs:352-354): every query misses.
    CK(cudaMemsetAsync(o.leaf, 0xFF, size_t(n) * 4, ctx->stream));
    if (o.toi) CK(cudaMemsetAsync(o.toi, 0, size_t(n) * 4, ctx->stream));
    if (o.sub_object) CK(cudaMemsetAsync(o.sub_object, 0xFF, size_t(n) * 4, ctx->stream));
    if (o.normal) CK(cudaMemsetAsync(o.normal, 0, size_t(n) * 4 * b->dim, ctx->stream));
    if (o.point) CK(cudaMemsetAsync(o.point, 0, size_t(n) * 4 * b->dim, ctx->stream));
    return SQ_OK;
  }
  QueryParams p;
  base_params(b, f, p);
  p.queries = d_q;
  p.max_toi_arr = d_mt;
  p.max_toi = max_toi;
  p.n = n;
  p.out_leaf = o.leaf;
  p.out_toi = o.toi;
  p.out_sub = o.sub_object;
  p.out_normal = o.normal;
  p.out_point = o.point;
  const bool near_first = ctx->order != SQ_ORDER_REFERENCE;
  const int st = stats ? 1 : 0;
  if (stats && !cast) p.stats = ctx->d_stats;
  const void* ref_fn = cast ? b->ks.cast_nearest[1] : b->ks.ray_nearest[1][st];
  const void* near_fn = cast ? b->ks.cast_nearest[0] : b->ks.ray_nearest[0][st];
  if (!ref_fn || !near_fn) return fail(ctx, SQ_ERR_UNSUPPORTED, "this scene's narrow phase has no such query");
  if (!near_first) return launch_persistent(ctx, ref_fn, p, b->depth, p.n);
  // Four-wide records for plain near-first rays: each visited record stacks
  // at most three children, so the stack holds 3 x (four-wide depth) + 1.
  if (!cast && !stats && ctx->layout == SQ_LAYOUT_WIDE && b->n_wide && b->ks.ray_nearest_wide)
    return near_first_launch(ctx, b, b->ks.ray_nearest_wide, ref_fn, p, 3 * b->wdepth + 1);
  if (!cast && !stats && ctx->layout == SQ_LAYOUT_QUANT && b->n_wide && b->d_qnodes && b->ks.ray_nearest_quant)
    return near_first_launch(ctx, b, b->ks.ray_nearest_quant, ref_fn, p, 3 * b->wdepth + 1);
  if (!cast && !stats && ctx->layout == SQ_LAYOUT_BINARY_REGTOP && b->ks.ray_nearest_regtop)
    return near_first_launch(ctx, b, b->ks.ray_nearest_regtop, ref_fn, p, b->depth);
  if (!cast && !stats && ctx->layout == SQ_LAYOUT_BINARY_VOTE && b->ks.ray_nearest_vote)
    return near_first_launch(ctx, b, b->ks.ray_nearest_vote, ref_fn, p, b->depth);
  return near_first_launch(ctx, b, near_fn, kReplayInKernel ? nullptr : ref_fn, p, b->depth);
}

int32_t list_core(sq_ctx* ctx, const sq_bvh* b, int kind, const float* d_q, uint32_t n, float max_toi,
                  const float* d_mt, const sq_filter* f, const sq_hit_lists& o, bool stats) {
  if (n == 0) return SQ_OK;
  if (!o.count || (o.k && (!o.leaf || !o.toi))) return fail(ctx, SQ_ERR_INVALID, "null list output");
  if (b->n_nodes == 0) {
    CK(cudaMemsetAsync(o.count, 0, size_t(n) * 4, ctx->stream));
    return SQ_OK;
  }
  QueryParams p;
  base_params(b, f, p);
  p.queries = d_q;
  p.max_toi_arr = d_mt;
  p.max_toi = max_toi;
  p.n = n;
  p.k = o.k;
  p.out_count = o.count;
  p.out_leaf = o.leaf;
  p.out_toi = o.toi;
  p.out_sub = o.sub_object;
  p.out_normal = o.normal;
  const void* fn;
  if (kind == kCastAll) {
    fn = b->ks.cast_all;
  } else {
    p.crossings = kind == 100 ? 1 : 0;
    fn = b->ks.ray_all[stats ? 1 : 0];
    if (stats) p.stats = ctx->d_stats;
  }
  if (!fn) return fail(ctx, SQ_ERR_UNSUPPORTED, "this scene's narrow phase has no such query");
  return launch_persistent(ctx, fn, p, b->depth, p.n);
}

int32_t stats_begin(sq_ctx* ctx, sq_query_stats* st) {
  if (st) CK(cudaMemsetAsync(ctx->d_stats, 0, 4 * sizeof(unsigned long long), ctx->stream));
  return SQ_OK;
}

int32_t stats_end(sq_ctx* ctx, sq_query_stats* st) {
  if (!st) return SQ_OK;
  unsigned long long h[4];
  CK(cudaMemcpyAsync(h, ctx->d_stats, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  st->nodes_visited = h[0];
  st->aabb_tests = h[1];
  st->narrow_tests = h[2];
  st->hits = h[3];
  return SQ_OK;
}

int32_t finish(sq_ctx* ctx) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, "kernel launch", e);
  return SQ_OK;
}

}  // namespace

// ============================================================================
// context
// ============================================================================

extern "C" int32_t sq_version(void) { return 1; }

extern "C" int32_t sq_ctx_create(int32_t device, sq_ctx** out) {
  if (!out) return SQ_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return SQ_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return SQ_ERR_INVALID;
  sq_ctx* ctx = new sq_ctx();
  ctx->device = device;
  auto bail = [&](cudaError_t e, const char* w) {
    fprintf(stderr, "sq_ctx_create: %s: %s\n", w, cudaGetErrorString(e));
    if (ctx->d_counters) cudaFree(ctx->d_counters);
    if (ctx->d_stats) cudaFree(ctx->d_stats);
    if (ctx->d_replays) cudaFree(ctx->d_replays);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return SQ_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
  ctx->stream = ctx->own;
  if ((e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
    return bail(e, "sm count");
  if ((e = cudaMalloc(&ctx->d_counters, kCounterSlots * sizeof(uint32_t))) != cudaSuccess) return bail(e, "counters");
  if ((e = cudaMalloc(&ctx->d_stats, 4 * sizeof(unsigned long long))) != cudaSuccess) return bail(e, "stats");
  if ((e = cudaMalloc(&ctx->d_replays, sizeof(uint32_t))) != cudaSuccess) return bail(e, "replays");
  if ((e = cudaMemset(ctx->d_replays, 0, sizeof(uint32_t))) != cudaSuccess) return bail(e, "replays");
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  if ((e = cudaMemPoolCreate(&ctx->pool, &props)) != cudaSuccess) return bail(e, "memory pool");
  uint64_t keep = ~uint64_t(0);
  if ((e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess)
    return bail(e, "memory pool");
  *out = ctx;
  return SQ_OK;
}

extern "C" int32_t sq_ctx_destroy(sq_ctx* ctx) {
  if (!ctx) return SQ_OK;
  cudaSetDevice(ctx->device);
  if (ctx->own) cudaStreamSynchronize(ctx->own);
  if (ctx->stream && ctx->stream != ctx->own) cudaStreamSynchronize(ctx->stream);
  if (ctx->lane) sq_ctx_destroy(ctx->lane);
  sqi::release_err_slot(ctx);
  if (ctx->arena.p) cudaFree(ctx->arena.p);
  if (ctx->d_replays) cudaFree(ctx->d_replays);
  if (ctx->replay_list.p) cudaFree(ctx->replay_list.p);
  if (ctx->d_counters) cudaFree(ctx->d_counters);
  if (ctx->d_stats) cudaFree(ctx->d_stats);
  if (ctx->s_in) cudaStreamDestroy(ctx->s_in);
  if (ctx->s_out) cudaStreamDestroy(ctx->s_out);
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  // A caller's stream may already be gone: no status of this teardown may be
  // left for a later call's launch check to report.
  cudaGetLastError();
  delete ctx;
  return SQ_OK;
}

extern "C" const char* sq_ctx_last_error(const sq_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" void* sq_ctx_stream(sq_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

namespace {
int32_t apply_l2_window(sq_ctx* ctx);
}

extern "C" int32_t sq_ctx_set_stream(sq_ctx* ctx, void* stream) {
  if (!ctx) return SQ_ERR_INVALID;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
  // An L2 window set with sq_ctx_set_l2_persist follows the context's stream.
  if (ctx->l2_window.num_bytes) return apply_l2_window(ctx);
  return SQ_OK;
}

extern "C" int32_t sq_ctx_synchronize(sq_ctx* ctx) {
  if (!ctx) return SQ_ERR_INVALID;
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

extern "C" int32_t sq_ctx_set_order(sq_ctx* ctx, int32_t order) {
  if (!ctx || (order != SQ_ORDER_NEAR_FIRST && order != SQ_ORDER_REFERENCE)) return SQ_ERR_INVALID;
  ctx->order = order;
  return SQ_OK;
}

extern "C" int32_t sq_ctx_set_layout(sq_ctx* ctx, int32_t layout) {
  if (!ctx || layout < SQ_LAYOUT_BINARY || layout > SQ_LAYOUT_BINARY_VOTE)
    return SQ_ERR_INVALID;
  ctx->layout = layout;
  return SQ_OK;
}

extern "C" int32_t sq_ctx_set_blocks_per_sm(sq_ctx* ctx, int32_t blocks) {
  if (!ctx || blocks < 0 || blocks > 64) return SQ_ERR_INVALID;
  ctx->blocks_per_sm = blocks;
  return SQ_OK;
}

extern "C" uint64_t sq_ctx_launch_count(const sq_ctx* ctx) { return ctx ? ctx->launches : 0; }

extern "C" int32_t sq_ctx_set_replay_window(sq_ctx* ctx, float window) {
  if (!ctx || !(window >= 0.f) || window > 1.f) return SQ_ERR_INVALID;
  ctx->window = window;
  return SQ_OK;
}

namespace {
int32_t apply_l2_window(sq_ctx* ctx) {
  cudaStreamAttrValue v{};
  v.accessPolicyWindow = ctx->l2_window;
  CK(cudaStreamSetAttribute(ctx->stream, cudaStreamAttributeAccessPolicyWindow, &v));
  return SQ_OK;
}
}  // namespace

extern "C" int32_t sq_ctx_set_l2_persist(sq_ctx* ctx, const sq_bvh* b, uint64_t bytes) {
  if (!ctx) return SQ_ERR_INVALID;
  if (b && b->device != ctx->device) return fail(ctx, SQ_ERR_INVALID, "scene on another device");
  CK(cudaSetDevice(ctx->device));
  ctx->l2_window = cudaAccessPolicyWindow{};
  if (b && bytes && b->d_nodes && b->n_interior) {
    int max_persist = 0, max_window = 0;
    CK(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ctx->device));
    CK(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, ctx->device));
    if (max_persist <= 0 || max_window <= 0) return fail(ctx, SQ_ERR_UNSUPPORTED, "no persisting L2 on this device");
    const size_t reserve = std::min<size_t>(bytes, size_t(max_persist));
    CK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, reserve));
    const size_t region = size_t(b->n_interior) * node_vec(b->dim) * 16;
    const size_t win = std::min<size_t>(region, size_t(max_window));
    ctx->l2_window.base_ptr = b->d_nodes;
    ctx->l2_window.num_bytes = win;
    ctx->l2_window.hitRatio = std::min(1.0f, float(double(reserve) / double(win)));
    ctx->l2_window.hitProp = cudaAccessPropertyPersisting;
    ctx->l2_window.missProp = cudaAccessPropertyStreaming;
  }
  int32_t rc = apply_l2_window(ctx);
  if (rc == SQ_OK && ctx->lane) rc = apply_l2_window(ctx->lane);
  if (rc) return rc;
  if (ctx->l2_window.num_bytes == 0) {
    // Lines marked persisting so far go back to normal.
    CK(cudaCtxResetPersistingL2Cache());
  }
  return SQ_OK;
}

extern "C" int32_t sq_ctx_last_replay_count(sq_ctx* ctx, uint32_t* out) {
  if (!ctx || !out) return SQ_ERR_INVALID;
  *out = 0;
  CK(cudaMemcpyAsync(out, ctx->d_replays, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

// ============================================================================
// upload / refit
// ============================================================================

// The shared upload. A consumer narrow phase (SQ_NARROW_CUSTOM) brings its
// run-time-compiled kernels in `custom` and the per-leaf AABBs the tree was
// built from in `prim_aabbs` (stored beside the leaf data).
static int32_t upload_impl(sq_ctx* ctx, int32_t dim, int32_t narrow, uint32_t n_nodes, const float* node_bounds,
                           const uint32_t* child_a, const uint32_t* child_b, const uint32_t* prim_count,
                           uint32_t n_prims, const uint32_t* prim_indices, const float* prim_data,
                           uint32_t prim_stride, const uint64_t* layers, const uint32_t* sub_objects,
                           const float* prim_aabbs, const KernelSet* custom, sq_bvh** out) {
  if (!ctx || !out) return SQ_ERR_INVALID;
  *out = nullptr;
  KernelSet ks;
  if (custom) {
    ks = *custom;
  } else {
    if (!kernel_set(dim, narrow, &ks))
      return fail(ctx, SQ_ERR_UNSUPPORTED, "no kernels for dim " + std::to_string(dim) + " narrow " +
                                               std::to_string(narrow));
    if (prim_stride != stride_of(dim, narrow))
      return fail(ctx, SQ_ERR_INVALID, "prim_stride does not match the narrow phase");
  }
  if (n_prims >= kLeafBit || n_nodes >= kLeafBit) return fail(ctx, SQ_ERR_INVALID, "too many nodes or leaves");
  if ((n_nodes == 0) != (n_prims == 0)) return fail(ctx, SQ_ERR_INVALID, "empty tree with leaves, or leaves without a tree");
  if (n_nodes && (!node_bounds || !child_a || !child_b || !prim_count || !prim_indices || !prim_data))
    return fail(ctx, SQ_ERR_INVALID, "null tree array");
  CK(cudaSetDevice(ctx->device));

  auto b = std::make_unique<sq_bvh>();
  b->device = ctx->device;
  b->dim = dim;
  b->narrow = narrow;
  b->n_nodes = n_nodes;
  b->n_prims = n_prims;
  b->stride = prim_stride;
  b->prim_vec = custom ? (prim_stride + 2 * dim + 1 + 3) / 4 : prim_vec(dim, narrow);
  b->ks = ks;
  if (n_nodes == 0) {
    *out = b.release();
    return SQ_OK;
  }

  // Validate the topology (children after their parent, leaf ranges inside
  // the index array) and compute the depth in one reverse pass.
  std::vector<uint32_t> depth(n_nodes, 1);
  for (uint32_t i = n_nodes; i-- > 0;) {
    if (prim_count[i] == 0) {
      if (child_a[i] <= i || child_b[i] <= i || child_a[i] >= n_nodes || child_b[i] >= n_nodes)
        return fail(ctx, SQ_ERR_INVALID, "interior node " + std::to_string(i) + " has a child out of order");
      depth[i] = 1 + std::max(depth[child_a[i]], depth[child_b[i]]);
    } else if (uint64_t(child_a[i]) + prim_count[i] > n_prims) {
      return fail(ctx, SQ_ERR_INVALID, "leaf node " + std::to_string(i) + " indexes past the primitives");
    }
  }
  b->depth = depth[0];
  if (b->depth > uint32_t(kMaxStack))
    return fail(ctx, SQ_ERR_DEPTH, "tree depth " + std::to_string(b->depth) + " exceeds the traversal stack");
  // The leaves must partition the index array and the index array must be a
  // permutation: every kernel walk of a leaf then ends on its own last
  // primitive, inside the array.
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

  // Interior record numbering (node order) and node codes.
  b->h_iidx.assign(n_nodes, kNoHit);
  uint32_t ni = 0;
  for (uint32_t i = 0; i < n_nodes; ++i)
    if (prim_count[i] == 0) b->h_iidx[i] = ni++;
  b->n_interior = ni;
  auto code = [&](uint32_t i) { return prim_count[i] == 0 ? b->h_iidx[i] : (kLeafBit | child_a[i]); };
  b->root_code = code(0);
  b->h_child_a.assign(child_a, child_a + n_nodes);
  b->h_child_b.assign(child_b, child_b + n_nodes);
  b->h_count.assign(prim_count, prim_count + n_nodes);

  const int D = dim;
  const uint32_t NV = node_vec(D), PV = b->prim_vec;
  std::vector<float> nodes(size_t(std::max<uint32_t>(ni, 1)) * NV * 4, 0.f);
  std::vector<uint32_t> parents(std::max<uint32_t>(ni, 1), kNoHit);
  std::vector<RefitLeaf> leaves;
  for (uint32_t i = 0; i < n_nodes; ++i) {
    if (prim_count[i] != 0) {
      if (i == 0) leaves.push_back(RefitLeaf{child_a[0], prim_count[0], kNoHit, 0});
      continue;
    }
    const uint32_t k = b->h_iidx[i];
    float* r = nodes.data() + size_t(k) * NV * 4;
    const uint32_t ch[2] = {child_a[i], child_b[i]};
    for (int s = 0; s < 2; ++s) {
      const float* cb = node_bounds + size_t(ch[s]) * 2 * D;
      for (int j = 0; j < 2 * D; ++j) r[s * 2 * D + j] = cb[j];
      uint32_t c = code(ch[s]);
      std::memcpy(&r[4 * D + s], &c, 4);
      if (prim_count[ch[s]] == 0) parents[b->h_iidx[ch[s]]] = (k << 1) | uint32_t(s);
      else leaves.push_back(RefitLeaf{child_a[ch[s]], prim_count[ch[s]], (k << 1) | uint32_t(s), 0});
    }
  }
  b->n_leaves = uint32_t(leaves.size());

  // Primitive records in leaf order: payload, then the id (flagged on the
  // last primitive of each leaf).
  const uint32_t payload = custom ? prim_stride + 2 * D
                                  : (narrow == SQ_NARROW_AABB ? 2 * D : (narrow == SQ_NARROW_TRIANGLE ? 9 : D + 1));
  std::vector<float> prims(size_t(n_prims) * PV * 4, 0.f);
  for (const RefitLeaf& L : leaves) {
    for (uint32_t j = 0; j < L.count; ++j) {
      const uint32_t pos = L.first + j;
      const uint32_t id = prim_indices[pos];
      float* r = prims.data() + size_t(pos) * PV * 4;
      if (custom) {
        std::memcpy(r, prim_data + size_t(id) * prim_stride, prim_stride * 4);
        std::memcpy(r + prim_stride, prim_aabbs + size_t(id) * 2 * D, 2 * D * 4);
      } else {
        std::memcpy(r, prim_data + size_t(id) * prim_stride, payload * 4);
      }
      uint32_t w = id | (j + 1 == L.count ? kLeafBit : 0u);
      std::memcpy(&r[payload], &w, 4);
    }
  }

  // Four-wide records: each binary interior node whose parent is not folded
  // into it heads a record holding its children, with each interior child
  // replaced by that child's two children (two to four slots). Numbered in
  // depth-first order; slot sources point at the binary record slot that
  // holds the same box (refit copies them from there).
  std::vector<float> wnodes;
  std::vector<uint32_t> wsrc;
  if (ni > 0 && ks.ray_nearest_wide) {
    const uint32_t WV = wide_vec(D);
    std::vector<uint32_t> parent_slot(n_nodes, kNoHit);  // binary record << 1 | slot holding node i's box
    for (uint32_t i = 0; i < n_nodes; ++i) {
      if (prim_count[i] != 0) continue;
      parent_slot[child_a[i]] = b->h_iidx[i] << 1;
      parent_slot[child_b[i]] = (b->h_iidx[i] << 1) | 1u;
    }
    struct Item { uint32_t node, rec, depth; };
    std::vector<Item> todo{{0u, 0u, 1u}};
    wnodes.assign(size_t(WV) * 4, 0.f);
    wsrc.assign(4, kNoHit);
    uint32_t wdepth = 0;
    while (!todo.empty()) {
      const Item it = todo.back();
      todo.pop_back();
      wdepth = std::max(wdepth, it.depth);
      uint32_t kids[4], nk = 0;
      for (uint32_t c : {child_a[it.node], child_b[it.node]}) {
        if (prim_count[c] == 0) {
          kids[nk++] = child_a[c];
          kids[nk++] = child_b[c];
        } else {
          kids[nk++] = c;
        }
      }
      float* r = wnodes.data() + size_t(it.rec) * WV * 4;
      for (uint32_t k = 0; k < 4; ++k) {
        uint32_t code = kNoHit;
        if (k < nk) {
          const uint32_t c = kids[k];
          std::memcpy(r + k * 2 * D, node_bounds + size_t(c) * 2 * D, 2 * D * 4);
          wsrc[size_t(it.rec) * 4 + k] = parent_slot[c];
          if (prim_count[c] != 0) {
            code = kLeafBit | child_a[c];
          } else {
            code = uint32_t(wnodes.size() / (size_t(WV) * 4));
            wnodes.resize(wnodes.size() + size_t(WV) * 4, 0.f);
            wsrc.resize(wsrc.size() + 4, kNoHit);
            r = wnodes.data() + size_t(it.rec) * WV * 4;  // the vector may have moved
            todo.push_back({c, code, it.depth + 1});
          }
        }
        std::memcpy(&r[8 * D + k], &code, 4);
      }
    }
    b->n_wide = uint32_t(wnodes.size() / (size_t(WV) * 4));
    b->wroot = 0;
    b->wdepth = wdepth;
  }
  // The quantised copies of the four-wide records (the kernels that walk them).
  std::vector<uint32_t> qnodes;
  if (b->n_wide && ks.ray_nearest_quant) {
    const uint32_t WV = wide_vec(D), QV = quant_vec(D);
    qnodes.assign(size_t(b->n_wide) * QV * 4, 0u);
    for (uint32_t r = 0; r < b->n_wide; ++r) {
      const float* rec = wnodes.data() + size_t(r) * WV * 4;
      uint32_t codes[4];
      std::memcpy(codes, rec + 8 * D, sizeof(codes));
      uint32_t* out = qnodes.data() + size_t(r) * QV * 4;
      switch (D) {
        case 2: quantize_record<2>(rec, codes, out); break;
        case 3: quantize_record<3>(rec, codes, out); break;
        case 4: quantize_record<4>(rec, codes, out); break;
        case 6: quantize_record<6>(rec, codes, out); break;
        default: break;
      }
    }
  }

  auto up = [&](void** dst, const void* src, size_t bytes) -> int32_t {
    CK(cudaMalloc(dst, std::max<size_t>(bytes, 16)));
    if (src && bytes) CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    b->bytes += bytes;
    return SQ_OK;
  };
  int32_t rc;
  auto cleanup = [&](int32_t code_) {
    sq_bvh_destroy(b.release());
    return code_;
  };
  if ((rc = up((void**)&b->d_nodes, nodes.data(), nodes.size() * 4))) return cleanup(rc);
  if (b->n_wide) {
    if ((rc = up((void**)&b->d_wnodes, wnodes.data(), wnodes.size() * 4))) return cleanup(rc);
    if ((rc = up((void**)&b->d_wsrc, wsrc.data(), wsrc.size() * 4))) return cleanup(rc);
    if (!qnodes.empty() && (rc = up((void**)&b->d_qnodes, qnodes.data(), qnodes.size() * 4))) return cleanup(rc);
  }
  if ((rc = up((void**)&b->d_prims, prims.data(), prims.size() * 4))) return cleanup(rc);
  if ((rc = up((void**)&b->d_root, node_bounds, size_t(2) * D * 4))) return cleanup(rc);
  if ((rc = up((void**)&b->d_prim_ids, prim_indices, size_t(n_prims) * 4))) return cleanup(rc);
  if ((rc = up((void**)&b->d_leaves, leaves.data(), leaves.size() * sizeof(RefitLeaf)))) return cleanup(rc);
  if ((rc = up((void**)&b->d_parents, parents.data(), parents.size() * 4))) return cleanup(rc);
  if ((rc = up((void**)&b->d_arrivals, nullptr, parents.size() * 4))) return cleanup(rc);
  if (layers && (rc = up((void**)&b->d_layers, layers, size_t(n_prims) * 8))) return cleanup(rc);
  if (sub_objects && (rc = up((void**)&b->d_sub, sub_objects, size_t(n_prims) * 4))) return cleanup(rc);
  int nonfinite = 0;
  for (size_t k = 0; k < size_t(n_nodes) * 2 * D; ++k)
    if (!std::isfinite(node_bounds[k])) nonfinite = 1;
  if ((rc = up((void**)&b->d_nonfinite, &nonfinite, sizeof(int)))) return cleanup(rc);
  *out = b.release();
  return SQ_OK;
}

extern "C" int32_t sq_bvh_upload(sq_ctx* ctx, int32_t dim, int32_t narrow, uint32_t n_nodes,
                                 const float* node_bounds, const uint32_t* child_a, const uint32_t* child_b,
                                 const uint32_t* prim_count, uint32_t n_prims, const uint32_t* prim_indices,
                                 const float* prim_data, uint32_t prim_stride, const uint64_t* layers,
                                 const uint32_t* sub_objects, sq_bvh** out) {
  if (narrow == SQ_NARROW_CUSTOM) return fail(ctx, SQ_ERR_INVALID, "a consumer narrow phase uploads through sq_bvh_upload_custom");
  return upload_impl(ctx, dim, narrow, n_nodes, node_bounds, child_a, child_b, prim_count, n_prims, prim_indices,
                     prim_data, prim_stride, layers, sub_objects, nullptr, nullptr, out);
}

extern "C" int32_t sq_bvh_upload_custom(sq_ctx* ctx, uint32_t n_nodes, const float* node_bounds,
                                        const uint32_t* child_a, const uint32_t* child_b, const uint32_t* prim_count,
                                        uint32_t n_prims, const uint32_t* prim_indices, const float* prim_data,
                                        uint32_t prim_stride, const float* prim_aabbs, const char* narrow_src,
                                        sq_bvh** out) {
  if (!ctx || !out) return SQ_ERR_INVALID;
  *out = nullptr;
  if (!narrow_src) return fail(ctx, SQ_ERR_INVALID, "null narrow-phase source");
  if (prim_stride == 0 || prim_stride > kMaxCustomStride)
    return fail(ctx, SQ_ERR_INVALID, "prim_stride must be 1.." + std::to_string(kMaxCustomStride));
  if (n_prims && (!prim_aabbs || !prim_data)) return fail(ctx, SQ_ERR_INVALID, "null primitive data or AABBs");
  KernelSet ks;
  std::string log;
  CK(cudaSetDevice(ctx->device));
  const int32_t rc = rtc_kernel_set(prim_stride, narrow_src, &ks, &log);
  if (rc != SQ_OK) return fail(ctx, rc, log);
  return upload_impl(ctx, 3, SQ_NARROW_CUSTOM, n_nodes, node_bounds, child_a, child_b, prim_count, n_prims,
                     prim_indices, prim_data, prim_stride, nullptr, nullptr, prim_aabbs, &ks, out);
}

extern "C" int32_t sq_bvh_destroy(sq_bvh* b) {
  if (!b) return SQ_OK;
  cudaSetDevice(b->device);
  void* ptrs[] = {b->d_nodes, b->d_prims, b->d_root, b->d_layers, b->d_sub, b->d_prim_ids,
                  b->d_leaves, b->d_parents, b->d_arrivals, b->d_refit_in, b->d_nonfinite,
                  b->d_nb64, b->d_nc64, b->d_prims64, b->d_wnodes, b->d_wsrc, b->d_qnodes};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete b;
  return SQ_OK;
}

extern "C" int32_t sq_bvh_info_get(const sq_bvh* b, sq_bvh_info* o) {
  if (!b || !o) return SQ_ERR_INVALID;
  o->dim = b->dim;
  o->narrow = b->narrow;
  o->n_nodes = b->n_nodes;
  o->n_prims = b->n_prims;
  o->max_depth = b->depth;
  o->n_interior = b->n_interior;
  o->device_bytes = b->bytes;
  o->node_record_bytes = node_vec(b->dim) * 16;
  o->prim_record_bytes = b->prim_vec * 16;
  return SQ_OK;
}

extern "C" int32_t sq_bvh_refit_d(sq_ctx* ctx, sq_bvh* b, const float* d_prim_data) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (b->n_nodes == 0) return SQ_OK;
  if (!d_prim_data) return fail(ctx, SQ_ERR_INVALID, "null prim data");
  if (!b->ks.refit_leaves) return fail(ctx, SQ_ERR_UNSUPPORTED, "this scene's narrow phase has no refit");
  CK(cudaMemsetAsync(b->d_arrivals, 0, size_t(std::max<uint32_t>(b->n_interior, 1)) * 4, ctx->stream));
  CK(cudaMemsetAsync(b->d_nonfinite, 0, sizeof(int), ctx->stream));
  RefitParams p;
  p.nonfinite = b->d_nonfinite;
  p.nodes = b->d_nodes;
  p.prims = b->d_prims;
  p.root_box = b->d_root;
  p.prim_data = d_prim_data;
  p.prim_ids = b->d_prim_ids;
  p.leaves = b->d_leaves;
  p.parents = b->d_parents;
  p.arrivals = b->d_arrivals;
  p.n_leaves = b->n_leaves;
  p.stride = b->stride;
  void* args[] = {&p};
  CK(cudaLaunchKernel(b->ks.refit_leaves, dim3((b->n_leaves + 255) / 256), dim3(256), args, 0, ctx->stream));
  ctx->launches++;
  if (b->n_wide && b->ks.wide_sync) {
    // The four-wide records take their boxes from the refit binary records.
    float4* wn = b->d_wnodes;
    const float4* bn = b->d_nodes;
    const uint32_t* src = b->d_wsrc;
    uint32_t slots = b->n_wide * 4;
    void* wargs[] = {&wn, &bn, &src, &slots};
    CK(cudaLaunchKernel(b->ks.wide_sync, dim3((slots + 255) / 256), dim3(256), wargs, 0, ctx->stream));
    ctx->launches++;
    if (b->d_qnodes && b->ks.quant_sync) {
      float4* qn = b->d_qnodes;
      const float4* wsrc4 = b->d_wnodes;
      uint32_t recs = b->n_wide;
      void* qargs[] = {&qn, &wsrc4, &recs};
      CK(cudaLaunchKernel(b->ks.quant_sync, dim3((recs + 127) / 128), dim3(128), qargs, 0, ctx->stream));
      ctx->launches++;
    }
  }
  return finish(ctx);
}

extern "C" int32_t sq_bvh_refit(sq_ctx* ctx, sq_bvh* b, const float* prim_data) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (b->n_nodes == 0) return SQ_OK;
  if (!prim_data) return fail(ctx, SQ_ERR_INVALID, "null prim data");
  size_t bytes = size_t(b->n_prims) * b->stride * 4;
  if (!b->d_refit_in) CK(cudaMalloc(&b->d_refit_in, bytes));
  CK(cudaMemcpyAsync(b->d_refit_in, prim_data, bytes, cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = sq_bvh_refit_d(ctx, b, b->d_refit_in))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

extern "C" int32_t sq_bvh_read_bounds(sq_ctx* ctx, const sq_bvh* b, float* node_bounds) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (b->n_nodes == 0) return SQ_OK;
  if (!node_bounds) return fail(ctx, SQ_ERR_INVALID, "null output");
  const int D = b->dim;
  const uint32_t NV = node_vec(D);
  std::vector<float> nodes(size_t(std::max<uint32_t>(b->n_interior, 1)) * NV * 4);
  std::vector<float> root(2 * D);
  CK(cudaMemcpyAsync(nodes.data(), b->d_nodes, nodes.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(root.data(), b->d_root, root.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::memcpy(node_bounds, root.data(), root.size() * 4);
  for (uint32_t i = 0; i < b->n_nodes; ++i) {
    if (b->h_count[i] != 0) continue;
    const float* r = nodes.data() + size_t(b->h_iidx[i]) * NV * 4;
    std::memcpy(node_bounds + size_t(b->h_child_a[i]) * 2 * D, r, 2 * D * 4);
    std::memcpy(node_bounds + size_t(b->h_child_b[i]) * 2 * D, r + 2 * D, 2 * D * 4);
  }
  return SQ_OK;
}

// ============================================================================
// queries: device-pointer entry points
// ============================================================================

extern "C" int32_t sq_raycast_nearest_d(sq_ctx* ctx, const sq_bvh* b, const float* d_rays, uint32_t n,
                                        float max_toi, const float* d_mt, const sq_filter* f, const sq_hits* o,
                                        sq_query_stats* st) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!o || (n && !d_rays)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  if ((rc = stats_begin(ctx, st))) return rc;
  if ((rc = nearest_core(ctx, b, false, d_rays, n, max_toi, d_mt, f, *o, st != nullptr))) return rc;
  if ((rc = finish(ctx))) return rc;
  return stats_end(ctx, st);
}

extern "C" int32_t sq_shapecast_nearest_d(sq_ctx* ctx, const sq_bvh* b, const float* d_casts, uint32_t n,
                                          float max_toi, const float* d_mt, const sq_filter* f, const sq_hits* o) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!o || (n && !d_casts)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  if ((rc = nearest_core(ctx, b, true, d_casts, n, max_toi, d_mt, f, *o, false))) return rc;
  return finish(ctx);
}

extern "C" int32_t sq_raycast_all_d(sq_ctx* ctx, const sq_bvh* b, const float* d_rays, uint32_t n, float max_toi,
                                    const float* d_mt, const sq_filter* f, const sq_hit_lists* o,
                                    sq_query_stats* st) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!o || (n && !d_rays)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  if ((rc = stats_begin(ctx, st))) return rc;
  if ((rc = list_core(ctx, b, kRayAll, d_rays, n, max_toi, d_mt, f, *o, st != nullptr))) return rc;
  if ((rc = finish(ctx))) return rc;
  return stats_end(ctx, st);
}

extern "C" int32_t sq_raycast_crossings_d(sq_ctx* ctx, const sq_bvh* b, const float* d_rays, uint32_t n,
                                          float max_toi, const float* d_mt, const sq_filter* f,
                                          const sq_hit_lists* o) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!o || (n && !d_rays)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  if ((rc = list_core(ctx, b, 100, d_rays, n, max_toi, d_mt, f, *o, false))) return rc;
  return finish(ctx);
}

extern "C" int32_t sq_shapecast_all_d(sq_ctx* ctx, const sq_bvh* b, const float* d_casts, uint32_t n,
                                      float max_toi, const float* d_mt, const sq_filter* f, const sq_hit_lists* o) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!o || (n && !d_casts)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  if ((rc = list_core(ctx, b, kCastAll, d_casts, n, max_toi, d_mt, f, *o, false))) return rc;
  return finish(ctx);
}

namespace {

// Overlap on device buffers: count pass, exclusive scan into offsets, total
// read back, fill pass. `scratch` holds n + 1 u32 counts and the scan's
// temporary storage (scratch_bytes from overlap_scratch_bytes).
size_t overlap_scan_temp(uint32_t n) {
  size_t temp = 0;
  cub::DeviceScan::ExclusiveScan(nullptr, temp, (const uint32_t*)nullptr, (unsigned long long*)nullptr,
                                 cuda::std::plus<>{}, 0ull, int(n) + 1);
  return temp;
}

// Scratch of overlap_core: per-region counts, the heavy-region list and
// flags, their counter and store cursor, the count pass's kept leaves, the
// heavy regions' staged-leaf slots and store (n entries each), then the
// scan's temporary storage.
size_t overlap_scratch_bytes(uint32_t n) {
  const auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  return al((size_t(n) + 1) * 4) + al(size_t(n) * 4 + 4) + al(size_t(n) + 1) + al(16) +
         al(size_t(n) * kOverlapKeep * 4) + 2 * al(size_t(n) * 4 + 4) + overlap_scan_temp(n) + 256;
}

// Records a region may visit before the block-per-region kernel takes it.
constexpr uint32_t kOverlapVisitBudget = 128;

// Launches overlap_heavy_kernel over the regions the count pass listed (a
// block per region, one shared stack of 256 x (depth + 1) entries).
int32_t launch_heavy(sq_ctx* ctx, const sq_bvh* b, QueryParams& p) {
  const uint32_t cap = 256u * (b->depth + 1);
  p.stack = int(cap);
  const size_t smem = size_t(cap) * 4;
  if (smem + kHeavyStage * 4 + 1024 > 48 * 1024) CK(cudaFuncSetAttribute(b->ks.overlap_heavy, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  void* args[] = {&p};
  CK(cudaLaunchKernel(b->ks.overlap_heavy, dim3(ctx->sm_count * 4), dim3(32 * kHeavyWarps), args, smem, ctx->stream));
  ctx->launches++;
  return SQ_OK;
}

int32_t overlap_core(sq_ctx* ctx, const sq_bvh* b, const float* d_regions, uint32_t n, const sq_filter* f,
                     uint64_t* d_offsets, uint32_t* d_leaves, uint64_t cap, uint64_t* total, void* scratch,
                     size_t scratch_bytes) {
  if (!b->ks.overlap) return fail(ctx, SQ_ERR_UNSUPPORTED, "this scene's narrow phase has no overlap query");
  const auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
  Carve sc;
  const size_t o_cnt = sc.take((size_t(n) + 1) * 4), o_hl = sc.take(size_t(n) * 4 + 4), o_hf = sc.take(size_t(n) + 1),
               o_hc = sc.take(16), o_keep = sc.take(size_t(n) * kOverlapKeep * 4),
               o_hst = sc.take(size_t(n) * 4 + 4), o_hsto = sc.take(size_t(n) * 4 + 4);
  (void)al;
  uint32_t* d_keep = (uint32_t*)((char*)scratch + o_keep);
  uint32_t* d_hstart = (uint32_t*)((char*)scratch + o_hst);
  uint32_t* d_hstore = (uint32_t*)((char*)scratch + o_hsto);
  uint32_t* d_counts = (uint32_t*)((char*)scratch + o_cnt);
  uint32_t* d_hlist = (uint32_t*)((char*)scratch + o_hl);
  uint8_t* d_hflag = (uint8_t*)((char*)scratch + o_hf);
  uint32_t* d_hcount = (uint32_t*)((char*)scratch + o_hc);
  void* temp = (char*)scratch + sc.off;
  size_t temp_bytes = scratch_bytes - sc.off;
  CK(cudaMemsetAsync(d_counts, 0, size_t(n + 1) * 4, ctx->stream));
  CK(cudaMemsetAsync(d_hflag, 0, size_t(n) + 1, ctx->stream));
  CK(cudaMemsetAsync(d_hcount, 0, 8, ctx->stream));  // list count, store cursor
  CK(cudaMemsetAsync(d_hstart, 0xFF, size_t(n) * 4, ctx->stream));
  const bool heavy = b->ks.overlap_heavy != nullptr;
  if (b->n_nodes != 0 && n != 0) {
    QueryParams p;
    base_params(b, f, p);
    p.queries = d_regions;
    p.n = n;
    p.out_count = d_counts;
    p.fill = 0;
    p.keep = d_keep;
    if (heavy) {
      p.heavy_list = d_hlist;
      p.heavy_count = d_hcount;
      p.heavy_flag = d_hflag;
      p.visit_budget = kOverlapVisitBudget;
      p.heavy_store = d_hstore;
      p.heavy_start = d_hstart;
      p.heavy_cursor = d_hcount + 1;
      p.heavy_cap = n;
    }
    int32_t rc = launch_persistent(ctx, b->ks.overlap, p, b->depth, p.n);
    if (rc) return rc;
    if (heavy && (rc = launch_heavy(ctx, b, p))) return rc;
  }
  CK(cub::DeviceScan::ExclusiveScan(temp, temp_bytes, d_counts, (unsigned long long*)d_offsets, cuda::std::plus<>{},
                                    0ull, int(n) + 1, ctx->stream));
  ctx->launches++;
  unsigned long long tot = 0;
  uint32_t hc = 0;
  CK(cudaMemcpyAsync(&tot, d_offsets + n, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&hc, d_hcount, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (hc & 0x80000000u) return fail(ctx, SQ_ERR_CAPACITY, "overlap: a heavy region's node stack overflowed");
  if (total) *total = tot;
  if (tot > cap) return fail(ctx, SQ_ERR_CAPACITY, "overlap results exceed leaf_capacity");
  if (tot && b->n_nodes != 0) {
    QueryParams p;
    base_params(b, f, p);
    p.queries = d_regions;
    p.n = n;
    p.out_count = d_counts;
    p.fill = 2;
    p.csr_offsets = (const unsigned long long*)d_offsets;
    p.csr_leaves = d_leaves;
    p.keep = d_keep;
    if (heavy) {
      p.heavy_list = d_hlist;
      p.heavy_count = d_hcount;
      p.heavy_flag = d_hflag;
      p.heavy_store = d_hstore;
      p.heavy_start = d_hstart;
    }
    int32_t rc = launch_persistent(ctx, b->ks.overlap, p, b->depth, p.n);
    if (rc) return rc;
    if (heavy && hc && (rc = launch_heavy(ctx, b, p))) return rc;
    if ((rc = sort_csr_segments(ctx, d_leaves, tot, d_offsets, n))) return rc;
  }
  return SQ_OK;
}

}  // namespace

extern "C" int32_t sq_overlap_d(sq_ctx* ctx, const sq_bvh* b, const float* d_regions, uint32_t n,
                                const sq_filter* f, uint64_t* d_offsets, uint32_t* d_leaves, uint64_t cap,
                                uint64_t* total) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!d_offsets || (n && !d_regions)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  size_t need = overlap_scratch_bytes(n);
  if ((rc = arena_reserve(ctx, need))) return rc;
  if ((rc = overlap_core(ctx, b, d_regions, n, f, d_offsets, d_leaves, cap, total, ctx->arena.p, need))) return rc;
  if ((rc = finish(ctx))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

// ============================================================================
// queries: host-buffer entry points (copy in, run, copy out, wait)
// ============================================================================

namespace {

struct HostRun {
  sq_ctx* ctx;
  Carve cv;
  char* base() const { return (char*)ctx->arena.p; }
};

int32_t h2d(sq_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return SQ_OK;
}
int32_t d2h(sq_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (dst && bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return SQ_OK;
}

int32_t host_nearest(sq_ctx* ctx, const sq_bvh* b, bool cast, const float* q, uint32_t n, float max_toi,
                     const float* mt, const sq_filter* f, const sq_hits* o, sq_query_stats* st) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!o || !o->leaf || (n && !q)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  if (n == 0) {
    if (st) *st = sq_query_stats{0, 0, 0, 0};
    return SQ_OK;
  }
  const int D = b->dim;
  const size_t qb = size_t(n) * (cast ? 4 : 2) * D * 4;
  Carve cv;
  size_t o_q = cv.take(qb), o_mt = mt ? cv.take(size_t(n) * 4) : 0;
  size_t o_leaf = cv.take(size_t(n) * 4), o_toi = o->toi ? cv.take(size_t(n) * 4) : 0;
  size_t o_sub = o->sub_object ? cv.take(size_t(n) * 4) : 0;
  size_t o_nrm = o->normal ? cv.take(size_t(n) * D * 4) : 0;
  size_t o_pt = o->point ? cv.take(size_t(n) * D * 4) : 0;
  if ((rc = arena_reserve(ctx, cv.off))) return rc;
  char* base = (char*)ctx->arena.p;
  sq_hits dh;
  dh.leaf = (uint32_t*)(base + o_leaf);
  dh.toi = o->toi ? (float*)(base + o_toi) : nullptr;
  dh.sub_object = o->sub_object ? (uint32_t*)(base + o_sub) : nullptr;
  dh.normal = o->normal ? (float*)(base + o_nrm) : nullptr;
  dh.point = o->point ? (float*)(base + o_pt) : nullptr;
  if (!st) {
    // Chunked: copies in and out overlap the traversal of other chunks.
    const size_t qw = size_t(cast ? 4 : 2) * D;
    auto in = [&](uint32_t s0, uint32_t m, cudaStream_t sm) -> int32_t {
      CK(cudaMemcpyAsync(base + o_q + size_t(s0) * qw * 4, q + size_t(s0) * qw, size_t(m) * qw * 4,
                         cudaMemcpyHostToDevice, sm));
      if (mt) CK(cudaMemcpyAsync(base + o_mt + size_t(s0) * 4, mt + s0, size_t(m) * 4, cudaMemcpyHostToDevice, sm));
      return SQ_OK;
    };
    auto run = [&](sq_ctx* lane, uint32_t s0, uint32_t m) -> int32_t {
      sq_hits c = dh;
      c.leaf += s0;
      if (c.toi) c.toi += s0;
      if (c.sub_object) c.sub_object += s0;
      if (c.normal) c.normal += size_t(s0) * D;
      if (c.point) c.point += size_t(s0) * D;
      return nearest_core(lane, b, cast, (const float*)(base + o_q) + size_t(s0) * qw, m, max_toi,
                          mt ? (const float*)(base + o_mt) + s0 : nullptr, f, c, false);
    };
    auto out = [&](uint32_t s0, uint32_t m, cudaStream_t sm) -> int32_t {
      auto cp = [&](void* dst, const void* src, size_t per) -> int32_t {
        if (dst) CK(cudaMemcpyAsync((char*)dst + size_t(s0) * per, (const char*)src + size_t(s0) * per, size_t(m) * per,
                                    cudaMemcpyDeviceToHost, sm));
        return SQ_OK;
      };
      int32_t r;
      if ((r = cp(o->leaf, dh.leaf, 4)) || (r = cp(o->toi, dh.toi, 4)) || (r = cp(o->sub_object, dh.sub_object, 4)) ||
          (r = cp(o->normal, dh.normal, size_t(D) * 4)) || (r = cp(o->point, dh.point, size_t(D) * 4)))
        return r;
      return SQ_OK;
    };
    if ((rc = pipelined(ctx, n, in, run, out))) return rc;
    return finish(ctx);
  }
  if ((rc = h2d(ctx, base + o_q, q, qb))) return rc;
  if (mt && (rc = h2d(ctx, base + o_mt, mt, size_t(n) * 4))) return rc;
  if ((rc = stats_begin(ctx, cast ? nullptr : st))) return rc;
  if ((rc = nearest_core(ctx, b, cast, (const float*)(base + o_q), n, max_toi,
                         mt ? (const float*)(base + o_mt) : nullptr, f, dh, st && !cast)))
    return rc;
  if ((rc = finish(ctx))) return rc;
  if ((rc = d2h(ctx, o->leaf, dh.leaf, size_t(n) * 4))) return rc;
  if ((rc = d2h(ctx, o->toi, dh.toi, size_t(n) * 4))) return rc;
  if ((rc = d2h(ctx, o->sub_object, dh.sub_object, size_t(n) * 4))) return rc;
  if ((rc = d2h(ctx, o->normal, dh.normal, size_t(n) * D * 4))) return rc;
  if ((rc = d2h(ctx, o->point, dh.point, size_t(n) * D * 4))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  if (!cast) return stats_end(ctx, st);
  return SQ_OK;
}

int32_t host_list(sq_ctx* ctx, const sq_bvh* b, int kind, const float* q, uint32_t n, float max_toi,
                  const float* mt, const sq_filter* f, const sq_hit_lists* o, sq_query_stats* st) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!o || !o->count || (n && !q) || (n && o->k && (!o->leaf || !o->toi)))
    return fail(ctx, SQ_ERR_INVALID, "null argument");
  if (n == 0) {
    if (st) *st = sq_query_stats{0, 0, 0, 0};
    return SQ_OK;
  }
  const int D = b->dim;
  const bool cast = kind == kCastAll;
  const size_t qb = size_t(n) * (cast ? 4 : 2) * D * 4;
  const size_t nk = size_t(n) * o->k;
  Carve cv;
  size_t o_q = cv.take(qb), o_mt = mt ? cv.take(size_t(n) * 4) : 0;
  size_t o_cnt = cv.take(size_t(n) * 4);
  size_t o_leaf = cv.take(nk * 4), o_toi = cv.take(nk * 4);
  size_t o_sub = o->sub_object ? cv.take(nk * 4) : 0;
  size_t o_nrm = o->normal ? cv.take(nk * D * 4) : 0;
  if ((rc = arena_reserve(ctx, cv.off))) return rc;
  char* base = (char*)ctx->arena.p;
  if ((rc = h2d(ctx, base + o_q, q, qb))) return rc;
  if (mt && (rc = h2d(ctx, base + o_mt, mt, size_t(n) * 4))) return rc;
  sq_hit_lists dl;
  dl.k = o->k;
  dl.count = (uint32_t*)(base + o_cnt);
  dl.leaf = (uint32_t*)(base + o_leaf);
  dl.toi = (float*)(base + o_toi);
  dl.sub_object = o->sub_object ? (uint32_t*)(base + o_sub) : nullptr;
  dl.normal = o->normal ? (float*)(base + o_nrm) : nullptr;
  // Entries past min(count, k) are unspecified; give them a defined value
  // in host-buffer calls so callers comparing whole buffers see no garbage.
  CK(cudaMemsetAsync(dl.leaf, 0xFF, nk * 4, ctx->stream));
  CK(cudaMemsetAsync(dl.toi, 0, nk * 4, ctx->stream));
  if (dl.sub_object) CK(cudaMemsetAsync(dl.sub_object, 0xFF, nk * 4, ctx->stream));
  if (dl.normal) CK(cudaMemsetAsync(dl.normal, 0, nk * D * 4, ctx->stream));
  if ((rc = stats_begin(ctx, st))) return rc;
  if ((rc = list_core(ctx, b, kind, (const float*)(base + o_q), n, max_toi, mt ? (const float*)(base + o_mt) : nullptr,
                      f, dl, st != nullptr)))
    return rc;
  if ((rc = finish(ctx))) return rc;
  if ((rc = d2h(ctx, o->count, dl.count, size_t(n) * 4))) return rc;
  if ((rc = d2h(ctx, o->leaf, dl.leaf, nk * 4))) return rc;
  if ((rc = d2h(ctx, o->toi, dl.toi, nk * 4))) return rc;
  if ((rc = d2h(ctx, o->sub_object, dl.sub_object, nk * 4))) return rc;
  if ((rc = d2h(ctx, o->normal, dl.normal, nk * D * 4))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return stats_end(ctx, st);
}

}  // namespace

extern "C" int32_t sq_raycast_nearest(sq_ctx* ctx, const sq_bvh* b, const float* rays, uint32_t n, float max_toi,
                                      const float* mt, const sq_filter* f, const sq_hits* o, sq_query_stats* st) {
  return host_nearest(ctx, b, false, rays, n, max_toi, mt, f, o, st);
}

extern "C" int32_t sq_shapecast_nearest(sq_ctx* ctx, const sq_bvh* b, const float* casts, uint32_t n,
                                        float max_toi, const float* mt, const sq_filter* f, const sq_hits* o) {
  return host_nearest(ctx, b, true, casts, n, max_toi, mt, f, o, nullptr);
}

extern "C" int32_t sq_raycast_all(sq_ctx* ctx, const sq_bvh* b, const float* rays, uint32_t n, float max_toi,
                                  const float* mt, const sq_filter* f, const sq_hit_lists* o, sq_query_stats* st) {
  return host_list(ctx, b, kRayAll, rays, n, max_toi, mt, f, o, st);
}

extern "C" int32_t sq_raycast_crossings(sq_ctx* ctx, const sq_bvh* b, const float* rays, uint32_t n,
                                        float max_toi, const float* mt, const sq_filter* f, const sq_hit_lists* o) {
  return host_list(ctx, b, 100, rays, n, max_toi, mt, f, o, nullptr);
}

extern "C" int32_t sq_shapecast_all(sq_ctx* ctx, const sq_bvh* b, const float* casts, uint32_t n, float max_toi,
                                    const float* mt, const sq_filter* f, const sq_hit_lists* o) {
  return host_list(ctx, b, kCastAll, casts, n, max_toi, mt, f, o, nullptr);
}

extern "C" int32_t sq_overlap(sq_ctx* ctx, const sq_bvh* b, const float* regions, uint32_t n, const sq_filter* f,
                              uint64_t* offsets, uint32_t* leaves, uint64_t cap, uint64_t* total) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!offsets || (n && !regions)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  const int D = b->dim;
  const size_t rb = size_t(n) * 2 * D * 4;
  const size_t scan = overlap_scratch_bytes(n);
  Carve cv;
  size_t o_r = cv.take(rb), o_off = cv.take((size_t(n) + 1) * 8), o_lv = cv.take(std::max<uint64_t>(cap, 1) * 4);
  size_t o_scr = cv.take(scan);
  if ((rc = arena_reserve(ctx, cv.off))) return rc;
  char* base = (char*)ctx->arena.p;
  if ((rc = h2d(ctx, base + o_r, regions, rb))) return rc;
  uint64_t tot = 0;
  rc = overlap_core(ctx, b, (const float*)(base + o_r), n, f, (uint64_t*)(base + o_off), (uint32_t*)(base + o_lv), cap,
                    &tot, base + o_scr, scan);
  if (total) *total = tot;
  if (rc && rc != SQ_ERR_CAPACITY) return rc;
  int32_t rc2;
  if ((rc2 = d2h(ctx, offsets, base + o_off, (size_t(n) + 1) * 8))) return rc2;
  if (rc == SQ_OK && (rc2 = d2h(ctx, leaves, base + o_lv, tot * 4))) return rc2;
  CK(cudaStreamSynchronize(ctx->stream));
  if ((rc2 = finish(ctx))) return rc2;
  return rc;
}

// ============================================================================
// Overlap without allocation.
//
// For callers that may not allocate device memory at query time: a host
// engine that owns a fixed device-memory budget and forbids driver
// allocations, a real-time loop where an allocation's latency is not
// allowed, or code that has no context object to hold one. The scratch this
// query needs -- per-region counts and the persistent kernels' work
// counters -- lives in one file-scope device array, sized for at most
// kNoAllocMaxRegions regions (about 4 MiB, held by every GPU that loads the
// library until the process exits).
// ============================================================================

namespace {

constexpr uint32_t kNoAllocMaxRegions = 1u << 20;
constexpr uint32_t kNoAllocCounters = 2;  // work counters of the count and fill launches

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocMaxRegions + 1 + kNoAllocCounters];

struct NoAllocDevice {
  bool ready = false;
  uint32_t* scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int sm_count = 0;
};

constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

// Exclusive prefix sum of n counts into offsets[0..n], offsets[n] = total, in
// one block (n <= kNoAllocMaxRegions) and no scratch beyond shared memory:
// tiles of 1,024 consecutive counts (one per thread, so the loads coalesce)
// are scanned block-wide (warp shuffles, then the 32 warp totals), and the
// running total carries from tile to tile.
__global__ void __launch_bounds__(1024) noalloc_scan_kernel(const uint32_t* counts, unsigned long long* offsets,
                                                            uint32_t n) {
  __shared__ unsigned long long warp_sum[32];
  constexpr unsigned FULL = 0xffffffffu;
  const uint32_t t = threadIdx.x, lane = t & 31u, w = t >> 5;
  unsigned long long carry = 0;
  for (uint32_t base = 0; base < n; base += 1024u) {
    const uint32_t i = base + t;
    const unsigned long long v = i < n ? counts[i] : 0ull;
    unsigned long long x = v;  // inclusive scan within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(FULL, x, o);
      if (lane >= uint32_t(o)) x += y;
    }
    if (lane == 31u) warp_sum[w] = x;
    __syncthreads();
    if (w == 0) {
      unsigned long long s = warp_sum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(FULL, s, o);
        if (lane >= uint32_t(o)) s += y;
      }
      warp_sum[lane] = s;  // inclusive over warps
    }
    __syncthreads();
    if (i < n) offsets[i] = carry + (w ? warp_sum[w - 1] : 0ull) + (x - v);
    carry += warp_sum[31];
    __syncthreads();  // warp_sum is rewritten by the next tile
  }
  if (t == 0) offsets[n] = carry;
}

}  // namespace

// The device address of the static scratch, looked up once per device (with
// that device current) by the first call on it.
static int32_t noalloc_setup(int device, NoAllocDevice** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return SQ_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc_dev[device];
  if (!d.ready) {
    if (cudaSetDevice(device) != cudaSuccess) return SQ_ERR_CUDA;
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) {
      cudaGetLastError();
      return SQ_ERR_CUDA;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return SQ_ERR_CUDA;
    d.scratch = static_cast<uint32_t*>(ptr);
    d.sm_count = sms;
    d.ready = true;
  }
  *out = &d;
  return SQ_OK;
}

extern "C" int32_t sq_overlap_noalloc(const sq_bvh* b, const float* d_regions, uint32_t n, const sq_filter* f,
                                      uint64_t* d_offsets, uint32_t* d_leaves, uint64_t leaf_capacity,
                                      uint64_t* total, void* stream) {
  if (!b || !d_offsets || !total || (n && !d_regions)) return SQ_ERR_INVALID;
  if (n > kNoAllocMaxRegions) return SQ_ERR_CAPACITY;  // beyond the static scratch
  if (!b->ks.overlap) return SQ_ERR_UNSUPPORTED;
  NoAllocDevice* d = nullptr;
  int32_t rc = noalloc_setup(b->device, &d);
  if (rc) return rc;
  if (cudaSetDevice(b->device) != cudaSuccess) return SQ_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t* counts = d->scratch;
  uint32_t* counters = d->scratch + kNoAllocMaxRegions + 1;
  // Every call shares the scratch: the counts and both work counters start at zero.
  if (cudaMemsetAsync(counts, 0, (size_t(n) + 1) * sizeof(uint32_t), s) != cudaSuccess ||
      cudaMemsetAsync(counters, 0, kNoAllocCounters * sizeof(uint32_t), s) != cudaSuccess)
    return SQ_ERR_CUDA;
  const int stack = int(std::max<uint32_t>(b->depth, 1));
  const size_t smem = size_t(stack) * kThreads * 8;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(b->ks.overlap, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return SQ_ERR_CUDA;
  // The persistent grid: the blocks of this scene's overlap kernel (its D,
  // narrow phase, consumer code) that fit at once with this tree's stack.
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, b->ks.overlap, kThreads, smem) != cudaSuccess || bps < 1)
    bps = 1;
  const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(d->sm_count) * bps,
                                                                  (uint64_t(n) + kThreads - 1) / kThreads));
  if (b->n_nodes != 0 && n != 0) {
    QueryParams p;
    base_params(b, f, p);
    p.queries = d_regions;
    p.n = n;
    p.out_count = counts;
    p.fill = 0;
    p.counter = counters;
    p.stack = stack;
    void* args[] = {&p};
    if (cudaLaunchKernel(b->ks.overlap, dim3(unsigned(grid)), dim3(kThreads), args, smem, s) != cudaSuccess)
      return SQ_ERR_CUDA;
  }
  {
    // Launched with cudaLaunchKernel so its status is this launch's own (a
    // stale error of the caller's earlier work is neither reported nor cleared).
    const uint32_t* c_counts = counts;
    unsigned long long* c_offsets = reinterpret_cast<unsigned long long*>(d_offsets);
    uint32_t c_n = n;
    void* args[] = {&c_counts, &c_offsets, &c_n};
    if (cudaLaunchKernel(reinterpret_cast<const void*>(noalloc_scan_kernel), dim3(1), dim3(1024), args, 0, s) !=
        cudaSuccess)
      return SQ_ERR_CUDA;
  }
  unsigned long long tot = 0;
  if (cudaMemcpyAsync(&tot, d_offsets + n, sizeof(tot), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return SQ_ERR_CUDA;
  *total = tot;
  if (tot > leaf_capacity) return SQ_ERR_CAPACITY;
  if (tot && b->n_nodes != 0) {
    if (!d_leaves) return SQ_ERR_INVALID;
    QueryParams p;
    base_params(b, f, p);
    p.queries = d_regions;
    p.n = n;
    p.out_count = counts;
    p.fill = 1;
    p.csr_offsets = reinterpret_cast<const unsigned long long*>(d_offsets);
    p.csr_leaves = d_leaves;
    p.counter = counters + 1;
    p.stack = stack;
    void* args[] = {&p};
    if (cudaLaunchKernel(b->ks.overlap, dim3(unsigned(grid)), dim3(kThreads), args, smem, s) != cudaSuccess)
      return SQ_ERR_CUDA;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return SQ_ERR_CUDA;
  return SQ_OK;
}

// ============================================================================
// learned-seeded nearest rays (the learned guide's query, include/sq_guide.h)
// ============================================================================

int32_t sqi::seeded_nearest(sq_ctx* ctx, const sq_bvh* b, const float* d_rays, uint32_t n, float max_toi,
                            const int32_t* d_bucket, const SeedTable& seeds, const sq_hits& o, sq_query_stats* st) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!o.leaf || (n && (!d_rays || !d_bucket))) return fail(ctx, SQ_ERR_INVALID, "null argument");
  if (!b->ks.ray_nearest_seeded[0]) return fail(ctx, SQ_ERR_UNSUPPORTED, "seeded queries need a D = 3 scene");
  if ((rc = stats_begin(ctx, st))) return rc;
  if (n && b->n_nodes == 0) {
    if ((rc = nearest_core(ctx, b, false, d_rays, n, max_toi, nullptr, nullptr, o, false))) return rc;
  } else if (n) {
    QueryParams p;
    base_params(b, nullptr, p);
    p.queries = d_rays;
    p.max_toi = max_toi;
    p.n = n;
    p.out_leaf = o.leaf;
    p.out_toi = o.toi;
    p.out_sub = o.sub_object;
    p.out_normal = o.normal;
    p.out_point = o.point;
    p.seed_bucket = d_bucket;
    p.buckets = seeds.buckets;
    p.bucket_sibs = seeds.sibs;
    p.n_buckets = seeds.n_buckets;
    p.sib_stride = seeds.sib_stride;
    // The walk after the bucket follows the context's order: near-first, or
    // the crate's own child order (still certified: the seed changes the
    // visiting order, so the crate's counters are not replayed).
    p.far_first = ctx->order == SQ_ORDER_REFERENCE ? 1 : 0;
    if (st) p.stats = ctx->d_stats;
    // The bucket's ancestors' other children wait on the stack (one per level
    // above the bucket) while the bucket is searched: no deeper than a plain
    // descent to the same node, so the tree's depth bounds the stack.
    if ((rc = near_first_launch(ctx, b, b->ks.ray_nearest_seeded[st ? 1 : 0],
                                kReplayInKernel ? nullptr : b->ks.ray_nearest[1][st ? 1 : 0], p,
                                b->depth + 1)))
      return rc;
  }
  if ((rc = finish(ctx))) return rc;
  return stats_end(ctx, st);
}

// Each query's CSR segment of leaves in ascending order: one segmented sort
// over all segments (the fill pass appends in walk order), with scratch
// from the context's memory pool.
int32_t sqi::sort_csr_segments(sq_ctx* ctx, uint32_t* d_leaves, uint64_t total, const uint64_t* d_offsets, uint32_t n) {
  if (total < 2) return SQ_OK;
  if (total > uint64_t(INT32_MAX)) return fail(ctx, SQ_ERR_CAPACITY, "more than 2^31 overlap results");
  const auto* beg = reinterpret_cast<const unsigned long long*>(d_offsets);
  size_t temp_bytes = 0;
  cub::DoubleBuffer<uint32_t> keys(d_leaves, nullptr);
  CK(cub::DeviceSegmentedSort::SortKeys(nullptr, temp_bytes, keys, int(total), int(n), beg, beg + 1, ctx->stream));
  const size_t alt_bytes = (size_t(total) * 4 + 255) & ~size_t(255);
  char* tmp = nullptr;
  CK(scratch_alloc(ctx, reinterpret_cast<void**>(&tmp), alt_bytes + temp_bytes));
  keys = cub::DoubleBuffer<uint32_t>(d_leaves, reinterpret_cast<uint32_t*>(tmp));
  cudaError_t e = cub::DeviceSegmentedSort::SortKeys(tmp + alt_bytes, temp_bytes, keys, int(total), int(n), beg, beg + 1,
                                                     ctx->stream);
  if (e == cudaSuccess && keys.Current() != d_leaves)
    e = cudaMemcpyAsync(d_leaves, keys.Current(), size_t(total) * 4, cudaMemcpyDeviceToDevice, ctx->stream);
  cudaFreeAsync(tmp, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, "segmented sort of overlap results", e);
  ctx->launches++;
  return SQ_OK;
}

int32_t sqi::second_lane(sq_ctx* ctx, sq_ctx** out) {
  if (!ctx->lane) {
    sq_ctx* l = nullptr;
    int32_t rc = sq_ctx_create(ctx->device, &l);
    if (rc) return fail(ctx, rc, "second compute lane");
    ctx->lane = l;
  }
  sq_ctx* lane = ctx->lane;
  lane->order = ctx->order;
  lane->blocks_per_sm = ctx->blocks_per_sm;
  lane->window = ctx->window;
  lane->layout = ctx->layout;
  if (lane->l2_window.num_bytes != ctx->l2_window.num_bytes || lane->l2_window.base_ptr != ctx->l2_window.base_ptr) {
    lane->l2_window = ctx->l2_window;
    int32_t rc = apply_l2_window(lane);
    if (rc) return fail(ctx, rc, lane->err.c_str());
  }
  *out = lane;
  return SQ_OK;
}

uint32_t sqi::pipeline_chunks(uint32_t n) {
  // Chunks of at least 262,144 queries: below that the launch tails cost
  // more than the copies they hide.
  if (n >= 1u << 20) return 4;
  if (n >= 1u << 19) return 2;
  return 1;
}

int32_t sqi::pipelined(sq_ctx* ctx, uint32_t n, const std::function<int32_t(uint32_t, uint32_t, cudaStream_t)>& in,
                       const std::function<int32_t(sq_ctx*, uint32_t, uint32_t)>& run,
                       const std::function<int32_t(uint32_t, uint32_t, cudaStream_t)>& out) {
  const uint32_t k = pipeline_chunks(n);
  int32_t rc;
  if (k == 1) {
    if ((rc = in(0, n, ctx->stream)) || (rc = run(ctx, 0, n)) || (rc = out(0, n, ctx->stream))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return SQ_OK;
  }
  if (!ctx->s_in) CK(cudaStreamCreateWithFlags(&ctx->s_in, cudaStreamNonBlocking));
  if (!ctx->s_out) CK(cudaStreamCreateWithFlags(&ctx->s_out, cudaStreamNonBlocking));
  sq_ctx* lane = nullptr;
  if ((rc = second_lane(ctx, &lane))) return rc;
  const uint64_t lane_launches = lane->launches;
  std::vector<cudaEvent_t> ev(2 * k + 2, nullptr);
  for (auto& e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  // The copies in and the second lane start after whatever the context's
  // stream holds (earlier calls may still be reading the scratch buffers).
  rc = SQ_OK;
  sq_ctx* failed = ctx;
  cudaError_t ce = cudaEventRecord(ev[2 * k], ctx->stream);
  if (ce == cudaSuccess) ce = cudaStreamWaitEvent(ctx->s_in, ev[2 * k], 0);
  if (ce == cudaSuccess) ce = cudaStreamWaitEvent(lane->stream, ev[2 * k], 0);
  const uint32_t step = (n + k - 1) / k;
  for (uint32_t c = 0; c < k && rc == SQ_OK && ce == cudaSuccess; ++c) {
    const uint32_t s0 = c * step, m = std::min(step, n - s0);
    sq_ctx* on = (c & 1) ? lane : ctx;
    if ((rc = in(s0, m, ctx->s_in))) break;
    if ((ce = cudaEventRecord(ev[2 * c], ctx->s_in)) != cudaSuccess) break;
    if ((ce = cudaStreamWaitEvent(on->stream, ev[2 * c], 0)) != cudaSuccess) break;
    if ((rc = run(on, s0, m))) {
      failed = on;
      break;
    }
    if ((ce = cudaEventRecord(ev[2 * c + 1], on->stream)) != cudaSuccess) break;
    if ((ce = cudaStreamWaitEvent(ctx->s_out, ev[2 * c + 1], 0)) != cudaSuccess) break;
    rc = out(s0, m, ctx->s_out);
  }
  // The context's stream takes the second lane's work back, and every stream
  // settles before the events go and before an error returns.
  if (cudaEventRecord(ev[2 * k + 1], lane->stream) == cudaSuccess) cudaStreamWaitEvent(ctx->stream, ev[2 * k + 1], 0);
  cudaStreamSynchronize(ctx->s_in);
  cudaStreamSynchronize(lane->stream);
  cudaStreamSynchronize(ctx->stream);
  const cudaError_t se = cudaStreamSynchronize(ctx->s_out);
  for (auto& e : ev) cudaEventDestroy(e);
  ctx->launches += lane->launches - lane_launches;
  if (rc) return failed == ctx ? rc : fail(ctx, rc, lane->err.c_str());
  if (ce != cudaSuccess) return cuda_fail(ctx, "chunked host-buffer call", ce);
  if (se != cudaSuccess) return cuda_fail(ctx, "chunked host-buffer call", se);
  return SQ_OK;
}

int32_t sqi::near_first_launch(sq_ctx* ctx, const sq_bvh* b, const void* fn, const void* ref_fn, QueryParams& p,
                               uint32_t stack) {
  p.window = ctx->window;
  if (!ref_fn) {
    // The kernel answers its uncertified queries again itself; only their
    // number is kept.
    CK(cudaMemsetAsync(ctx->d_replays, 0, sizeof(uint32_t), ctx->stream));
    p.replay_count = ctx->d_replays;
    p.replay_list = nullptr;
    return launch_persistent(ctx, fn, p, stack, p.n);
  }
  // The replay list holds at most every query of the batch; it grows here,
  // outside any stream capture once a batch of this size has run.
  const size_t need = size_t(std::max<uint32_t>(p.n, 1)) * sizeof(uint32_t);
  if (ctx->replay_list.cap < need) {
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->replay_list.p) CK(cudaFree(ctx->replay_list.p));
    ctx->replay_list.p = nullptr;
    ctx->replay_list.cap = 0;
    CK(cudaMalloc(&ctx->replay_list.p, need));
    ctx->replay_list.cap = need;
  }
  CK(cudaMemsetAsync(ctx->d_replays, 0, sizeof(uint32_t), ctx->stream));
  p.replay_count = ctx->d_replays;
  p.replay_list = static_cast<uint32_t*>(ctx->replay_list.p);
  p.window = ctx->window;
  int32_t rc = launch_persistent(ctx, fn, p, stack, p.n);
  if (rc) return rc;
  // A box leaf's hit is its own slab entry, so box answers are always
  // certified and nothing is ever appended: no replay launch.
  if (b->narrow == SQ_NARROW_AABB) return SQ_OK;
  // The uncertified queries again, in the reference order, unseeded.
  QueryParams r = p;
  r.replay_count = nullptr;
  r.replay_list = nullptr;
  r.seed_bucket = nullptr;
  r.q_list = static_cast<const uint32_t*>(ctx->replay_list.p);
  r.q_count = ctx->d_replays;
  return launch_persistent(ctx, ref_fn, r, b->depth, p.n);
}

// ============================================================================
// autotuner (include/sq.h)
// ============================================================================

extern "C" int32_t sq_autotune_nearest_d(sq_ctx* ctx, const sq_bvh* b, const float* d_rays, uint32_t n, float max_toi,
                                         uint32_t reps, sq_tune_result* out) {
  int32_t rc = check_scene(ctx, b);
  if (rc) return rc;
  if (!out || !d_rays || n == 0) return fail(ctx, SQ_ERR_INVALID, "autotune needs rays and a result");
  std::memset(out, 0, sizeof(*out));
  reps = std::max<uint32_t>(reps, 1);
  uint32_t* d_leaf = nullptr;
  float* d_toi = nullptr;
  if ((rc = arena_reserve(ctx, size_t(n) * 8 + 512))) return rc;
  d_leaf = static_cast<uint32_t*>(ctx->arena.p);
  d_toi = reinterpret_cast<float*>(static_cast<char*>(ctx->arena.p) + ((size_t(n) * 4 + 255) & ~size_t(255)));
  sq_hits o{};
  o.leaf = d_leaf;
  o.toi = d_toi;
  const int saved_order = ctx->order, saved_bps = ctx->blocks_per_sm, saved_layout = ctx->layout;
  // (order, layout): near-first over child-pair records, over four-wide
  // records and over quantised four-wide records (when the scene has them),
  // over child-pair records with the register-held stack top or the
  // warp-vote child order, the reference order.
  const int orders[6] = {SQ_ORDER_NEAR_FIRST, SQ_ORDER_NEAR_FIRST, SQ_ORDER_NEAR_FIRST, SQ_ORDER_NEAR_FIRST,
                         SQ_ORDER_NEAR_FIRST, SQ_ORDER_REFERENCE};
  const int layouts[6] = {SQ_LAYOUT_BINARY,        SQ_LAYOUT_WIDE,        SQ_LAYOUT_QUANT,
                          SQ_LAYOUT_BINARY_REGTOP, SQ_LAYOUT_BINARY_VOTE, SQ_LAYOUT_BINARY};
  const int bps[8] = {0, 2, 4, 6, 8, 10, 12, 16};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 0.f;
  for (int oi = 0; oi < 6 && rc == SQ_OK; ++oi) {
    if (layouts[oi] == SQ_LAYOUT_WIDE && !(b->n_wide && b->ks.ray_nearest_wide)) continue;
    if (layouts[oi] == SQ_LAYOUT_QUANT && !(b->n_wide && b->d_qnodes && b->ks.ray_nearest_quant)) continue;
    if (layouts[oi] == SQ_LAYOUT_BINARY_REGTOP && !b->ks.ray_nearest_regtop) continue;
    if (layouts[oi] == SQ_LAYOUT_BINARY_VOTE && !b->ks.ray_nearest_vote) continue;
    for (int bi = 0; bi < 8 && rc == SQ_OK; ++bi) {
      ctx->order = orders[oi];
      ctx->layout = layouts[oi];
      ctx->blocks_per_sm = bps[bi];
      // warm, then the best of `reps`
      if ((rc = nearest_core(ctx, b, false, d_rays, n, max_toi, nullptr, nullptr, o, false))) break;
      float t_best = 0.f;
      for (uint32_t r = 0; r < reps; ++r) {
        CK(cudaEventRecord(e0, ctx->stream));
        if ((rc = nearest_core(ctx, b, false, d_rays, n, max_toi, nullptr, nullptr, o, false))) break;
        CK(cudaEventRecord(e1, ctx->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (r == 0 || ms < t_best) t_best = ms;
      }
      if (rc) break;
      sq_tune_entry& e = out->entries[out->n_entries];
      e.order = orders[oi];
      e.blocks_per_sm = bps[bi];
      e.ms = t_best;
      e.layout = layouts[oi];
      if (out->n_entries == 0 || t_best < best) {
        best = t_best;
        out->best = int32_t(out->n_entries);
      }
      ++out->n_entries;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    ctx->order = saved_order;
    ctx->blocks_per_sm = saved_bps;
    ctx->layout = saved_layout;
    return rc;
  }
  ctx->order = out->entries[out->best].order;
  ctx->blocks_per_sm = out->entries[out->best].blocks_per_sm;
  ctx->layout = out->entries[out->best].layout;
  return finish(ctx);
}
