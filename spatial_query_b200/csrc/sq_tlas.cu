// C ABI of the two-level path (accel/tlas.rs): BLAS sets, Tlas upload and
// refit, Tlas queries, the mixed persistent launch, and CUDA-graph capture of
// a frame (refit + queries).
#include <cuda_runtime.h>

#include <cmath>
#include <memory>
#include <vector>

#include "sq_internal.cuh"
#include "tlas.cuh"

namespace sq {
bool tlas_kernel_set(int dim, int kind, TlasKernelSet* out);
}  // namespace sq

using namespace sq;
using namespace sqi;

struct sq_blas_set {
  int device = 0;
  uint32_t n_blas = 0;
  float4* d_nodes = nullptr;
  float4* d_prims = nullptr;
  BlasRoot* d_roots = nullptr;
  std::vector<float> h_root;  // per BLAS: min[3], max[3]
  uint32_t max_depth = 0;
  bool finite = true;  // every node bound is finite
  size_t bytes = 0;
};

struct sq_tlas {
  int device = 0, dim = 0, kind = 0;
  uint32_t n_inst = 0, n_nodes = 0, n_interior = 0, depth = 0, n_leaves = 0, stack = 1;
  uint32_t root_code = 0;
  float4* d_nodes = nullptr;
  float4* d_insts = nullptr;
  float* d_root = nullptr;
  float* d_local = nullptr;
  float* d_world = nullptr;
  uint64_t* d_layers = nullptr;
  uint32_t* d_sub = nullptr;
  RefitLeaf* d_leaves = nullptr;
  uint32_t* d_parents = nullptr;
  uint32_t* d_arrivals = nullptr;
  int* d_nonfinite = nullptr;
  float* d_stage = nullptr;  // host refit staging (rot + trans)
  const sq_blas_set* blas = nullptr;
  TlasKernelSet ks{};
  float baseline = 0.f;
  size_t bytes = 0;
  std::vector<uint32_t> h_iidx, h_child_a, h_child_b, h_count, h_inst_indices;
};

struct sq_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

// A host tree converted to child-pair records (see traverse.cuh), with node
// codes offset by node_off / prim_off so several trees can share arrays.
struct TreeConv {
  std::vector<float> records;
  std::vector<uint32_t> iidx;
  std::vector<RefitLeaf> leaves;
  std::vector<uint32_t> parents;
  uint32_t n_interior = 0, depth = 0, root_code = 0;
};

int32_t convert_tree(sq_ctx* ctx, int D, uint32_t n_nodes, const float* bounds, const uint32_t* ca,
                     const uint32_t* cb, const uint32_t* pc, uint32_t n_prims, const uint32_t* pidx,
                     uint32_t node_off, uint32_t prim_off, TreeConv& T) {
  if (n_nodes == 0) return n_prims == 0 ? SQ_OK : fail(ctx, SQ_ERR_INVALID, "leaves without a tree");
  if (!bounds || !ca || !cb || !pc || !pidx) return fail(ctx, SQ_ERR_INVALID, "null tree array");
  std::vector<uint32_t> depth(n_nodes, 1);
  for (uint32_t i = n_nodes; i-- > 0;) {
    if (pc[i] == 0) {
      if (ca[i] <= i || cb[i] <= i || ca[i] >= n_nodes || cb[i] >= n_nodes)
        return fail(ctx, SQ_ERR_INVALID, "interior node with a child out of order");
      depth[i] = 1 + std::max(depth[ca[i]], depth[cb[i]]);
    } else if (uint64_t(ca[i]) + pc[i] > n_prims) {
      return fail(ctx, SQ_ERR_INVALID, "leaf indexes past the primitives");
    }
  }
  T.depth = depth[0];
  std::vector<uint8_t> seen(n_prims, 0), covered(n_prims, 0);
  for (uint32_t k = 0; k < n_prims; ++k) {
    if (pidx[k] >= n_prims || seen[pidx[k]]) return fail(ctx, SQ_ERR_INVALID, "indices are not a permutation");
    seen[pidx[k]] = 1;
  }
  for (uint32_t i = 0; i < n_nodes; ++i) {
    if (pc[i] == 0) continue;
    for (uint32_t k = ca[i]; k < ca[i] + pc[i]; ++k) {
      if (covered[k]) return fail(ctx, SQ_ERR_INVALID, "leaf ranges overlap");
      covered[k] = 1;
    }
  }
  for (uint32_t k = 0; k < n_prims; ++k)
    if (!covered[k]) return fail(ctx, SQ_ERR_INVALID, "leaf ranges leave a primitive uncovered");
  T.iidx.assign(n_nodes, kNoHit);
  uint32_t ni = 0;
  for (uint32_t i = 0; i < n_nodes; ++i)
    if (pc[i] == 0) T.iidx[i] = ni++;
  T.n_interior = ni;
  auto code = [&](uint32_t i) { return pc[i] == 0 ? node_off + T.iidx[i] : (kLeafBit | (prim_off + ca[i])); };
  T.root_code = code(0);
  const uint32_t NV = node_vec(D);
  T.records.assign(size_t(ni) * NV * 4, 0.f);
  T.parents.assign(ni, kNoHit);
  if (pc[0] != 0) T.leaves.push_back(RefitLeaf{prim_off + ca[0], pc[0], kNoHit, 0});
  for (uint32_t i = 0; i < n_nodes; ++i) {
    if (pc[i] != 0) continue;
    const uint32_t k = T.iidx[i];
    float* r = T.records.data() + size_t(k) * NV * 4;
    const uint32_t ch[2] = {ca[i], cb[i]};
    for (int s = 0; s < 2; ++s) {
      const float* cbx = bounds + size_t(ch[s]) * 2 * D;
      for (int j = 0; j < 2 * D; ++j) r[s * 2 * D + j] = cbx[j];
      uint32_t c = code(ch[s]);
      std::memcpy(&r[4 * D + s], &c, 4);
      const uint32_t slot = ((node_off + k) << 1) | uint32_t(s);
      if (pc[ch[s]] == 0) T.parents[T.iidx[ch[s]]] = slot;
      else T.leaves.push_back(RefitLeaf{prim_off + ca[ch[s]], pc[ch[s]], slot, 0});
    }
  }
  return SQ_OK;
}

// Isometry::transform_aabb (maths/isometry.rs:84-97), host side.
void host_transform_aabb(int D, const float* R, const float* t, const float* llo, const float* lhi, float* wlo,
                         float* whi) {
  float c[8], h[8];
  for (int i = 0; i < D; ++i) {
    c[i] = (llo[i] + lhi[i]) * 0.5f;
    h[i] = (lhi[i] - llo[i]) * 0.5f;
  }
  for (int i = 0; i < D; ++i) {
    float acc = 0.f;
    for (int j = 0; j < D; ++j) acc += R[i * D + j] * c[j];
    const float wc = acc + t[i];
    float ah = 0.f;
    for (int j = 0; j < D; ++j) ah += std::fabs(R[i * D + j]) * h[j];
    wlo[i] = wc - ah;
    whi[i] = wc + ah;
  }
}

// The instance's local AABB: s * mesh AABB, [-h, h] or [-r, r].
int32_t local_aabb(int D, int kind, const float* param, uint32_t i, const uint32_t* blas_id, const sq_blas_set* blas,
                   float* lo, float* hi) {
  if (kind == SQ_INSTANCE_MESH) {
    if (!blas || !blas_id || blas_id[i] >= blas->n_blas) return SQ_ERR_INVALID;
    const float s = param[i];
    const float* m = blas->h_root.data() + size_t(blas_id[i]) * 6;
    for (int k = 0; k < 3; ++k) {
      lo[k] = m[k] * s;
      hi[k] = m[3 + k] * s;
    }
  } else if (kind == SQ_INSTANCE_BOX) {
    for (int k = 0; k < D; ++k) {
      lo[k] = param[size_t(i) * D + k] * -1.0f;
      hi[k] = param[size_t(i) * D + k];
    }
  } else {
    for (int k = 0; k < D; ++k) {
      lo[k] = param[i] * -1.0f;
      hi[k] = param[i];
    }
  }
  return SQ_OK;
}

float half_surface_sum(int D, uint32_t n_nodes, const uint32_t* pc, const float* bounds) {
  // tree.rs:104-110 with Aabb::half_surface (aabb.rs:84-97), in node order.
  float sum = 0.f;
  for (uint32_t i = 0; i < n_nodes; ++i) {
    if (pc[i] != 0) continue;
    const float* b = bounds + size_t(i) * 2 * D;
    float hs = 0.f;
    for (int a = 0; a < D; ++a) {
      float prod = 1.f;
      for (int j = 0; j < D; ++j)
        if (j != a) prod *= (b[D + j] - b[j]);
      hs += prod;
    }
    sum += hs;
  }
  return sum;
}

int32_t check_tlas(sq_ctx* ctx, const sq_tlas* t) {
  if (!ctx) return SQ_ERR_INVALID;
  if (!t) return fail(ctx, SQ_ERR_INVALID, "null tlas");
  if (t->device != ctx->device) return fail(ctx, SQ_ERR_INVALID, "tlas and context are on different devices");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, "cudaSetDevice", e);
  return SQ_OK;
}

void tlas_base(const sq_tlas* t, const sq_filter* f, TlasParams& p) {
  std::memset(&p, 0, sizeof(p));
  p.nodes = t->d_nodes;
  p.insts = t->d_insts;
  p.root_box = t->d_root;
  p.nonfinite = t->d_nonfinite;
  p.local_aabbs = t->d_local;
  p.world_aabbs = t->d_world;
  p.layers = t->d_layers;
  p.sub = t->d_sub;
  if (t->blas) {
    p.bnodes = t->blas->d_nodes;
    p.bprims = t->blas->d_prims;
    p.broots = t->blas->d_roots;
    p.blas_finite = t->blas->finite ? 1 : 0;
  }
  p.root_code = t->root_code;
  p.mask = f ? f->layer_mask : ~0ull;
  p.exclude = f ? f->exclude : -1;
}

int32_t tlas_run(sq_ctx* ctx, const sq_tlas* t, TlasParams& p, bool stats) {
  const uint64_t n = uint64_t(p.n_ray) + p.n_cast + p.n_region;
  if (n == 0 || t->n_nodes == 0) return SQ_OK;
  const int st = stats ? 1 : 0;
  if (stats) p.stats = ctx->d_stats;
  if (ctx->order == SQ_ORDER_REFERENCE) return launch_persistent(ctx, t->ks.query[1][st], p, t->stack, n);
  // Near-first; flagged queries are answered again in reference order in-kernel.
  CK(cudaMemsetAsync(ctx->d_replays, 0, sizeof(uint32_t), ctx->stream));
  p.replay_count = ctx->d_replays;
  p.window = ctx->window;
  return launch_persistent(ctx, t->ks.query[0][st], p, t->stack, n);
}

// Writes "no hit" into nearest outputs and zero counts (empty Tlas).
int32_t tlas_empty_outputs(sq_ctx* ctx, const sq_tlas* t, uint32_t n, const sq_hits* h, const sq_hit_lists* l) {
  if (h) {
    CK(cudaMemsetAsync(h->leaf, 0xFF, size_t(n) * 4, ctx->stream));
    if (h->toi) CK(cudaMemsetAsync(h->toi, 0, size_t(n) * 4, ctx->stream));
    if (h->sub_object) CK(cudaMemsetAsync(h->sub_object, 0xFF, size_t(n) * 4, ctx->stream));
    if (h->normal) CK(cudaMemsetAsync(h->normal, 0, size_t(n) * 4 * t->dim, ctx->stream));
    if (h->point) CK(cudaMemsetAsync(h->point, 0, size_t(n) * 4 * t->dim, ctx->stream));
  }
  if (l) CK(cudaMemsetAsync(l->count, 0, size_t(n) * 4, ctx->stream));
  return SQ_OK;
}

}  // namespace

// ============================================================================
// BLAS sets
// ============================================================================

extern "C" int32_t sq_blas_set_upload(sq_ctx* ctx, uint32_t n_blas, const uint32_t* node_offsets,
                                      const float* node_bounds, const uint32_t* child_a, const uint32_t* child_b,
                                      const uint32_t* prim_count, const uint32_t* tri_offsets,
                                      const uint32_t* prim_indices, const float* tris, sq_blas_set** out) {
  if (!ctx || !out || (n_blas && (!node_offsets || !tri_offsets))) return SQ_ERR_INVALID;
  *out = nullptr;
  CK(cudaSetDevice(ctx->device));
  auto B = std::make_unique<sq_blas_set>();
  B->device = ctx->device;
  B->n_blas = n_blas;
  std::vector<float> records, prims;
  std::vector<BlasRoot> roots(std::max<uint32_t>(n_blas, 1));
  B->h_root.assign(size_t(std::max<uint32_t>(n_blas, 1)) * 6, 0.f);
  uint32_t node_off = 0;
  const uint32_t total_tris = n_blas ? tri_offsets[n_blas] : 0;
  if (total_tris >= kLeafBit) return fail(ctx, SQ_ERR_INVALID, "too many triangles");
  prims.assign(size_t(total_tris) * 12, 0.f);
  for (uint32_t b = 0; b < n_blas; ++b) {
    const uint32_t n0 = node_offsets[b], n1 = node_offsets[b + 1];
    const uint32_t t0 = tri_offsets[b], t1 = tri_offsets[b + 1];
    if (n1 < n0 || t1 < t0) return fail(ctx, SQ_ERR_INVALID, "offsets decrease");
    TreeConv T;
    int32_t rc = convert_tree(ctx, 3, n1 - n0, node_bounds + size_t(n0) * 6, child_a + n0, child_b + n0,
                              prim_count + n0, t1 - t0, prim_indices + t0, node_off, t0, T);
    if (rc) return rc;
    B->max_depth = std::max(B->max_depth, T.depth);
    for (size_t k = size_t(n0) * 6; k < size_t(n1) * 6; ++k)
      if (!std::isfinite(node_bounds[k])) B->finite = false;
    records.insert(records.end(), T.records.begin(), T.records.end());
    node_off += T.n_interior;
    BlasRoot R{};
    if (n1 > n0) {
      R.code = T.root_code;
      for (int k = 0; k < 3; ++k) {
        R.lo[k] = node_bounds[size_t(n0) * 6 + k];
        R.hi[k] = node_bounds[size_t(n0) * 6 + 3 + k];
      }
    } else {
      for (int k = 0; k < 3; ++k) {
        R.lo[k] = INFINITY;
        R.hi[k] = -INFINITY;
      }
    }
    roots[b] = R;
    for (int k = 0; k < 3; ++k) {
      B->h_root[size_t(b) * 6 + k] = R.lo[k];
      B->h_root[size_t(b) * 6 + 3 + k] = R.hi[k];
    }
    for (const RefitLeaf& L : T.leaves) {
      for (uint32_t j = 0; j < L.count; ++j) {
        const uint32_t pos = L.first + j;  // global
        const uint32_t id = prim_indices[pos];  // local to the mesh
        float* r = prims.data() + size_t(pos) * 12;
        std::memcpy(r, tris + (size_t(t0) + id) * 9, 36);
        uint32_t w = id | (j + 1 == L.count ? kLeafBit : 0u);
        std::memcpy(&r[9], &w, 4);
      }
    }
  }
  if (B->max_depth > uint32_t(kMaxStack)) return fail(ctx, SQ_ERR_DEPTH, "a mesh tree is deeper than the stack");
  auto up = [&](void** dst, const void* src, size_t bytes) -> int32_t {
    CK(cudaMalloc(dst, std::max<size_t>(bytes, 16)));
    if (src && bytes) CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    B->bytes += bytes;
    return SQ_OK;
  };
  int32_t rc;
  if ((rc = up((void**)&B->d_nodes, records.data(), records.size() * 4)) ||
      (rc = up((void**)&B->d_prims, prims.data(), prims.size() * 4)) ||
      (rc = up((void**)&B->d_roots, roots.data(), roots.size() * sizeof(BlasRoot)))) {
    sq_blas_set_destroy(B.release());
    return rc;
  }
  *out = B.release();
  return SQ_OK;
}

extern "C" int32_t sq_blas_set_destroy(sq_blas_set* b) {
  if (!b) return SQ_OK;
  cudaSetDevice(b->device);
  if (b->d_nodes) cudaFree(b->d_nodes);
  if (b->d_prims) cudaFree(b->d_prims);
  if (b->d_roots) cudaFree(b->d_roots);
  delete b;
  return SQ_OK;
}

extern "C" int32_t sq_instance_world_aabbs(int32_t dim, int32_t kind, uint32_t n, const float* rot,
                                           const float* trans, const float* param, const uint32_t* blas_id,
                                           const sq_blas_set* blas, float* out) {
  if (dim < 1 || dim > 8 || (n && (!rot || !trans || !param || !out))) return SQ_ERR_INVALID;
  if (kind == SQ_INSTANCE_MESH && dim != 3) return SQ_ERR_INVALID;
  for (uint32_t i = 0; i < n; ++i) {
    float lo[8], hi[8];
    if (local_aabb(dim, kind, param, i, blas_id, blas, lo, hi)) return SQ_ERR_INVALID;
    host_transform_aabb(dim, rot + size_t(i) * dim * dim, trans + size_t(i) * dim, lo, hi, out + size_t(i) * 2 * dim,
                        out + size_t(i) * 2 * dim + dim);
  }
  return SQ_OK;
}

// ============================================================================
// Tlas upload / refit
// ============================================================================

extern "C" int32_t sq_tlas_upload(sq_ctx* ctx, int32_t dim, int32_t kind, uint32_t n_inst, const float* rot,
                                  const float* trans, const float* param, const uint32_t* blas_id,
                                  const sq_blas_set* blas, uint32_t n_nodes, const float* node_bounds,
                                  const uint32_t* child_a, const uint32_t* child_b, const uint32_t* prim_count,
                                  const uint32_t* inst_indices, const uint64_t* layers, const uint32_t* sub_objects,
                                  sq_tlas** out) {
  if (!ctx || !out) return SQ_ERR_INVALID;
  *out = nullptr;
  TlasKernelSet ks;
  if (!tlas_kernel_set(dim, kind, &ks))
    return fail(ctx, SQ_ERR_UNSUPPORTED, "no two-level kernels for this dimension / instance kind");
  if (kind == SQ_INSTANCE_MESH && (!blas || !blas_id || blas->device != ctx->device))
    return fail(ctx, SQ_ERR_INVALID, "mesh instances need a BLAS set on the same device");
  if (n_inst && (!rot || !trans || !param)) return fail(ctx, SQ_ERR_INVALID, "null instance array");
  if (n_inst >= kLeafBit) return fail(ctx, SQ_ERR_INVALID, "too many instances");
  CK(cudaSetDevice(ctx->device));
  auto T = std::make_unique<sq_tlas>();
  T->device = ctx->device;
  T->dim = dim;
  T->kind = kind;
  T->n_inst = n_inst;
  T->n_nodes = n_nodes;
  T->blas = kind == SQ_INSTANCE_MESH ? blas : nullptr;
  T->ks = ks;
  const int D = dim;
  TreeConv C;
  int32_t rc = convert_tree(ctx, D, n_nodes, node_bounds, child_a, child_b, prim_count, n_inst, inst_indices, 0, 0, C);
  if (rc) return rc;
  if (n_nodes == 0) {
    *out = T.release();
    return SQ_OK;
  }
  if (kind == SQ_INSTANCE_MESH)
    for (uint32_t i = 0; i < n_inst; ++i)
      if (blas_id[i] >= blas->n_blas) return fail(ctx, SQ_ERR_INVALID, "blas id out of range");
  T->depth = C.depth;
  T->n_interior = C.n_interior;
  T->n_leaves = uint32_t(C.leaves.size());
  T->root_code = C.root_code;
  T->stack = C.depth + (kind == SQ_INSTANCE_MESH ? blas->max_depth : 0);
  if (T->stack > uint32_t(kMaxStack)) return fail(ctx, SQ_ERR_DEPTH, "two-level depth exceeds the stack");
  T->h_iidx = C.iidx;
  T->h_child_a.assign(child_a, child_a + n_nodes);
  T->h_child_b.assign(child_b, child_b + n_nodes);
  T->h_count.assign(prim_count, prim_count + n_nodes);
  T->h_inst_indices.assign(inst_indices, inst_indices + n_inst);
  T->baseline = half_surface_sum(D, n_nodes, prim_count, node_bounds);

  const int P = kind == SQ_INSTANCE_BOX ? D : 1;
  const int words = D * D + D + P + 2;
  const int vec = (words + 3) / 4;
  std::vector<float> insts(size_t(n_inst) * vec * 4, 0.f);
  std::vector<float> local(size_t(n_inst) * 2 * D), world(size_t(n_inst) * 2 * D);
  for (const RefitLeaf& L : C.leaves) {
    for (uint32_t j = 0; j < L.count; ++j) {
      const uint32_t pos = L.first + j;
      const uint32_t id = inst_indices[pos];
      float* r = insts.data() + size_t(pos) * vec * 4;
      std::memcpy(r, rot + size_t(id) * D * D, sizeof(float) * D * D);
      std::memcpy(r + D * D, trans + size_t(id) * D, sizeof(float) * D);
      std::memcpy(r + D * D + D, param + size_t(id) * P, sizeof(float) * P);
      uint32_t bw = kind == SQ_INSTANCE_MESH ? blas_id[id] : 0u;
      std::memcpy(r + D * D + D + P, &bw, 4);
      uint32_t w = id | (j + 1 == L.count ? kLeafBit : 0u);
      std::memcpy(r + D * D + D + P + 1, &w, 4);
      float* lo = local.data() + size_t(pos) * 2 * D;
      if (local_aabb(D, kind, param, id, blas_id, blas, lo, lo + D))
        return fail(ctx, SQ_ERR_INVALID, "bad instance");
      host_transform_aabb(D, rot + size_t(id) * D * D, trans + size_t(id) * D, lo, lo + D,
                          world.data() + size_t(pos) * 2 * D, world.data() + size_t(pos) * 2 * D + D);
    }
  }
  int nonfinite = 0;
  for (size_t k = 0; k < size_t(n_nodes) * 2 * D; ++k)
    if (!std::isfinite(node_bounds[k])) nonfinite = 1;

  auto up = [&](void** dst, const void* src, size_t bytes) -> int32_t {
    CK(cudaMalloc(dst, std::max<size_t>(bytes, 16)));
    if (src && bytes) CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    T->bytes += bytes;
    return SQ_OK;
  };
  std::vector<uint32_t> parents = C.parents;
  if (parents.empty()) parents.push_back(kNoHit);
  if ((rc = up((void**)&T->d_nodes, C.records.data(), C.records.size() * 4)) ||
      (rc = up((void**)&T->d_insts, insts.data(), insts.size() * 4)) ||
      (rc = up((void**)&T->d_root, node_bounds, size_t(2) * D * 4)) ||
      (rc = up((void**)&T->d_local, local.data(), local.size() * 4)) ||
      (rc = up((void**)&T->d_world, world.data(), world.size() * 4)) ||
      (rc = up((void**)&T->d_leaves, C.leaves.data(), C.leaves.size() * sizeof(RefitLeaf))) ||
      (rc = up((void**)&T->d_parents, parents.data(), parents.size() * 4)) ||
      (rc = up((void**)&T->d_arrivals, nullptr, parents.size() * 4)) ||
      (rc = up((void**)&T->d_nonfinite, &nonfinite, sizeof(int))) ||
      (layers && (rc = up((void**)&T->d_layers, layers, size_t(n_inst) * 8))) ||
      (sub_objects && (rc = up((void**)&T->d_sub, sub_objects, size_t(n_inst) * 4)))) {
    sq_tlas_destroy(T.release());
    return rc;
  }
  *out = T.release();
  return SQ_OK;
}

extern "C" int32_t sq_tlas_destroy(sq_tlas* t) {
  if (!t) return SQ_OK;
  cudaSetDevice(t->device);
  void* ptrs[] = {t->d_nodes, t->d_insts, t->d_root, t->d_local, t->d_world, t->d_layers, t->d_sub,
                  t->d_leaves, t->d_parents, t->d_arrivals, t->d_nonfinite, t->d_stage};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete t;
  return SQ_OK;
}

extern "C" int32_t sq_tlas_refit_d(sq_ctx* ctx, sq_tlas* t, const float* d_rot, const float* d_trans,
                                   const float* d_delta, const float* d_param) {
  int32_t rc = check_tlas(ctx, t);
  if (rc) return rc;
  if (t->n_nodes == 0) return SQ_OK;
  CK(cudaMemsetAsync(t->d_arrivals, 0, size_t(std::max<uint32_t>(t->n_interior, 1)) * 4, ctx->stream));
  CK(cudaMemsetAsync(t->d_nonfinite, 0, sizeof(int), ctx->stream));
  TlasRefitParams p;
  p.nonfinite = t->d_nonfinite;
  p.nodes = t->d_nodes;
  p.insts = t->d_insts;
  p.root_box = t->d_root;
  p.local_aabbs = t->d_local;
  p.world_aabbs = t->d_world;
  p.new_rot = d_rot;
  p.new_trans = d_trans;
  p.delta = d_delta;
  p.new_param = d_param;
  p.local_aabbs_w = t->d_local;
  p.broots = t->blas ? t->blas->d_roots : nullptr;
  p.leaves = t->d_leaves;
  p.parents = t->d_parents;
  p.arrivals = t->d_arrivals;
  p.n_leaves = t->n_leaves;
  void* args[] = {&p};
  CK(cudaLaunchKernel(t->ks.refit, dim3((t->n_leaves + 255) / 256), dim3(256), args, 0, ctx->stream));
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, "tlas refit", e);
  return SQ_OK;
}

extern "C" int32_t sq_tlas_refit(sq_ctx* ctx, sq_tlas* t, const float* rot, const float* trans,
                                 const float* param) {
  int32_t rc = check_tlas(ctx, t);
  if (rc) return rc;
  if (t->n_nodes == 0) return SQ_OK;
  if (!trans) return fail(ctx, SQ_ERR_INVALID, "null translations");
  const int D = t->dim;
  const int P = t->kind == SQ_INSTANCE_BOX ? D : 1;
  const size_t rb = size_t(t->n_inst) * D * D * 4, tb = size_t(t->n_inst) * D * 4, pb = size_t(t->n_inst) * P * 4;
  if (!t->d_stage) CK(cudaMalloc(&t->d_stage, rb + tb + pb));
  float* d_rot = t->d_stage;
  float* d_trans = (float*)((char*)t->d_stage + rb);
  float* d_param = (float*)((char*)t->d_stage + rb + tb);
  if (rot) CK(cudaMemcpyAsync(d_rot, rot, rb, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_trans, trans, tb, cudaMemcpyHostToDevice, ctx->stream));
  if (param) CK(cudaMemcpyAsync(d_param, param, pb, cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = sq_tlas_refit_d(ctx, t, rot ? d_rot : nullptr, d_trans, nullptr, param ? d_param : nullptr))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

extern "C" int32_t sq_tlas_read_bounds(sq_ctx* ctx, const sq_tlas* t, float* node_bounds, float* world_aabbs) {
  int32_t rc = check_tlas(ctx, t);
  if (rc) return rc;
  if (t->n_nodes == 0) return SQ_OK;
  const int D = t->dim;
  const uint32_t NV = node_vec(D);
  std::vector<float> nodes(size_t(std::max<uint32_t>(t->n_interior, 1)) * NV * 4), root(2 * D),
      world(size_t(t->n_inst) * 2 * D);
  CK(cudaMemcpyAsync(nodes.data(), t->d_nodes, size_t(t->n_interior) * NV * 16, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(root.data(), t->d_root, root.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(world.data(), t->d_world, world.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (node_bounds) {
    std::memcpy(node_bounds, root.data(), root.size() * 4);
    for (uint32_t i = 0; i < t->n_nodes; ++i) {
      if (t->h_count[i] != 0) continue;
      const float* r = nodes.data() + size_t(t->h_iidx[i]) * NV * 4;
      std::memcpy(node_bounds + size_t(t->h_child_a[i]) * 2 * D, r, 2 * D * 4);
      std::memcpy(node_bounds + size_t(t->h_child_b[i]) * 2 * D, r + 2 * D, 2 * D * 4);
    }
  }
  if (world_aabbs)
    for (uint32_t pos = 0; pos < t->n_inst; ++pos)
      std::memcpy(world_aabbs + size_t(t->h_inst_indices[pos]) * 2 * D, world.data() + size_t(pos) * 2 * D, 2 * D * 4);
  return SQ_OK;
}

extern "C" int32_t sq_tlas_needs_rebuild(sq_ctx* ctx, const sq_tlas* t, float factor, int32_t* out) {
  int32_t rc = check_tlas(ctx, t);
  if (rc) return rc;
  if (!out) return fail(ctx, SQ_ERR_INVALID, "null output");
  *out = 0;
  if (t->n_nodes == 0) return SQ_OK;
  std::vector<float> b(size_t(t->n_nodes) * 2 * t->dim);
  if ((rc = sq_tlas_read_bounds(ctx, t, b.data(), nullptr))) return rc;
  const float now = half_surface_sum(t->dim, t->n_nodes, t->h_count.data(), b.data());
  *out = (t->baseline > 0.f && now > factor * t->baseline) ? 1 : 0;  // tlas.rs:58-60
  return SQ_OK;
}

// ============================================================================
// Tlas queries
// ============================================================================

extern "C" int32_t sq_tlas_mixed_d(sq_ctx* ctx, const sq_tlas* t, const sq_mixed_batch* m, const sq_filter* f) {
  int32_t rc = check_tlas(ctx, t);
  if (rc) return rc;
  if (!m) return fail(ctx, SQ_ERR_INVALID, "null batch");
  if ((m->n_rays && (!m->rays || !m->ray_hits.leaf)) || (m->n_casts && (!m->casts || !m->cast_hits.leaf)) ||
      (m->n_regions && (!m->regions || !m->region_count || (m->region_k && !m->region_leaves))))
    return fail(ctx, SQ_ERR_INVALID, "null batch array");
  if (t->n_nodes == 0) {
    if (m->n_rays && (rc = tlas_empty_outputs(ctx, t, m->n_rays, &m->ray_hits, nullptr))) return rc;
    if (m->n_casts && (rc = tlas_empty_outputs(ctx, t, m->n_casts, &m->cast_hits, nullptr))) return rc;
    if (m->n_regions) CK(cudaMemsetAsync(m->region_count, 0, size_t(m->n_regions) * 4, ctx->stream));
    return SQ_OK;
  }
  TlasParams p;
  tlas_base(t, f, p);
  p.n_ray = m->n_rays;
  p.n_cast = m->n_casts;
  p.n_region = m->n_regions;
  p.ray_kind = kTRayNearest;
  p.cast_kind = kTCastNearest;
  p.region_kind = kTOverlapList;
  p.rays = m->rays;
  p.ray_mt = m->ray_max_toi_per_query;
  p.ray_max_toi = m->ray_max_toi;
  p.casts = m->casts;
  p.cast_mt = m->cast_max_toi_per_query;
  p.cast_max_toi = m->cast_max_toi;
  p.regions = m->regions;
  p.r_leaf = m->ray_hits.leaf;
  p.r_toi = m->ray_hits.toi;
  p.r_sub = m->ray_hits.sub_object;
  p.r_normal = m->ray_hits.normal;
  p.r_point = m->ray_hits.point;
  p.c_leaf = m->cast_hits.leaf;
  p.c_toi = m->cast_hits.toi;
  p.c_sub = m->cast_hits.sub_object;
  p.c_normal = m->cast_hits.normal;
  p.c_point = m->cast_hits.point;
  p.o_count = m->region_count;
  p.o_leaves = m->region_leaves;
  p.o_k = m->region_k;
  if ((rc = tlas_run(ctx, t, p, false))) return rc;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, "tlas mixed launch", e);
  return SQ_OK;
}

namespace {

// Host-buffer wrapper for one query kind of the Tlas (copy in, run, copy out).
int32_t tlas_host(sq_ctx* ctx, const sq_tlas* t, int kind, const float* q, uint32_t n, float max_toi,
                  const float* mt, const sq_filter* f, const sq_hits* h, const sq_hit_lists* l, sq_query_stats* st) {
  int32_t rc = check_tlas(ctx, t);
  if (rc) return rc;
  const bool cast = kind == kTCastNearest || kind == kTCastAll;
  const bool nearest = kind == kTRayNearest || kind == kTCastNearest;
  if ((nearest && (!h || !h->leaf)) || (!nearest && (!l || !l->count || (n && l->k && (!l->leaf || !l->toi)))) ||
      (n && !q))
    return fail(ctx, SQ_ERR_INVALID, "null argument");
  if (st) *st = sq_query_stats{0, 0, 0, 0};
  if (n == 0) return SQ_OK;
  const int D = t->dim;
  const size_t qb = size_t(n) * (cast ? 4 : 2) * D * 4;
  const size_t nk = nearest ? 0 : size_t(n) * l->k;
  Carve cv;
  size_t o_q = cv.take(qb), o_mt = mt ? cv.take(size_t(n) * 4) : 0;
  size_t o_leaf = cv.take(nearest ? size_t(n) * 4 : nk * 4), o_toi = cv.take(nearest ? size_t(n) * 4 : nk * 4);
  size_t o_sub = cv.take(nearest ? size_t(n) * 4 : nk * 4);
  size_t o_nrm = cv.take(nearest ? size_t(n) * D * 4 : nk * D * 4);
  size_t o_pt = cv.take(nearest ? size_t(n) * D * 4 : 0);
  size_t o_cnt = cv.take(size_t(n) * 4);
  if ((rc = arena_reserve(ctx, cv.off))) return rc;
  char* base = (char*)ctx->arena.p;
  CK(cudaMemcpyAsync(base + o_q, q, qb, cudaMemcpyHostToDevice, ctx->stream));
  if (mt) CK(cudaMemcpyAsync(base + o_mt, mt, size_t(n) * 4, cudaMemcpyHostToDevice, ctx->stream));
  TlasParams p;
  tlas_base(t, f, p);
  uint32_t* dl = (uint32_t*)(base + o_leaf);
  float* dt = (float*)(base + o_toi);
  uint32_t* ds = (uint32_t*)(base + o_sub);
  float* dn = (float*)(base + o_nrm);
  float* dp = (float*)(base + o_pt);
  uint32_t* dc = (uint32_t*)(base + o_cnt);
  if (!nearest) {
    CK(cudaMemsetAsync(dl, 0xFF, nk * 4, ctx->stream));
    CK(cudaMemsetAsync(dt, 0, nk * 4, ctx->stream));
    CK(cudaMemsetAsync(ds, 0xFF, nk * 4, ctx->stream));
    CK(cudaMemsetAsync(dn, 0, nk * D * 4, ctx->stream));
  }
  if (cast) {
    p.n_cast = n;
    p.cast_kind = kind;
    p.casts = (const float*)(base + o_q);
    p.cast_mt = mt ? (const float*)(base + o_mt) : nullptr;
    p.cast_max_toi = max_toi;
    p.c_leaf = dl; p.c_toi = dt; p.c_sub = ds; p.c_normal = dn; p.c_point = dp; p.c_count = dc;
    p.c_k = nearest ? 0 : l->k;
  } else {
    p.n_ray = n;
    p.ray_kind = kind;
    p.rays = (const float*)(base + o_q);
    p.ray_mt = mt ? (const float*)(base + o_mt) : nullptr;
    p.ray_max_toi = max_toi;
    p.r_leaf = dl; p.r_toi = dt; p.r_sub = ds; p.r_normal = dn; p.r_point = dp; p.r_count = dc;
    p.r_k = nearest ? 0 : l->k;
  }
  if (t->n_nodes == 0) {
    if (nearest) {
      sq_hits e{dl, dt, ds, dn, dp};
      if ((rc = tlas_empty_outputs(ctx, t, n, &e, nullptr))) return rc;
    } else {
      CK(cudaMemsetAsync(dc, 0, size_t(n) * 4, ctx->stream));
    }
  } else {
    if (st) CK(cudaMemsetAsync(ctx->d_stats, 0, 32, ctx->stream));
    if ((rc = tlas_run(ctx, t, p, st != nullptr && !cast))) return rc;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, "tlas launch", e);
  }
  auto d2h = [&](void* dst, const void* src, size_t bytes) -> int32_t {
    if (dst && bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return SQ_OK;
  };
  if (nearest) {
    if ((rc = d2h(h->leaf, dl, size_t(n) * 4)) || (rc = d2h(h->toi, dt, size_t(n) * 4)) ||
        (rc = d2h(h->sub_object, ds, size_t(n) * 4)) || (rc = d2h(h->normal, dn, size_t(n) * D * 4)) ||
        (rc = d2h(h->point, dp, size_t(n) * D * 4)))
      return rc;
  } else {
    if ((rc = d2h(l->count, dc, size_t(n) * 4)) || (rc = d2h(l->leaf, dl, nk * 4)) || (rc = d2h(l->toi, dt, nk * 4)) ||
        (rc = d2h(l->sub_object, ds, nk * 4)) || (rc = d2h(l->normal, dn, nk * D * 4)))
      return rc;
  }
  unsigned long long hs[4] = {0, 0, 0, 0};
  if (st && t->n_nodes) CK(cudaMemcpyAsync(hs, ctx->d_stats, 32, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (st) *st = sq_query_stats{hs[0], hs[1], hs[2], hs[3]};
  return SQ_OK;
}

}  // namespace

extern "C" int32_t sq_tlas_raycast_nearest(sq_ctx* ctx, const sq_tlas* t, const float* rays, uint32_t n,
                                           float max_toi, const float* mt, const sq_filter* f, const sq_hits* out,
                                           sq_query_stats* st) {
  return tlas_host(ctx, t, kTRayNearest, rays, n, max_toi, mt, f, out, nullptr, st);
}

extern "C" int32_t sq_tlas_raycast_all(sq_ctx* ctx, const sq_tlas* t, const float* rays, uint32_t n, float max_toi,
                                       const float* mt, const sq_filter* f, const sq_hit_lists* out) {
  return tlas_host(ctx, t, kTRayAll, rays, n, max_toi, mt, f, nullptr, out, nullptr);
}

extern "C" int32_t sq_tlas_raycast_crossings(sq_ctx* ctx, const sq_tlas* t, const float* rays, uint32_t n,
                                             float max_toi, const float* mt, const sq_filter* f,
                                             const sq_hit_lists* out) {
  return tlas_host(ctx, t, kTRayCross, rays, n, max_toi, mt, f, nullptr, out, nullptr);
}

extern "C" int32_t sq_tlas_shapecast_nearest(sq_ctx* ctx, const sq_tlas* t, const float* casts, uint32_t n,
                                             float max_toi, const float* mt, const sq_filter* f, const sq_hits* out) {
  return tlas_host(ctx, t, kTCastNearest, casts, n, max_toi, mt, f, out, nullptr, nullptr);
}

extern "C" int32_t sq_tlas_shapecast_all(sq_ctx* ctx, const sq_tlas* t, const float* casts, uint32_t n,
                                         float max_toi, const float* mt, const sq_filter* f, const sq_hit_lists* out) {
  return tlas_host(ctx, t, kTCastAll, casts, n, max_toi, mt, f, nullptr, out, nullptr);
}

extern "C" int32_t sq_tlas_overlap(sq_ctx* ctx, const sq_tlas* t, const float* regions, uint32_t n,
                                   const sq_filter* f, uint64_t* offsets, uint32_t* leaves, uint64_t cap,
                                   uint64_t* total) {
  int32_t rc = check_tlas(ctx, t);
  if (rc) return rc;
  if (!offsets || (n && !regions)) return fail(ctx, SQ_ERR_INVALID, "null argument");
  const int D = t->dim;
  Carve cv;
  size_t o_r = cv.take(size_t(n) * 2 * D * 4), o_cnt = cv.take(size_t(n) * 4),
         o_lv = cv.take(std::max<uint64_t>(cap, 1) * 4), o_off = cv.take((size_t(n) + 1) * 8);
  if ((rc = arena_reserve(ctx, cv.off))) return rc;
  char* base = (char*)ctx->arena.p;
  if (n) CK(cudaMemcpyAsync(base + o_r, regions, size_t(n) * 2 * D * 4, cudaMemcpyHostToDevice, ctx->stream));
  uint32_t* dc = (uint32_t*)(base + o_cnt);
  CK(cudaMemsetAsync(dc, 0, size_t(n) * 4 + 4, ctx->stream));
  TlasParams p;
  tlas_base(t, f, p);
  p.n_region = n;
  p.region_kind = kTOverlapCount;
  p.regions = (const float*)(base + o_r);
  p.o_count = dc;
  if ((rc = tlas_run(ctx, t, p, false))) return rc;
  std::vector<uint32_t> counts(n);
  if (n) CK(cudaMemcpyAsync(counts.data(), dc, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  offsets[0] = 0;
  for (uint32_t i = 0; i < n; ++i) offsets[i + 1] = offsets[i] + counts[i];
  const uint64_t tot = offsets[n];
  if (total) *total = tot;
  if (tot > cap) return fail(ctx, SQ_ERR_CAPACITY, "overlap results exceed leaf_capacity");
  if (tot) {
    CK(cudaMemcpyAsync(base + o_off, offsets, (size_t(n) + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    TlasParams q;
    tlas_base(t, f, q);
    q.n_region = n;
    q.region_kind = kTOverlapFill;
    q.regions = (const float*)(base + o_r);
    q.o_offsets = (const unsigned long long*)(base + o_off);
    q.o_leaves = (uint32_t*)(base + o_lv);
    if ((rc = tlas_run(ctx, t, q, false))) return rc;
    if ((rc = sort_csr_segments(ctx, (uint32_t*)(base + o_lv), tot, (const uint64_t*)(base + o_off), n))) return rc;
    CK(cudaMemcpyAsync(leaves, base + o_lv, tot * 4, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, "tlas overlap", e);
  return SQ_OK;
}

// ============================================================================
// CUDA graphs: capture the calls made on the context's stream between begin
// and end (device-pointer calls only: host-buffer calls synchronise), then
// replay them with one launch.
// ============================================================================

extern "C" int32_t sq_graph_begin(sq_ctx* ctx) {
  if (!ctx) return SQ_ERR_INVALID;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  return SQ_OK;
}

extern "C" int32_t sq_graph_end(sq_ctx* ctx, sq_graph** out) {
  if (!ctx || !out) return SQ_ERR_INVALID;
  *out = nullptr;
  auto g = std::make_unique<sq_graph>();
  CK(cudaStreamEndCapture(ctx->stream, &g->graph));
  cudaError_t e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g->graph);
    return cuda_fail(ctx, "cudaGraphInstantiate", e);
  }
  *out = g.release();
  return SQ_OK;
}

extern "C" int32_t sq_graph_launch(sq_ctx* ctx, const sq_graph* g) {
  if (!ctx || !g) return SQ_ERR_INVALID;
  CK(cudaGraphLaunch(g->exec, ctx->stream));
  return SQ_OK;
}

extern "C" int32_t sq_graph_destroy(sq_graph* g) {
  if (!g) return SQ_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return SQ_OK;
}
