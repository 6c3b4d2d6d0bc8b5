// Internal declarations shared by the C ABI translation units: the context
// object and the launch / staging helpers.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <functional>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/sq.h"
#include "traverse.cuh"

namespace sq {
bool kernel_set_d2(int narrow, KernelSet* out);
bool kernel_set_d3(int narrow, KernelSet* out);
bool kernel_set_d4(int narrow, KernelSet* out);
bool kernel_set_d6(int narrow, KernelSet* out);
}  // namespace sq


namespace sqi {

constexpr uint32_t kCounterSlots = 4096;

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

}  // namespace sqi

struct sq_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  int sm_count = 0;
  int order = SQ_ORDER_NEAR_FIRST;  // certified near-first; the reference order on request
  int blocks_per_sm = 0;
  uint32_t* d_counters = nullptr;
  uint32_t slot = 0;
  unsigned long long* d_stats = nullptr;
  sqi::DevBuf arena;
  uint32_t* d_replays = nullptr;  // queries of the last near-first launch answered again in reference order
  sqi::DevBuf replay_list;        // their indices (grown to the largest batch)
  float window = 0x1p-16f;        // relative window past the limit within which near-first still visits nodes
  int layout = SQ_LAYOUT_BINARY;  // node records of near-first nearest rays (SQ_LAYOUT_*)
  cudaStream_t s_in = nullptr, s_out = nullptr;  // copy streams of the chunked host-buffer calls (made on first use)
  sq_ctx* lane = nullptr;  // second compute lane of the chunked host-buffer calls (own stream and scratch; made on first use)
  uint64_t launches = 0;
  std::unordered_map<uint64_t, int> occ;  // (kernel, dynamic smem) -> resident blocks per SM
  cudaMemPool_t pool = nullptr;  // stream-ordered scratch that stays reserved between calls (scratch_alloc)
  cudaAccessPolicyWindow l2_window{};  // sq_ctx_set_l2_persist (num_bytes 0: none)
};

// An uploaded scene: device records plus the host topology (kept for the
// learned guide's bucket table and for reading bounds back).
struct sq_bvh {
  int device = 0;
  int dim = 0;
  int narrow = 0;
  uint32_t n_nodes = 0, n_prims = 0, n_interior = 0, depth = 0, n_leaves = 0;
  uint32_t stride = 0;
  uint32_t prim_vec = 0;  // 16-byte vectors per primitive record
  uint32_t root_code = 0;
  float4* d_nodes = nullptr;
  float4* d_prims = nullptr;
  float* d_root = nullptr;
  uint64_t* d_layers = nullptr;
  uint32_t* d_sub = nullptr;
  uint32_t* d_prim_ids = nullptr;
  sq::RefitLeaf* d_leaves = nullptr;
  uint32_t* d_parents = nullptr;
  uint32_t* d_arrivals = nullptr;
  float* d_refit_in = nullptr;  // staging for host refit data
  int* d_nonfinite = nullptr;   // non-zero when some node bound is not finite
  sq::KernelSet ks{};
  size_t bytes = 0;
  std::vector<uint32_t> h_iidx;  // host node -> interior record (or kNoHit)
  std::vector<uint32_t> h_child_a, h_child_b, h_count;
  // Four-wide records (WideLayout) built at upload for near-first rays, and
  // for each of their slots the binary record slot holding the same box.
  float4* d_wnodes = nullptr;
  uint32_t* d_wsrc = nullptr;
  uint32_t n_wide = 0, wroot = 0, wdepth = 0;
  // The same four-wide records quantised (QuantLayout), same numbering.
  float4* d_qnodes = nullptr;
  // An f64 scene (sq_bvh_upload_f64): node boxes, node links and leaf
  // parameters in double, answered only by the _f64 entry points.
  int prec = 32;
  double* d_nb64 = nullptr;   // [n_nodes][2D]
  uint2* d_nc64 = nullptr;    // [n_nodes]: (child_a, child_b), or (first, count | kLeafBit)
  double* d_prims64 = nullptr;  // [n_prims][stride], leaf order
};

namespace sqi {

using namespace sq;

// Near-first nearest launch `fn` followed by the reference-order replay
// (`ref_fn`) of the queries it could not certify; with `ref_fn` null the
// kernel answers those queries again itself (sq_api.cu).
constexpr bool kReplayInKernel = SQ_REPLAY_IN_KERNEL && !SQ_POSTPONE_LEAVES;
int32_t near_first_launch(sq_ctx* ctx, const sq_bvh* b, const void* fn, const void* ref_fn, QueryParams& p,
                          uint32_t stack);

// Consumer narrow phases (rtc.cpp): the kernels of a D = 3 scene whose
// narrow phase is `src` with `stride` floats per leaf, compiled with NVRTC
// (cached per stride and source). SQ_ERR_COMPILE with the compiler log.
constexpr uint32_t kMaxCustomStride = 32;
int32_t rtc_kernel_set(uint32_t stride, const char* src, KernelSet* out, std::string* log);

// Host-buffer calls in chunks: chunk c's inputs are copied in on the
// context's copy-in stream while earlier chunks run, and their results are
// copied out on the copy-out stream meanwhile (sq_api.cu). Chunks alternate
// between two compute lanes, the context itself and ctx->lane (its own
// stream, launch counters and replay list), so that one chunk's first
// launches fill the SMs left idle by the other's last long queries.
// in(s, m, stream) / out(s, m, stream) enqueue the copies of queries
// [s, s + m); run(lane, s, m) enqueues the work on lane->stream using only
// that lane's scratch. One chunk when n is small. Returns when every copy out
// has landed.
uint32_t pipeline_chunks(uint32_t n);
// Frees the learned guide's per-context error flag (guide.cu); called when
// the context is destroyed.
void release_err_slot(sq_ctx* ctx);
// ctx->lane, made on first use, with the context's traversal settings.
int32_t second_lane(sq_ctx* ctx, sq_ctx** out);
int32_t pipelined(sq_ctx* ctx, uint32_t n, const std::function<int32_t(uint32_t, uint32_t, cudaStream_t)>& in,
                  const std::function<int32_t(sq_ctx*, uint32_t, uint32_t)>& run,
                  const std::function<int32_t(uint32_t, uint32_t, cudaStream_t)>& out);

// Sorts each CSR segment [offsets[i], offsets[i+1]) of `leaves` ascending
// (sq_api.cu): the fill passes append in walk order.
int32_t sort_csr_segments(sq_ctx* ctx, uint32_t* d_leaves, uint64_t total, const uint64_t* d_offsets, uint32_t n);

// The learned guide's buckets on the device: per bucket its node code and
// the slot of its box (parent record << 1 | slot, kNoHit for the root), and
// the slots of its ancestors' other children, root level first, sib_stride
// per bucket (kNoHit past the bucket's depth).
struct SeedTable {
  const uint2* buckets = nullptr;
  const uint32_t* sibs = nullptr;
  uint32_t n_buckets = 0;
  uint32_t sib_stride = 0;
};

// Learned-seeded nearest rays (sq_api.cu): enqueues the SEED kernel.
int32_t seeded_nearest(sq_ctx* ctx, const sq_bvh* b, const float* d_rays, uint32_t n, float max_toi,
                       const int32_t* d_bucket, const SeedTable& seeds, const sq_hits& o, sq_query_stats* st);

inline int32_t fail(sq_ctx* c, int32_t code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

inline int32_t cuda_fail(sq_ctx* c, const char* what, cudaError_t e) {
  return fail(c, SQ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(x)                                          \
  do {                                                 \
    cudaError_t e_ = (x);                              \
    if (e_ != cudaSuccess) return cuda_fail(ctx, #x, e_); \
  } while (0)

inline bool kernel_set(int dim, int narrow, KernelSet* out) {
  switch (dim) {
    case 2: return kernel_set_d2(narrow, out);
    case 3: return kernel_set_d3(narrow, out);
    case 4: return kernel_set_d4(narrow, out);
    case 6: return kernel_set_d6(narrow, out);
    default: return false;
  }
}

inline uint32_t stride_of(int dim, int narrow) {
  switch (narrow) {
    case SQ_NARROW_AABB: return 2 * dim;
    case SQ_NARROW_SPHERE:
    case SQ_NARROW_SPHERE_NEAR: return dim + 1;
    case SQ_NARROW_TRIANGLE: return 9;
    default: return 0;
  }
}

inline uint32_t prim_vec(int dim, int narrow) {
  uint32_t payload = narrow == SQ_NARROW_AABB ? 2 * dim : (narrow == SQ_NARROW_TRIANGLE ? 9 : dim + 1);
  return (payload + 1 + 3) / 4;
}

inline uint32_t node_vec(int dim) { return (4 * dim + 2 + 3) / 4; }
inline uint32_t wide_vec(int dim) { return (8 * dim + 4 + 3) / 4; }
inline uint32_t quant_vec(int dim) { return (dim + (dim + 3) / 4 + 2 * dim + 4 + 3) / 4; }

// Stream-ordered scratch on the context's stream from the context's own
// memory pool. The pool keeps what is freed for the next call (no release
// threshold); the device's default pool hands freed memory back to the
// driver at every synchronisation, and mapping it again cost 1-5 ms per
// call (197 ms once) in a D = 6 overlap query whose kernels take 2 ms.
inline cudaError_t scratch_alloc(sq_ctx* ctx, void** p, size_t bytes) {
  return cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream);
}

inline int32_t arena_reserve(sq_ctx* ctx, size_t bytes) {
  if (ctx->arena.cap >= bytes) return SQ_OK;
  if (ctx->arena.p) {
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(ctx->arena.p));
    ctx->arena.p = nullptr;
    ctx->arena.cap = 0;
  }
  size_t cap = std::max<size_t>(bytes, size_t(1) << 20);
  CK(cudaMalloc(&ctx->arena.p, cap));
  ctx->arena.cap = cap;
  return SQ_OK;
}

// Carves 256-byte-aligned pieces out of the arena.
struct Carve {
  size_t off = 0;
  size_t take(size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  }
};

inline int occupancy(sq_ctx* ctx, const void* fn, size_t smem) {
  const uint64_t key = uint64_t(uintptr_t(fn)) * 131 + smem;
  auto it = ctx->occ.find(key);
  if (it != ctx->occ.end()) return it->second;
  int nb = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kThreads, smem) != cudaSuccess || nb < 1) nb = 1;
  ctx->occ[key] = nb;
  return nb;
}

// The persistent grid: (resident blocks per SM) x (SM count), no more blocks
// than the queries need. The traversal stack is dynamic shared memory sized
// to the tree depth, so shallow trees leave room for more resident warps.
// Launches a persistent kernel whose single parameter is *params (with its
// counter and stack fields set here) on the context's stream.
template <class Params>
inline int32_t launch_persistent(sq_ctx* ctx, const void* fn, Params& p, uint32_t depth, uint64_t n);

template <class Params>
inline int32_t launch_persistent(sq_ctx* ctx, const void* fn, Params& p, uint32_t depth, uint64_t n) {
  uint32_t* ctr = ctx->d_counters + (ctx->slot++ % kCounterSlots);
  CK(cudaMemsetAsync(ctr, 0, sizeof(uint32_t), ctx->stream));
  p.counter = ctr;
  p.stack = int(std::max<uint32_t>(depth, 1));
  const size_t smem = size_t(p.stack) * kThreads * 8;
  if (smem > 48 * 1024) CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int bps = ctx->blocks_per_sm > 0 ? ctx->blocks_per_sm : occupancy(ctx, fn, smem);
  uint64_t want = (n + kThreads - 1) / kThreads;
  uint64_t grid = std::min<uint64_t>(uint64_t(ctx->sm_count) * bps, std::max<uint64_t>(want, 1));
  void* args[] = {&p};
  CK(cudaLaunchKernel(fn, dim3(unsigned(grid)), dim3(kThreads), args, smem, ctx->stream));
  ctx->launches++;
  return SQ_OK;
}


}  // namespace sqi
