// Device build of the crate's median-split tree: tree::build
// (crates/spatial-query/src/accel/tree.rs:39-49, 112-163) on the GPU. The
// output is the host restatement's (sq_tree_build, tree_build.cpp) array for
// array: preorder nodes with the root at 0; a leaf holds <= 4 primitives
// unless all its centroids coincide within f32::EPSILON on the longest
// centroid axis; the split axis is the first longest axis of the centroid
// bounds; the primitives of a node are stably sorted by that centroid
// coordinate under f32::total_cmp and split at start + count / 2.
//
// How: the recursion runs a level at a time. For every segment of a level
// (a node's range of the primitive order) the node's box and its centroid
// box are reduced (one warp per segment on the wide levels; many blocks per
// segment with order-preserving integer atomics on the top levels, whose
// few segments are long), leaf or split is decided, and each primitive of a
// split segment gets the sort key (segment start << 32 | its split-axis key);
// every other position keeps (position << 32). One stable radix sort of the
// level on those keys then orders every split segment in place, which is the
// per-node stable sort of the crate (ties keep the order the parent's sort
// left), and leaves every other position where it is. Nodes are numbered in
// level order as they are made; preorder numbers follow from subtree sizes
// (bottom-up, a level at a time) and left-subtree offsets (top-down).
//
// The host never waits inside the build: a median split halves the longest
// segment, so the number of levels and a bound on each level's segment count
// follow from n alone; grids are sized by those bounds and every kernel reads
// the level's true segment count from device memory (a one-thread kernel
// closes each level). The one synchronisation is at the end, for the node
// count the call returns.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <vector>

#include "sq_internal.cuh"

using sqi::cuda_fail;

namespace {

constexpr uint32_t kLeafSize = 4;
constexpr float kEps = 1.1920928955078125e-7f;  // f32::EPSILON
constexpr int kMaxDim = 8;
constexpr uint32_t kNone = 0xFFFFFFFFu;

struct Seg {
  uint32_t s, e, node;  // positions [s, e) of the primitive order; level-order node id
};

struct LNode {
  uint32_t s, e, a, b;  // range; children's level-order ids (a == kNone: leaf)
};

// f32::total_cmp as an unsigned order: negative values bit-inverted,
// non-negative values with the sign bit set.
__device__ __forceinline__ uint32_t total_ukey(float x) {
  const uint32_t b = __float_as_uint(x);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Aabb::center (aabb.rs:56-58): (min + max) * 0.5 per axis.
__device__ __forceinline__ float centre(const float* box, int D, int k) {
  return __fmul_rn(__fadd_rn(box[k], box[D + k]), 0.5f);
}

__global__ void keys_kernel(const float* __restrict__ aabbs, uint32_t n, int D, uint32_t* keys, uint32_t* idx) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    idx[i] = i;
    const float* b = aabbs + size_t(i) * 2 * D;
    for (int k = 0; k < D; ++k) keys[size_t(k) * n + i] = total_ukey(centre(b, D, k));
  }
}

struct LevelParams {
  const float* aabbs;
  int D;
  uint32_t n;
  const uint32_t* keys;  // [D][n]
  const uint32_t* idx;   // the current primitive order
  const Seg* cur;
  const uint32_t* m;     // segments of this level (device memory)
  Seg* next;             // the next level's segments (appended)
  uint32_t* counters;    // [0] next segments, [1] nodes made, [2] split segments
  LNode* nodes;          // by level-order id
  float* bounds;         // by level-order id: min[D], max[D]
  unsigned long long* sort_keys;  // per position: (segment start << 32) | split-axis key, or (position << 32)
  uint32_t* red;         // top levels: per segment 4 x kMaxDim ordered bounds (box lo, hi, centroid lo, hi)
  int* axis;             // top levels: per segment the split axis, -1 for a leaf
  uint32_t chunk;        // top levels: positions per block
};

// f32 <-> an unsigned key with the same order (total_ukey), for min / max
// by integer atomics; NaN coordinates are skipped, as fminf / fmaxf skip them.
__device__ __forceinline__ float ukey_float(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Leaf or split of segment sg from its reduced boxes (tree.rs:129-154):
// writes the node's bounds and record, appends the children's segments,
// and returns the split axis (-1: leaf). One thread per segment.
__device__ int decide(const LevelParams& p, const Seg& sg, const float* lo, const float* hi, const float* clo,
                      const float* chi) {
  const int D = p.D;
  const uint32_t count = sg.e - sg.s;
  float* bo = p.bounds + size_t(sg.node) * 2 * D;
  for (int k = 0; k < D; ++k) {
    bo[k] = lo[k];
    bo[D + k] = hi[k];
  }
  LNode nd{sg.s, sg.e, kNone, kNone};
  int axis = -1;
  if (count > kLeafSize) {
    int ax = 0;
    float ext[kMaxDim];
    for (int k = 0; k < D; ++k) ext[k] = __fsub_rn(chi[k], clo[k]);
    for (int k = 1; k < D; ++k)
      if (ext[k] > ext[ax]) ax = k;
    if (ext[ax] > kEps) {
      axis = ax;
      const uint32_t mid = sg.s + count / 2;
      const uint32_t c0 = atomicAdd(&p.counters[0], 2u);
      const uint32_t id0 = atomicAdd(&p.counters[1], 2u);
      p.next[c0] = Seg{sg.s, mid, id0};
      p.next[c0 + 1] = Seg{mid, sg.e, id0 + 1};
      nd.a = id0;
      nd.b = id0 + 1;
      atomicAdd(&p.counters[2], 1u);
    }
  }
  p.nodes[sg.node] = nd;
  return axis;
}

// Closes level L: the next level's segments were appended with level-order
// ids [made - count, made); records them and clears the per-level counters.
__global__ void advance_kernel(uint32_t* counters, uint32_t* level_info, uint32_t L) {
  const uint32_t m_next = counters[0], made = counters[1];
  level_info[2 * (L + 1)] = made - m_next;
  level_info[2 * (L + 1) + 1] = m_next;
  counters[0] = 0;
  counters[2] = 0;
}

// Every position keeps its place unless a split segment claims it.
__global__ void place_keys_kernel(unsigned long long* sort_keys, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    sort_keys[i] = (unsigned long long)i << 32;
}

// Top levels: empty per-segment bounds (+inf for the minima, -inf for the maxima).
__global__ void red_init_kernel(uint32_t* red, uint32_t m) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m * 4 * kMaxDim) return;
  const uint32_t part = (i / kMaxDim) % 4;  // 0 lo, 1 hi, 2 centroid lo, 3 centroid hi
  red[i] = (part == 0 || part == 2) ? total_ukey(INFINITY) : total_ukey(-INFINITY);
}

// Top levels: block (c, g) reduces positions [s + c * chunk, s + (c + 1) * chunk)
// of segment g and folds its result into the segment's bounds.
__global__ void __launch_bounds__(256) red_kernel(const LevelParams p) {
  const uint32_t g = blockIdx.y;
  if (g >= *p.m) return;  // the grid covers the level's bound
  const Seg sg = p.cur[g];
  const uint64_t b0 = uint64_t(sg.s) + uint64_t(blockIdx.x) * p.chunk;
  if (b0 >= sg.e) return;  // uniform per block
  const uint32_t b1 = uint32_t(std::min<uint64_t>(sg.e, b0 + p.chunk));
  const int D = p.D;
  float lo[kMaxDim], hi[kMaxDim], clo[kMaxDim], chi[kMaxDim];
#pragma unroll
  for (int k = 0; k < kMaxDim; ++k) {
    lo[k] = clo[k] = INFINITY;
    hi[k] = chi[k] = -INFINITY;
  }
  for (uint32_t pos = uint32_t(b0) + threadIdx.x; pos < b1; pos += blockDim.x) {
    const float* b = p.aabbs + size_t(p.idx[pos]) * 2 * D;
#pragma unroll
    for (int k = 0; k < kMaxDim; ++k) {
      if (k < D) {
        lo[k] = fminf(lo[k], b[k]);
        hi[k] = fmaxf(hi[k], b[D + k]);
        const float c = centre(b, D, k);
        clo[k] = fminf(clo[k], c);
        chi[k] = fmaxf(chi[k], c);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < kMaxDim; ++k) {
      if (k < D) {
        lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
        hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        clo[k] = fminf(clo[k], __shfl_xor_sync(0xffffffffu, clo[k], o));
        chi[k] = fmaxf(chi[k], __shfl_xor_sync(0xffffffffu, chi[k], o));
      }
    }
  }
  if ((threadIdx.x & 31) == 0) {
    uint32_t* r = p.red + size_t(g) * 4 * kMaxDim;
    for (int k = 0; k < D; ++k) {
      if (!isnan(lo[k])) atomicMin(&r[k], total_ukey(lo[k]));
      if (!isnan(hi[k])) atomicMax(&r[kMaxDim + k], total_ukey(hi[k]));
      if (!isnan(clo[k])) atomicMin(&r[2 * kMaxDim + k], total_ukey(clo[k]));
      if (!isnan(chi[k])) atomicMax(&r[3 * kMaxDim + k], total_ukey(chi[k]));
    }
  }
}

// Top levels: leaf or split per segment from the reduced bounds.
__global__ void decide_kernel(const LevelParams p) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= *p.m) return;
  const uint32_t* r = p.red + size_t(g) * 4 * kMaxDim;
  float lo[kMaxDim], hi[kMaxDim], clo[kMaxDim], chi[kMaxDim];
  for (int k = 0; k < p.D; ++k) {
    lo[k] = ukey_float(r[k]);
    hi[k] = ukey_float(r[kMaxDim + k]);
    clo[k] = ukey_float(r[2 * kMaxDim + k]);
    chi[k] = ukey_float(r[3 * kMaxDim + k]);
  }
  p.axis[g] = decide(p, p.cur[g], lo, hi, clo, chi);
}

// Top levels: the sort keys of the split segments' positions, chunked like red_kernel.
__global__ void split_keys_kernel(const LevelParams p) {
  const uint32_t g = blockIdx.y;
  if (g >= *p.m) return;
  const int axis = p.axis[g];
  if (axis < 0) return;
  const Seg sg = p.cur[g];
  const uint64_t b0 = uint64_t(sg.s) + uint64_t(blockIdx.x) * p.chunk;
  if (b0 >= sg.e) return;
  const uint32_t b1 = uint32_t(std::min<uint64_t>(sg.e, b0 + p.chunk));
  const uint32_t* key = p.keys + size_t(axis) * p.n;
  for (uint32_t pos = uint32_t(b0) + threadIdx.x; pos < b1; pos += blockDim.x)
    p.sort_keys[pos] = ((unsigned long long)sg.s << 32) | key[p.idx[pos]];
}

// Wide levels: one warp per segment.
template <int TPS>
__global__ void __launch_bounds__(256) level_kernel(const LevelParams p) {
  static_assert(TPS == 32, "one warp per segment");
  const uint32_t groups = blockDim.x / TPS;
  const uint32_t g = blockIdx.x * groups + threadIdx.x / TPS;
  const uint32_t lane = threadIdx.x % TPS;
  if (g >= *p.m) return;  // uniform per warp
  const int D = p.D;
  const Seg sg = p.cur[g];
  float lo[kMaxDim], hi[kMaxDim], clo[kMaxDim], chi[kMaxDim];
#pragma unroll
  for (int k = 0; k < kMaxDim; ++k) {
    lo[k] = clo[k] = INFINITY;
    hi[k] = chi[k] = -INFINITY;
  }
  for (uint32_t pos = sg.s + lane; pos < sg.e; pos += TPS) {
    const float* b = p.aabbs + size_t(p.idx[pos]) * 2 * D;
#pragma unroll
    for (int k = 0; k < kMaxDim; ++k) {
      if (k < D) {
        lo[k] = fminf(lo[k], b[k]);
        hi[k] = fmaxf(hi[k], b[D + k]);
        const float c = centre(b, D, k);
        clo[k] = fminf(clo[k], c);
        chi[k] = fmaxf(chi[k], c);
      }
    }
  }
  // Group reduction (min / max are exact in any order).
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < kMaxDim; ++k) {
      if (k < D) {
        lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
        hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        clo[k] = fminf(clo[k], __shfl_xor_sync(0xffffffffu, clo[k], o));
        chi[k] = fmaxf(chi[k], __shfl_xor_sync(0xffffffffu, chi[k], o));
      }
    }
  }
  // Leaf or split, decided by the warp's first lane.
  int axis = -1;
  if (lane == 0) axis = decide(p, sg, lo, hi, clo, chi);
  axis = __shfl_sync(0xffffffffu, axis, 0);
  if (axis < 0) return;
  const uint32_t* key = p.keys + size_t(axis) * p.n;
  for (uint32_t pos = sg.s + lane; pos < sg.e; pos += TPS)
    p.sort_keys[pos] = ((unsigned long long)sg.s << 32) | key[p.idx[pos]];
}

// Subtree node counts, one level at a time from the deepest (level L's ids
// are [level_info[2L], + level_info[2L + 1])).
__global__ void sizes_kernel(const LNode* __restrict__ nodes, const uint32_t* level_info, uint32_t L, uint32_t* size) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= level_info[2 * L + 1]) return;
  const uint32_t id = level_info[2 * L] + i;
  const LNode nd = nodes[id];
  size[id] = nd.a == kNone ? 1u : 1u + size[nd.a] + size[nd.b];
}

// Preorder numbers, one level at a time from the root: the left child
// follows its parent, the right child follows the left subtree.
__global__ void preorder_kernel(const LNode* __restrict__ nodes, const uint32_t* level_info, uint32_t L,
                                const uint32_t* size, uint32_t* pre) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= level_info[2 * L + 1]) return;
  const uint32_t id = level_info[2 * L] + i;
  const LNode nd = nodes[id];
  if (nd.a == kNone) return;
  pre[nd.a] = pre[id] + 1;
  pre[nd.b] = pre[id] + 1 + size[nd.a];
}

// The crate's node arrays in preorder (tree::Node: bounds, and either the
// children's indices or the leaf's first position and count).
__global__ void emit_kernel(const LNode* __restrict__ nodes, const float* __restrict__ lbounds,
                            const uint32_t* __restrict__ pre, const uint32_t* made, uint32_t capacity, int D,
                            float* node_bounds, uint32_t* child_a, uint32_t* child_b, uint32_t* prim_count) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= *made || id >= capacity) return;
  const LNode nd = nodes[id];
  const uint32_t i = pre[id];
  for (int k = 0; k < 2 * D; ++k) node_bounds[size_t(i) * 2 * D + k] = lbounds[size_t(id) * 2 * D + k];
  if (nd.a == kNone) {
    child_a[i] = nd.s;
    child_b[i] = 0;
    prim_count[i] = nd.e - nd.s;
  } else {
    child_a[i] = pre[nd.a];
    child_b[i] = pre[nd.b];
    prim_count[i] = 0;
  }
}

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return uint32_t(std::max<uint64_t>(1, (n + t - 1) / t)); }

}  // namespace

extern "C" int32_t sq_tree_build_d(sq_ctx* ctx, int32_t dim, uint32_t n, const float* d_prim_aabbs,
                                   uint32_t node_capacity, uint32_t* n_nodes_out, float* d_node_bounds,
                                   uint32_t* d_child_a, uint32_t* d_child_b, uint32_t* d_prim_count,
                                   uint32_t* d_prim_indices) {
  using sqi::fail;
  if (!ctx || !n_nodes_out) return SQ_ERR_INVALID;
  *n_nodes_out = 0;
  if (dim < 1 || dim > kMaxDim) return fail(ctx, SQ_ERR_INVALID, "dim must be 1..8");
  if (n == 0) return SQ_OK;
  if (!d_prim_aabbs || !d_node_bounds || !d_child_a || !d_child_b || !d_prim_count || !d_prim_indices)
    return fail(ctx, SQ_ERR_INVALID, "null tree array");
  if (uint64_t(node_capacity) < 2ull * n - 1) return fail(ctx, SQ_ERR_CAPACITY, "node_capacity below 2n - 1");
  if (n >= sq::kLeafBit) return fail(ctx, SQ_ERR_INVALID, "too many primitives");
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int D = dim;
  const size_t N2 = size_t(2) * n;  // node capacity of the level-order arrays

  // The levels: a median split halves the longest segment, and a segment of
  // at most kLeafSize primitives is a leaf, so the level where the longest
  // segment first fits a leaf is the last; level L has at most min(2^L, n)
  // segments.
  std::vector<uint64_t> longest_at{n};
  while (longest_at.back() > kLeafSize) longest_at.push_back((longest_at.back() + 1) / 2);
  const uint32_t n_levels = uint32_t(longest_at.size());
  auto bound_at = [&](uint32_t L) { return L >= 32 ? uint64_t(n) : std::min<uint64_t>(uint64_t(1) << L, n); };

  // Scratch, carved from one stream-ordered allocation.
  sqi::Carve cv;
  constexpr uint32_t kWide = 1024;  // levels with this many segments or more: one warp per segment
  size_t sort_bytes = 0;
  int pos_bits = 1;
  while (pos_bits < 32 && (uint64_t(1) << pos_bits) < n) ++pos_bits;
  const int end_bit = 32 + pos_bits;  // positions fit in the keys' high word
  CK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, static_cast<unsigned long long*>(nullptr),
                                     static_cast<unsigned long long*>(nullptr), static_cast<uint32_t*>(nullptr),
                                     static_cast<uint32_t*>(nullptr), int(n), 0, end_bit, st));
  const size_t o_keys = cv.take(size_t(D) * n * 4), o_idx0 = cv.take(size_t(n) * 4), o_idx1 = cv.take(size_t(n) * 4),
               o_sk0 = cv.take(size_t(n) * 8), o_sk1 = cv.take(size_t(n) * 8),
               o_seg0 = cv.take((size_t(n) + 1) * sizeof(Seg)), o_seg1 = cv.take((size_t(n) + 1) * sizeof(Seg)),
               o_red = cv.take(size_t(kWide) * 4 * kMaxDim * 4), o_axis = cv.take(size_t(kWide) * 4),
               o_nodes = cv.take(N2 * sizeof(LNode)), o_lb = cv.take(N2 * 2 * D * 4), o_size = cv.take(N2 * 4),
               o_pre = cv.take(N2 * 4), o_ctr = cv.take(16), o_lv = cv.take(size_t(2) * (n_levels + 1) * 4),
               o_sort = cv.take(sort_bytes);
  char* base = nullptr;
  CK(sqi::scratch_alloc(ctx, reinterpret_cast<void**>(&base), cv.off));
  uint32_t* keys = reinterpret_cast<uint32_t*>(base + o_keys);
  uint32_t* idx = reinterpret_cast<uint32_t*>(base + o_idx0);
  uint32_t* idx_alt = reinterpret_cast<uint32_t*>(base + o_idx1);
  unsigned long long* skeys = reinterpret_cast<unsigned long long*>(base + o_sk0);
  unsigned long long* skeys_alt = reinterpret_cast<unsigned long long*>(base + o_sk1);
  Seg* cur = reinterpret_cast<Seg*>(base + o_seg0);
  Seg* nxt = reinterpret_cast<Seg*>(base + o_seg1);
  uint32_t* red = reinterpret_cast<uint32_t*>(base + o_red);
  int* axis = reinterpret_cast<int*>(base + o_axis);
  LNode* nodes = reinterpret_cast<LNode*>(base + o_nodes);
  float* lbounds = reinterpret_cast<float*>(base + o_lb);
  uint32_t* size = reinterpret_cast<uint32_t*>(base + o_size);
  uint32_t* pre = reinterpret_cast<uint32_t*>(base + o_pre);
  uint32_t* ctr = reinterpret_cast<uint32_t*>(base + o_ctr);
  uint32_t* level_info = reinterpret_cast<uint32_t*>(base + o_lv);
  void* temp = base + o_sort;
  auto done = [&](int32_t code) {
    cudaFreeAsync(base, st);
    return code;
  };
#define CKB(x)                                                  \
  do {                                                          \
    cudaError_t e_ = (x);                                       \
    if (e_ != cudaSuccess) return done(cuda_fail(ctx, #x, e_)); \
  } while (0)

  keys_kernel<<<std::min<uint32_t>(blocks_for(n, 256), 148 * 16), 256, 0, st>>>(d_prim_aabbs, n, D, keys, idx);
  CKB(cudaGetLastError());
  const Seg root{0, n, 0};
  CKB(cudaMemcpyAsync(cur, &root, sizeof(Seg), cudaMemcpyHostToDevice, st));
  const uint32_t init[4] = {0, 1, 0, 0};  // next segments, nodes made, split segments
  CKB(cudaMemcpyAsync(ctr, init, sizeof(init), cudaMemcpyHostToDevice, st));
  const uint32_t root_level[2] = {0, 1};  // level 0: id 0, one segment
  CKB(cudaMemcpyAsync(level_info, root_level, sizeof(root_level), cudaMemcpyHostToDevice, st));
  uint64_t own_launches = 1;  // keys_kernel
  for (uint32_t L = 0; L < n_levels; ++L) {
    const uint64_t bound = bound_at(L), longest = longest_at[L];
    const bool may_split = longest > kLeafSize;  // false only on the last level
    if (may_split) place_keys_kernel<<<std::min<uint32_t>(blocks_for(n, 256), 148 * 8), 256, 0, st>>>(skeys, n);
    LevelParams p{d_prim_aabbs, D, n, keys, idx, cur, level_info + 2 * L + 1, nxt, ctr, nodes, lbounds, skeys, red,
                  axis, 4096u};
    if (bound >= kWide) {
      level_kernel<32><<<blocks_for(bound, 8), 256, 0, st>>>(p);
      own_launches += 1;
    } else {
      const dim3 grid(uint32_t(std::max<uint64_t>(1, (longest + p.chunk - 1) / p.chunk)), uint32_t(bound));
      red_init_kernel<<<blocks_for(bound * 4 * kMaxDim, 256), 256, 0, st>>>(red, uint32_t(bound));
      red_kernel<<<grid, 256, 0, st>>>(p);
      decide_kernel<<<blocks_for(bound, 128), 128, 0, st>>>(p);
      split_keys_kernel<<<grid, 256, 0, st>>>(p);
      own_launches += 4;
    }
    advance_kernel<<<1, 1, 0, st>>>(ctr, level_info, L);
    own_launches += 1 + (may_split ? 1 : 0);
    CKB(cudaGetLastError());
    if (may_split) {
      size_t need = sort_bytes;
      CKB(cub::DeviceRadixSort::SortPairs(temp, need, skeys, skeys_alt, idx, idx_alt, int(n), 0, end_bit, st));
      std::swap(idx, idx_alt);
      own_launches += 1;
    }
    std::swap(cur, nxt);
  }
  for (uint32_t L = n_levels; L-- > 0;)
    sizes_kernel<<<blocks_for(bound_at(L), 256), 256, 0, st>>>(nodes, level_info, L, size);
  CKB(cudaMemsetAsync(pre, 0, 4, st));
  for (uint32_t L = 0; L < n_levels; ++L)
    preorder_kernel<<<blocks_for(bound_at(L), 256), 256, 0, st>>>(nodes, level_info, L, size, pre);
  emit_kernel<<<blocks_for(uint64_t(2) * n - 1, 256), 256, 0, st>>>(nodes, lbounds, pre, ctr + 1, node_capacity, D,
                                                                    d_node_bounds, d_child_a, d_child_b, d_prim_count);
  CKB(cudaGetLastError());
  CKB(cudaMemcpyAsync(d_prim_indices, idx, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
  uint32_t n_nodes = 0;
  CKB(cudaMemcpyAsync(&n_nodes, ctr + 1, 4, cudaMemcpyDeviceToHost, st));
  ctx->launches += own_launches + 2 * n_levels + 1;
  int32_t rc = done(SQ_OK);
  CK(cudaStreamSynchronize(st));
  if (n_nodes > node_capacity) return fail(ctx, SQ_ERR_CAPACITY, "node_capacity too small");
  *n_nodes_out = n_nodes;
#undef CKB
  return rc;
}
