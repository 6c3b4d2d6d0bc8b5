// Persistent, warp-pulled BVH traversal kernels for sm_100a.
//
// Replaces the WGSL `main` of crates/spatial-query/src/gpu/mod.rs:159-226 (one
// invocation per ray, 48-byte nodes, no ordering) with:
//  * a child-pair node record: an interior node holds both children's boxes
//    and codes in 16-byte vectors (64 B at D = 3), so one record fetch tests
//    two boxes;
//  * a persistent grid (a multiple of the SM count) whose warps pull batches
//    of 32 queries from an atomic counter, so uneven per-query work balances;
//  * a per-thread traversal stack in shared memory ([depth][thread], so
//    consecutive lanes hit consecutive banks), each entry carrying the child's
//    slab entry so it can be re-checked exactly against the shrunk limit when
//    popped;
//  * near-first child ordering for nearest queries, or the reference's own
//    order (push child_a, then child_b, pop child_b first; accel/bvh.rs:119-120)
//    when REF is set, which replays the CPU decisions one for one.
//
// Node code: an interior record index, or kLeafBit | the first position of the
// leaf's primitives in the leaf-ordered primitive array. The last primitive of
// a leaf carries kLeafBit in its id word.
#pragma once

#include "sq_math.cuh"

namespace sq {

enum Narrow : int { kNarrowAabb = 0, kNarrowSphere = 1, kNarrowSphereNear = 2, kNarrowTri = 3, kNarrowCustom = 4 };

// A consumer narrow phase (kNarrowCustom) is compiled at run time with NVRTC
// into the same kernels: its source defines
//   __device__ bool sq_narrow(const float* prim, uint32_t leaf, const float* ro, const float* rd,
//                             float max_toi, float* toi, float* normal);
// and SQ_CUSTOM_STRIDE is the number of floats per leaf. Its primitive
// record holds those floats, then the leaf's AABB (the box the tree was built
// from, used to certify near-first answers), then the id word.
#ifndef SQ_CUSTOM_STRIDE
#define SQ_CUSTOM_STRIDE 1
#endif
#ifdef SQ_RTC_CUSTOM
__device__ bool sq_narrow(const float* prim, uint32_t leaf, const float* ro, const float* rd, float max_toi, float* toi,
                          float* normal);
#endif
// Optionally the source also defines every crossing of a leaf
// (QueryGeometry::test_ray_crossings, consumed by Bvh::raycast_crossings,
// accel/bvh.rs:286-328); SQ_RTC_CROSSINGS is then defined and
// raycast_crossings lists each emit(toi, normal) call:
//   template <class Emit>
//   __device__ void sq_narrow_crossings(const float* prim, uint32_t leaf, const float* ro, const float* rd,
//                                       float max_toi, Emit& emit);
#ifdef SQ_RTC_CROSSINGS
template <class Emit>
__device__ void sq_narrow_crossings(const float* prim, uint32_t leaf, const float* ro, const float* rd, float max_toi,
                                    Emit& emit);
#endif
enum QKind : int { kRayNearest = 0, kRayAll = 1, kCastNearest = 2, kCastAll = 3, kOverlap = 4 };

// Leaves per region the overlap count pass keeps (QueryParams::keep).
constexpr uint32_t kOverlapKeep = 4;

constexpr int kThreads = 128;

// Two walk variants, measured on the 1,048,576-triangle terrain and off by
// default (each slower there; both together are also built as the WALK = 1
// instantiation, SQ_LAYOUT_BINARY_REGTOP, which the autotuner can pick):
//  * SQ_POSTPONE_LEAVES: a lane that reaches a leaf holds it and keeps
//    descending until the whole warp holds leaves (Aila and Laine's
//    speculative traversal): 0.697 ms against 0.621 ms per 1,048,576 rays;
//    the nodes it visits before the leaf's hit tightens the limit cost more
//    than the leaf tests gain from running together.
//  * SQ_REG_TOP (with postponed leaves): the stack's top entry in registers,
//    older entries in the shared-memory stack: 0.729 ms; five more registers
//    per thread cut the resident blocks from nine to eight, and the saved
//    shared-memory round trip is short next to a node fetch from L2.
#ifndef SQ_POSTPONE_LEAVES
#define SQ_POSTPONE_LEAVES 0
#endif
#ifndef SQ_REG_TOP
#define SQ_REG_TOP 0
#endif
// Uncertified near-first answers answered again by the same lane at its
// next refill (1), or listed for a reference-order launch (0, the default).
// The lane replay removes the second launch (about 20 us per 1,048,576-ray
// call, the serial walk of the one or two listed rays) but measured 0.918 ms
// against 0.619 ms for the child-pair walk of the terrain's rays, with the
// same single replay in both: the replay state in the refill loop costs the
// whole walk far more than the launch it saves.
#ifndef SQ_REPLAY_IN_KERNEL
#define SQ_REPLAY_IN_KERNEL 0
#endif
// Child order by warp vote (1) in the certified near-first walk: the lanes
// that open the same record with both children hit take the order most of
// them prefer (a __match_any_sync group and a ballot), so lanes that agree
// on a node stay on the same path; 0 (the default): each lane's own nearer
// child first (WALK = 2 builds it as SQ_LAYOUT_BINARY_VOTE). Measured on the
// terrain's 1,048,576 rays (answers identical):
// 0.652 ms against 0.616 ms for each lane's own order; the vote costs every
// node step, and a lane outvoted takes its farther child first.
#ifndef SQ_WARP_ORDER
#define SQ_WARP_ORDER 0
#endif
constexpr int kMaxStack = 96;  // deepest tree accepted (96 KB of stack per block)

template <int D> struct NodeLayout {
  static constexpr int words = 4 * D + 2;  // a.lo a.hi b.lo b.hi code_a code_b
  static constexpr int vec = (words + 3) / 4;
};

// Four-wide records (the binary tree with every other level folded into its
// parent): up to four children's boxes, then their codes (kNoHit: an empty
// slot). Same boxes as the binary records, so the walk prunes exactly the
// subtrees the binary walk would, in half the dependent fetches.
template <int D> struct WideLayout {
  static constexpr int words = 8 * D + 4;  // c0.lo c0.hi ... c3.lo c3.hi code0 .. code3
  static constexpr int vec = (words + 3) / 4;
};

// Quantised four-wide records: the same four-wide tree (same numbering and
// codes), each child's box stored as 8-bit steps from the record's origin
// (the lower corner of the union of its children) in a power-of-two step per
// axis, rounded outward: a stored box always contains the exact one, so its
// slab entry is never later and the walk never prunes a subtree the exact
// boxes would keep (it may visit a few more; answers are certified as for
// every near-first walk). Words: origin[D] (f32), the D step exponents
// (biased by 127, one byte each), the 8 x D step counts (child k, axis i: lo
// at byte 2Dk + i, hi at byte 2Dk + D + i), then the four codes.
template <int D> struct QuantLayout {
  static constexpr int exp_words = (D + 3) / 4;
  static constexpr int o_exp = D;
  static constexpr int o_q = D + exp_words;
  static constexpr int o_code = D + exp_words + 2 * D;
  static constexpr int words = o_code + 4;
  static constexpr int vec = (words + 3) / 4;
};

// origin + q x 2^e, in the arithmetic both the quantiser and the walk use.
__host__ __device__ __forceinline__ float q_decode(float origin, uint32_t q, float step) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(origin, __fmul_rn(float(q), step));
#else
  volatile float m = float(q) * step;  // exact: q < 256 and step a power of two
  return origin + m;
#endif
}

__host__ __device__ __forceinline__ float q_step(uint32_t biased) {
  union { uint32_t u; float f; } v;
  v.u = biased << 23;
  return v.f;
}

__host__ __device__ __forceinline__ uint32_t q_byte(const uint32_t* words, int index) {
  return (words[index >> 2] >> (8 * (index & 3))) & 0xFFu;
}

// Quantises one four-wide record: lo/hi of child k at box + 2Dk, codes[k]
// (kNoHit: an empty slot). Writes QuantLayout<D>::words words. Non-finite
// bounds give a record of zeros (the walk reads the exact records of a scene
// with non-finite bounds).
template <int D>
__host__ __device__ void quantize_record(const float* box, const uint32_t* codes, uint32_t* out) {
  using QL = QuantLayout<D>;
  for (int w = 0; w < QL::words; ++w) out[w] = 0u;
  for (int k = 0; k < 4; ++k) out[QL::o_code + k] = codes[k];
  float plo[D], phi[D];
  bool finite = true, any = false;
  for (int i = 0; i < D; ++i) {
    plo[i] = 3.4028235e38f;
    phi[i] = -3.4028235e38f;
  }
  for (int k = 0; k < 4; ++k) {
    if (codes[k] == kNoHit) continue;
    any = true;
    for (int i = 0; i < D; ++i) {
      const float lo = box[2 * D * k + i], hi = box[2 * D * k + D + i];
      finite = finite && (lo - lo == 0.f) && (hi - hi == 0.f);  // false for inf and NaN
      plo[i] = lo < plo[i] ? lo : plo[i];
      phi[i] = hi > phi[i] ? hi : phi[i];
    }
  }
  if (!finite || !any) return;
  union { float f; uint32_t u; } cv;
  for (int i = 0; i < D; ++i) {
    cv.f = plo[i];
    out[i] = cv.u;
    // the smallest step whose 255th multiple reaches the upper corner
    uint32_t e = 1;  // biased exponent 1..254
    const float ext = phi[i] - plo[i];
    if (ext > 0.f) {
      cv.f = ext;
      const int ex = int((cv.u >> 23) & 0xFFu) - 127;  // ext in [2^ex, 2^(ex+1)) for normal ext
      int b = ex - 7 + 127;  // 255 x 2^(ex-7) < 2^(ex+1): start just below
      b = b < 1 ? 1 : (b > 254 ? 254 : b);
      e = uint32_t(b);
      while (e < 254 && q_decode(plo[i], 255u, q_step(e)) < phi[i]) ++e;
      while (e > 1 && q_decode(plo[i], 255u, q_step(e - 1)) >= phi[i]) --e;
    }
    out[QL::o_exp + (i >> 2)] |= e << (8 * (i & 3));
    const float step = q_step(e);
    for (int k = 0; k < 4; ++k) {
      if (codes[k] == kNoHit) continue;
      const float lo = box[2 * D * k + i], hi = box[2 * D * k + D + i];
      // lo: the largest q whose decoded value is <= lo (q = 0 decodes to the origin <= lo)
      float fq = (lo - plo[i]) / step;
      uint32_t ql = fq <= 0.f ? 0u : (fq >= 255.f ? 255u : uint32_t(fq));
      while (ql > 0 && q_decode(plo[i], ql, step) > lo) --ql;
      while (ql < 255 && q_decode(plo[i], ql + 1, step) <= lo) ++ql;
      // hi: the smallest q whose decoded value is >= hi (q = 255 reaches the upper corner)
      fq = (hi - plo[i]) / step;
      uint32_t qh = fq <= 0.f ? 0u : (fq >= 255.f ? 255u : uint32_t(fq));
      while (qh < 255 && q_decode(plo[i], qh, step) < hi) ++qh;
      while (qh > ql && q_decode(plo[i], qh - 1, step) >= hi) --qh;
      const int bl = 2 * D * k + i, bh = 2 * D * k + D + i;
      out[QL::o_q + (bl >> 2)] |= ql << (8 * (bl & 3));
      out[QL::o_q + (bh >> 2)] |= qh << (8 * (bh & 3));
    }
  }
}

template <int D, int N> struct PrimLayout {
  static constexpr int payload = (N == kNarrowAabb)     ? 2 * D
                                 : (N == kNarrowTri)    ? 9
                                 : (N == kNarrowCustom) ? SQ_CUSTOM_STRIDE + 2 * D
                                                        : D + 1;
  static constexpr int id_word = payload;
  static constexpr int vec = (payload + 1 + 3) / 4;
};

template <int K> struct QueryLayout {
  // floats per query record: rays o,d; casts o,d,probe.min,probe.max; regions lo,hi
};

struct QueryParams {
  const float4* __restrict__ nodes;
  const float4* __restrict__ wnodes;  // four-wide records (WIDE kernels)
  const float4* __restrict__ qnodes;  // quantised four-wide records (QUANT kernels; same numbering)
  uint32_t wroot;                     // the root's four-wide code
  const float4* __restrict__ prims;
  const uint64_t* __restrict__ layers;
  const uint32_t* __restrict__ sub;
  const float* __restrict__ queries;
  const float* __restrict__ max_toi_arr;
  uint32_t* counter;
  uint32_t* out_leaf;
  float* out_toi;
  uint32_t* out_sub;
  float* out_normal;
  float* out_point;
  uint32_t* out_count;
  const unsigned long long* csr_offsets;
  uint32_t* csr_leaves;
  unsigned long long* stats;
  uint32_t* query_stats;  // optional per-query counters [n][4] (u32)
  uint32_t* replay_count;  // near-first: number of uncertified queries appended to replay_list
  uint32_t* replay_list;   // near-first: their indices
  const uint32_t* q_list;  // optional: work item i is query q_list[i] ...
  const uint32_t* q_count; // ... for i < *q_count (the reference-order replay of replay_list)
  float window;            // relative window past the limit within which near-first still visits nodes
  unsigned long long mask;
  long long exclude;
  const float* root_box;  // min[D], max[D] of the root (device memory: refit updates it)
  const int32_t* seed_bucket;  // learned guide: predicted bucket per query (seeded launches)
  const uint2* buckets;        // per bucket: node code, parent record << 1 | slot (kNoHit: the root)
  const uint32_t* bucket_sibs; // per bucket, sib_stride slots (record << 1 | slot) of its ancestors' other children
  uint32_t n_buckets;
  uint32_t sib_stride;
  const int* nonfinite;   // non-zero when some node bound is not finite (device memory)
  float max_toi;
  int stack;              // traversal-stack entries per thread (dynamic shared memory)
  uint32_t root_code;
  uint32_t n;
  uint32_t k;
  int crossings;
  int fill;  // overlap: 0 count, 1 fill in ascending order, 2 fill in walk order
  int far_first;  // seeded walks: after the bucket, the crate's child order (push a, push b) instead of near-first
  // Overlap regions that visit more than visit_budget records in the count
  // pass are left to overlap_heavy_kernel (a block per region): listed in
  // heavy_list, flagged in heavy_flag (1; the fill pass skips them). With
  // keep set, the regions counted with more than kOverlapKeep results are
  // listed too (flag 2) and filled by that kernel alone.
  uint32_t* heavy_list;
  uint32_t* heavy_count;
  uint8_t* heavy_flag;
  uint32_t visit_budget;
  // Overlap: the count pass writes each region's first kOverlapKeep accepted
  // leaves here ([n][kOverlapKeep]); the fill pass copies, sorted, the
  // segment of every region with no more results instead of walking it again.
  uint32_t* keep;
  // Overlap: overlap_heavy_kernel's staged leaves (see that kernel).
  uint32_t* heavy_store;
  uint32_t* heavy_start;   // per heavy_list entry
  uint32_t* heavy_cursor;
  uint32_t heavy_cap;      // entries of heavy_store
};

__device__ __forceinline__ bool accepts(const QueryParams& p, uint32_t id) {
  if (!p.layers) return true;
  if (p.exclude >= 0 && (unsigned long long)p.exclude == id) return false;
  return (__ldg(p.layers + id) & p.mask) != 0ull;
}

template <int NV> __device__ __forceinline__ void load_vec(const float4* __restrict__ src, float* dst) {
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    float4 v = __ldg(src + j);
    dst[4 * j + 0] = v.x;
    dst[4 * j + 1] = v.y;
    dst[4 * j + 2] = v.z;
    dst[4 * j + 3] = v.w;
  }
}

// Near-first traversal visits nodes in another order than the reference, so
// its answer is certified before it counts. The reference's limit never
// drops below the global minimum hit h, and every box enclosing h's
// primitive has a slab entry no later than the entry of the primitive's own
// AABB; so when h.toi is not before that entry, the reference's walk reaches
// h whatever its order and answers h. Near-first prunes a node only when its
// entry lies past the best hit by more than a small relative window (2^-16 by
// default), which finds h whenever no hit is computed that far before the
// entry of a box enclosing its primitive. A query whose answer comes before
// its own primitive's AABB entry is not certified: it is appended to a list
// that a second launch answers again in the reference order.
__device__ __forceinline__ float near_limit(float limit, float window) {
  return __fadd_rn(limit, __fadd_rn(__fmul_rn(fabsf(limit), window), 0x1p-20f));
}

// The slab entry of a primitive's own AABB for a ray or sweep (computed only
// when the primitive is hit): a hit before it is a hit before every box that
// encloses the primitive.
template <int D, int N, bool CAST>
__device__ __forceinline__ float prim_entry(const float* rec, const RayPre<D>& r, const float* pmin, const float* pmax,
                                            bool fast) {
  float lo[D], hi[D], te;
  int ax;
  const float inf = __int_as_float(0x7f800000);
  if constexpr (N == kNarrowTri) {
    tri_aabb(rec, rec + 3, rec + 6, lo, hi);
  } else if constexpr (N == kNarrowCustom) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      lo[i] = rec[SQ_CUSTOM_STRIDE + i];
      hi[i] = rec[SQ_CUSTOM_STRIDE + D + i];
    }
  } else if constexpr (N == kNarrowSphere || N == kNarrowSphereNear) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      lo[i] = fsub(rec[i], rec[D]);
      hi[i] = fadd(rec[i], rec[D]);
    }
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      lo[i] = rec[i];
      hi[i] = rec[D + i];
    }
  }
  if constexpr (CAST) {
    if (fast) slab_grown_fast<D>(r, lo, hi, pmin, pmax, inf, te);
    else slab_grown<D>(r, lo, hi, pmin, pmax, inf, te, ax);
  } else {
    if (fast) slab_fast<D>(r, lo, hi, inf, te);
    else slab<D>(r, lo, hi, inf, te, ax);
  }
  return te;
}

// One primitive's ray test (QueryGeometry::test_ray for the built-in providers).
template <int D, int N>
__device__ __forceinline__ bool narrow_ray(const float* rec, const RayPre<D>& r, float max_toi, float& t, float* n) {
  if constexpr (N == kNarrowAabb) {
    int axis;
    if (!slab<D>(r, rec, rec + D, max_toi, t, axis)) return false;
    entry_normal<D>(r.d, axis, n);
    return true;
  } else if constexpr (N == kNarrowSphere || N == kNarrowSphereNear) {
    return ray_ball<D, N == kNarrowSphere>(r.o, r.d, rec, rec[D], max_toi, t, n);
  } else if constexpr (N == kNarrowCustom) {
#ifdef SQ_RTC_CUSTOM
    const uint32_t leaf = __float_as_uint(rec[PrimLayout<D, N>::id_word]) & ~kLeafBit;
    if (!sq_narrow(rec, leaf, r.o, r.d, max_toi, &t, n)) return false;
    return !(t > max_toi);
#else
    return false;
#endif
  } else {
    if (!ray_triangle(r.o, r.d, rec, rec + 3, rec + 6, t)) return false;
    if (t > max_toi) return false;
    tri_normal(rec, rec + 3, rec + 6, n);
    return true;
  }
}

// One primitive's swept-probe test (QueryGeometry::test_shape_cast).
template <int D, int N>
__device__ __forceinline__ bool narrow_cast(const float* rec, const RayPre<D>& r, const float* pmin, const float* pmax,
                                            float max_toi, float& t, float* n) {
  if constexpr (N == kNarrowAabb) {
    int axis;
    if (!slab_grown<D>(r, rec, rec + D, pmin, pmax, max_toi, t, axis)) return false;
    entry_normal<D>(r.d, axis, n);
    return true;
  } else if constexpr (N == kNarrowSphere || N == kNarrowSphereNear) {
    return ray_ball<D, N == kNarrowSphere>(r.o, r.d, rec, fadd(rec[D], pmax[0]), max_toi, t, n);
  } else {
    float lo[3], hi[3];
    tri_aabb(rec, rec + 3, rec + 6, lo, hi);
    int axis;
    if (!slab_grown<3>(r, lo, hi, pmin, pmax, max_toi, t, axis)) return false;
    entry_normal<3>(r.d, axis, n);
    return true;
  }
}

// One primitive's overlap test (QueryGeometry::test_overlap): the box itself,
// point_to_aabb <= radius for balls (tests/shape_overlap.rs:59-72,113-115),
// the triangle's AABB for triangles.
template <int D, int N>
__device__ __forceinline__ bool narrow_overlap(const float* rec, const float* qlo, const float* qhi) {
  if constexpr (N == kNarrowAabb) {
    return box_overlap<D>(rec, rec + D, qlo, qhi);
  } else if constexpr (N == kNarrowSphere || N == kNarrowSphereNear) {
    float d2 = 0.f;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      float c = rec[i];
      float v = (c < qlo[i]) ? fsub(qlo[i], c) : ((c > qhi[i]) ? fsub(c, qhi[i]) : 0.f);
      d2 = fadd(d2, fmul(v, v));
    }
    return fsqrt(d2) <= rec[D];
  } else {
    float lo[3], hi[3];
    tri_aabb(rec, rec + 3, rec + 6, lo, hi);
    return box_overlap<3>(lo, hi, qlo, qhi);
  }
}

// Sorted insertion into query q's bounded hit list (hit_ordering, stable:
// an equal key goes after the entries already present). `count` is the full
// number of hits so far; the first min(count, k) entries are kept.
template <int D>
__device__ __forceinline__ void list_put(uint32_t k, uint32_t* o_leaf, float* o_toi, uint32_t* o_sub, float* o_nrm,
                                         uint32_t q, uint32_t& count, float t, uint32_t leaf, uint32_t subv,
                                         const float* n) {
  uint32_t m = count < k ? count : k;
  ++count;
  if (k == 0) return;
  const size_t base = size_t(q) * k;
  if (m == k) {
    if (!hit_before(t, leaf, o_toi[base + k - 1], o_leaf[base + k - 1])) return;
    m = k - 1;
  }
  uint32_t j = m;
  while (j > 0 && hit_before(t, leaf, o_toi[base + j - 1], o_leaf[base + j - 1])) {
    o_toi[base + j] = o_toi[base + j - 1];
    o_leaf[base + j] = o_leaf[base + j - 1];
    if (o_sub) o_sub[base + j] = o_sub[base + j - 1];
    if (o_nrm)
#pragma unroll
      for (int i = 0; i < D; ++i) o_nrm[(base + j) * D + i] = o_nrm[(base + j - 1) * D + i];
    --j;
  }
  o_toi[base + j] = t;
  o_leaf[base + j] = leaf;
  if (o_sub) o_sub[base + j] = subv;
  if (o_nrm)
#pragma unroll
    for (int i = 0; i < D; ++i) o_nrm[(base + j) * D + i] = n[i];
}

template <int D>
__device__ __forceinline__ void list_insert(const QueryParams& p, uint32_t q, uint32_t& count, float t, uint32_t leaf,
                                            const float* n) {
  list_put<D>(p.k, p.out_leaf, p.out_toi, p.out_sub, p.out_normal, q, count, t, leaf,
              p.sub ? __ldg(p.sub + leaf) : kNoHit, n);
}

// Per-lane traversal state of one query.
template <int D, int K> struct Lane {
  RayPre<D> r;
  float pmin[D], pmax[D];
  float limit;       // nodes whose entry lies past this are pruned (near-first: the best hit plus the window)
  uint32_t best_pos; // near-first: primitive position of the best hit (for its certification)
  uint32_t q;
  uint32_t code;
  float code_t;      // entry of the node in code (postponed-leaf walks re-check it after a leaf)
  uint32_t top_code; // postponed-leaf walks: the stack's top entry, held in registers
  float top_t;
  bool has_top;
  bool ref;          // this walk answers the query again in the crate's own order (unseeded, exact limit)
  int sp;
  bool fast;
  uint32_t best_leaf;
  float best_t;
  float best_n[D];
  uint32_t count;
  unsigned long long csr_base;
  uint32_t v_nodes, v_nar, v_hit;
};

// The persistent query kernel. Each warp keeps 32 queries in flight; a lane
// whose query finishes takes the next one from the shared counter at the top
// of the loop (one atomic per warp per refill), so a warp never idles on its
// slowest query. Between refills a lane descends interior records until it
// reaches a leaf, tests that leaf's primitives and pops the next waiting
// child (Aila and Laine's while-while loop with dynamic fetch).
//
// SEED (nearest rays only): the learned guide's predicted bucket, a subtree
// at a fixed depth, is searched first; its nearest hit becomes the limit for
// the rest of the tree, which is exactly the other children of the bucket's
// ancestors: they wait on the stack from the start and are walked after the
// bucket (no ancestor's record is read twice, so a right seed never costs
// more box tests than the plain walk). The answer is certified exactly as in
// near-first, so it is the reference's whatever the seed.
// WIDE (near-first nearest rays, no counters, no seed): the walk reads the
// four-wide records; a step tests up to four children, goes to the nearest
// and stacks the others farthest first.
// WALK (near-first nearest rays over child-pair records, no counters): 1 =
// postponed leaves with the stack's top entry held in registers; 2 = child
// order by warp vote.
template <int D, int N, int K, bool REF, bool STATS, bool SEED = false, bool WIDE = false, bool QUANT = false,
          int WALK = 0>
__global__ void __launch_bounds__(kThreads) query_kernel(const QueryParams p) {
  static_assert(!WIDE || (K == kRayNearest && !REF && !STATS && !SEED), "four-wide walks serve near-first rays only");
  static_assert(!QUANT || WIDE, "quantised records are a four-wide layout");
  constexpr bool kNearest = (K == kRayNearest || K == kCastNearest);
  constexpr bool kCast = (K == kCastNearest || K == kCastAll);
  constexpr bool kList = (K == kRayAll || K == kCastAll);
  constexpr int QW = kCast ? 4 * D : 2 * D;
  using PL = PrimLayout<D, N>;
  using NL = NodeLayout<D>;
  using WL = WideLayout<D>;
  constexpr uint32_t FULL = 0xffffffffu;

  extern __shared__ uint32_t smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int S = p.stack;
  uint32_t* s_code = smem;
  float* s_t = reinterpret_cast<float*>(smem + S * kThreads);
  const uint32_t lt_mask = (1u << lane) - 1u;
  const bool scene_finite = p.nonfinite ? (*p.nonfinite == 0) : true;

  unsigned long long c_vis = 0, c_nar = 0, c_hit = 0;
  Lane<D, K> L;
  bool live = false, exhausted = false;
  const uint32_t n_queries = p.q_count ? *p.q_count : p.n;

  constexpr bool DETECT = kNearest && !REF;
  // Postponed leaves for the certified near-first walks (their answers do
  // not depend on the order of the visits); the counting and reference-order
  // walks keep the crate's sequence.
  constexpr bool SPEC = (SQ_POSTPONE_LEAVES || WALK == 1) && DETECT && !STATS && !WIDE;
  constexpr bool kRegTop = SQ_REG_TOP || WALK == 1;
  // An uncertified answer is answered again by the same lane, in the crate's
  // order over the child-pair records, at its next refill (no second launch
  // walking a handful of rays while the GPU idles). Four-wide walks list
  // such queries for a reference-order launch over the child-pair records.
  constexpr bool INREPLAY = SQ_REPLAY_IN_KERNEL && DETECT && !WIDE && !SPEC;
  bool pending = false;
  uint32_t pending_q = 0;
  const float kInf = __int_as_float(0x7f800000);

  // Box test of one child (or the root) against the lane's query: the slab
  // without the limit, then the entry against the limit (the same verdict as
  // the reference's slab clipped to the limit, aabb.rs:118-148).
  auto test_box = [&](const float* lo, const float* hi, float& te) -> bool {
    if constexpr (K == kOverlap) {
      te = 0.f;
      return box_overlap<D>(lo, hi, L.r.o, L.r.d);  // region lo / hi sit in o / d
    } else {
      bool geo;
      int ax;
      if constexpr (kCast) {
        geo = L.fast ? slab_grown_fast<D>(L.r, lo, hi, L.pmin, L.pmax, kInf, te)
                     : slab_grown<D>(L.r, lo, hi, L.pmin, L.pmax, kInf, te, ax);
      } else {
        geo = L.fast ? slab_fast<D>(L.r, lo, hi, kInf, te) : slab<D>(L.r, lo, hi, kInf, te, ax);
      }
      return geo && te <= L.limit;
    }
  };

  // Pops the next waiting child whose entry still lies within the limit
  // (exactly the reference's slab verdict at pop time). False: stack empty.
  auto pop = [&]() -> bool {
    if constexpr (SPEC && kRegTop) {
      if (L.has_top) {
        L.has_top = false;
        L.code = L.top_code;
        L.code_t = L.top_t;
        if (L.top_t <= L.limit) return true;
      }
    }
    while (L.sp > 0) {
      --L.sp;
      L.code = s_code[L.sp * kThreads + tid];
      const float t = s_t[L.sp * kThreads + tid];
      L.code_t = t;
      if (!kNearest || t <= L.limit) return true;
    }
    return false;
  };

  auto finish = [&]() {
    const uint32_t q = L.q;
    if constexpr (DETECT && N != kNarrowAabb) {
      // Certify the answer: not before its own primitive's AABB entry.
      if (L.best_leaf != kNoHit && !L.ref) {
        float rec[PL::vec * 4];
        load_vec<PL::vec>(p.prims + size_t(L.best_pos) * PL::vec, rec);
        if (L.best_t < prim_entry<D, N, kCast>(rec, L.r, L.pmin, L.pmax, L.fast)) {
          if constexpr (INREPLAY) {
            // Answered again by this lane in the crate's order; this walk's
            // counters still count, its answer is not written.
            pending = true;
            pending_q = q;
            if (p.replay_count) atomicAdd(p.replay_count, 1u);
            if (STATS) {
              c_vis += L.v_nodes;
              c_nar += L.v_nar;
              c_hit += L.v_hit;
            }
            return;
          } else {
            p.replay_list[atomicAdd(p.replay_count, 1u)] = q;
          }
        }
      }
    }
    if constexpr (kNearest) {
      p.out_leaf[q] = L.best_leaf;
      if (p.out_toi) p.out_toi[q] = L.best_t;
      if (p.out_sub) p.out_sub[q] = (L.best_leaf != kNoHit && p.sub) ? __ldg(p.sub + L.best_leaf) : kNoHit;
      if (p.out_normal) {
#pragma unroll
        for (int i = 0; i < D; ++i) p.out_normal[size_t(q) * D + i] = L.best_n[i];
      }
      if (p.out_point) {
        float pt[D];
        if (L.best_leaf != kNoHit) {
          ray_at<D>(L.r.o, L.r.d, L.best_t, pt);
        } else {
#pragma unroll
          for (int i = 0; i < D; ++i) pt[i] = 0.f;
        }
#pragma unroll
        for (int i = 0; i < D; ++i) p.out_point[size_t(q) * D + i] = pt[i];
      }
    } else if constexpr (kList) {
      p.out_count[q] = L.count;  // entries past min(count, k) are left as they were
    } else {
      if (!p.fill) {
        p.out_count[q] = L.count;
        // A counted region with more results than the kept leaves (and not
        // given up on) is filled by the block-per-region kernel too, so the
        // fill pass walks no region again on one lane (flag 2: counted).
        if (p.heavy_list && p.keep && L.count > kOverlapKeep && L.v_nar <= p.visit_budget) {
          p.heavy_flag[q] = 2;
          p.heavy_list[atomicAdd(p.heavy_count, 1u)] = q;
        }
      }
    }
    if (STATS) {
      c_vis += L.v_nodes;
      c_nar += L.v_nar;
      c_hit += L.v_hit;
      if (p.query_stats) {
        p.query_stats[size_t(q) * 4 + 0] = L.v_nodes;
        p.query_stats[size_t(q) * 4 + 1] = L.v_nodes;
        p.query_stats[size_t(q) * 4 + 2] = L.v_nar;
        p.query_stats[size_t(q) * 4 + 3] = L.v_hit;
      }
    }
  };

  // Loads query q and tests the root. False when the query is already done.
  auto start = [&](uint32_t q, bool ref) -> bool {
    L.q = q;
    L.ref = ref;
    const float* src = p.queries + size_t(q) * QW;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      L.r.o[i] = src[i];
      L.r.d[i] = src[D + i];
      if constexpr (kCast) {
        L.pmin[i] = src[2 * D + i];
        L.pmax[i] = src[3 * D + i];
      }
    }
    L.limit = p.max_toi_arr ? p.max_toi_arr[q] : p.max_toi;
    if constexpr (K != kOverlap) {
      ray_prep<D>(L.r);
      bool f = scene_finite && L.r.par == 0u && !isnan(L.limit);
#pragma unroll
      for (int i = 0; i < D; ++i) {
        f = f && isfinite(L.r.o[i]) && isfinite(L.r.d[i]);
        if constexpr (kCast) f = f && isfinite(L.pmin[i]) && isfinite(L.pmax[i]);
      }
      L.fast = f;
    } else {
      L.fast = false;
    }
    L.best_leaf = kNoHit;
    L.best_t = 0.f;
#pragma unroll
    for (int i = 0; i < D; ++i) L.best_n[i] = 0.f;
    L.count = 0;
    L.csr_base = 0;
    if constexpr (K == kOverlap) {
      if (p.fill) L.csr_base = p.csr_offsets[q];
      if (p.fill && p.heavy_flag && p.heavy_flag[q]) return false;  // filled by the block-per-region kernel
      if (p.fill && p.keep) {
        // Every result of a region with at most kOverlapKeep of them was kept
        // by the count pass (the same walk finds the same leaves): written
        // ascending, with no second walk. Most regions have none.
        const uint32_t c = uint32_t(p.csr_offsets[q + 1] - L.csr_base);
        if (c <= kOverlapKeep) {
          if (c) {
            const uint4 k4 = __ldcs(reinterpret_cast<const uint4*>(p.keep) + q);
            uint32_t v0 = k4.x, v1 = c > 1 ? k4.y : kNoHit, v2 = c > 2 ? k4.z : kNoHit, v3 = c > 3 ? k4.w : kNoHit;
            const auto cas = [](uint32_t& a, uint32_t& b) {
              const uint32_t lo = min(a, b);
              b = max(a, b);
              a = lo;
            };
            cas(v0, v1);  // sorting network on four: (0,1) (2,3) (0,2) (1,3) (1,2)
            cas(v2, v3);
            cas(v0, v2);
            cas(v1, v3);
            cas(v1, v2);
            uint32_t* out = p.csr_leaves + L.csr_base;
            out[0] = v0;
            if (c > 1) out[1] = v1;
            if (c > 2) out[2] = v2;
            if (c > 3) out[3] = v3;
          }
          return false;
        }
      }
    }
    L.v_nodes = STATS ? 1u : 0u;
    L.v_nar = 0;
    L.v_hit = 0;
    L.sp = 0;
    L.has_top = false;
    L.code = WIDE ? p.wroot : p.root_code;
    float lo[D], hi[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      lo[i] = p.root_box[i];
      hi[i] = p.root_box[D + i];
    }
    float te;
    const bool hit_root = test_box(lo, hi, te);
    L.code_t = te;
    if constexpr (SEED) if (!L.ref) {
      const int32_t bk = p.seed_bucket[q];
      if (hit_root && bk >= 0 && uint32_t(bk) < p.n_buckets) {
        const uint2 e = __ldg(p.buckets + bk);
        if (e.x != p.root_code) {
          const float* box = (e.y == kNoHit) ? p.root_box
                                             : reinterpret_cast<const float*>(p.nodes + size_t(e.y >> 1) * NL::vec) +
                                                   (e.y & 1u) * 2 * D;
          float blo[D], bhi[D], tb;
#pragma unroll
          for (int i = 0; i < D; ++i) {
            blo[i] = box[i];
            bhi[i] = box[D + i];
          }
          if (STATS) L.v_nodes += 1;
          if (test_box(blo, bhi, tb)) {
            // The bucket goes first. The siblings of its ancestors wait on
            // the stack, the root's child deepest, so the bucket's nearest
            // neighbours in the tree come up first; each is tested against
            // the ray now and against the (shrunk) limit when popped. Their
            // records are independent loads, not a dependent descent.
            const uint32_t* sibs = p.bucket_sibs + size_t(bk) * p.sib_stride;
            for (uint32_t i = 0; i < p.sib_stride; ++i) {
              const uint32_t sl = __ldg(sibs + i);
              if (sl == kNoHit) break;
              float rec[NL::vec * 4];
              load_vec<NL::vec>(p.nodes + size_t(sl >> 1) * NL::vec, rec);
              const bool second = (sl & 1u) != 0u;
              float slo[D], shi[D];
#pragma unroll
              for (int k = 0; k < D; ++k) {
                slo[k] = second ? rec[2 * D + k] : rec[k];
                shi[k] = second ? rec[3 * D + k] : rec[D + k];
              }
              const uint32_t sc = __float_as_uint(second ? rec[4 * D + 1] : rec[4 * D]);
              float ts;
              if (STATS) L.v_nodes += 1;
              if (test_box(slo, shi, ts)) {
                s_code[L.sp * kThreads + tid] = sc;
                s_t[L.sp * kThreads + tid] = ts;
                ++L.sp;
              }
            }
            L.code = e.x;
            L.code_t = tb;
          }
        }
      }
    }
    return hit_root;
  };

  // Tests the primitives of the leaf in L.code.
  auto leaf = [&](uint32_t code) {
    uint32_t pos = code & ~kLeafBit;
    for (;;) {
      float rec[PL::vec * 4];
      load_vec<PL::vec>(p.prims + size_t(pos) * PL::vec, rec);
      const uint32_t idw = __float_as_uint(rec[PL::id_word]);
      const uint32_t id = idw & ~kLeafBit;
      if (accepts(p, id)) {
        if constexpr (K == kOverlap) {
          if (narrow_overlap<D, N>(rec, L.r.o, L.r.d)) {
            if (!p.fill && p.keep && L.count < kOverlapKeep) p.keep[size_t(L.q) * kOverlapKeep + L.count] = id;
            if (p.fill == 2) {
              // appended in walk order; a segmented sort orders each segment afterwards
              p.csr_leaves[L.csr_base + L.count] = id;
            } else if (p.fill) {
              // ascending leaf order within the query's CSR segment, kept by
              // insertion (the allocation-free path, which has no sort scratch)
              uint32_t j = L.count;
              while (j > 0 && p.csr_leaves[L.csr_base + j - 1] > id) {
                p.csr_leaves[L.csr_base + j] = p.csr_leaves[L.csr_base + j - 1];
                --j;
              }
              p.csr_leaves[L.csr_base + j] = id;
            }
            ++L.count;
          }
        } else {
          if (STATS) L.v_nar += 1;
          float t, nrm[D];
          if constexpr (K == kRayNearest || K == kCastNearest) {
            bool h;
            if constexpr (K == kRayNearest) h = narrow_ray<D, N>(rec, L.r, L.limit, t, nrm);
            else h = narrow_cast<D, N>(rec, L.r, L.pmin, L.pmax, L.limit, t, nrm);
            if (h) {
              if (STATS) L.v_hit += 1;
              if (L.best_leaf == kNoHit || hit_before(t, id, L.best_t, L.best_leaf)) {
                L.best_leaf = id;
                L.best_t = t;
                if (DETECT && !L.ref) {
                  L.limit = near_limit(t, p.window);
                  L.best_pos = pos;
                } else {
                  L.limit = t;
                }
#pragma unroll
                for (int i = 0; i < D; ++i) L.best_n[i] = nrm[i];
              }
            }
          } else if constexpr (K == kRayAll) {
            if constexpr (N == kNarrowSphere) {
              if (p.crossings) {
                // Both roots of the unbounded ray (tests/crossings.rs:505-521).
                float oc[D];
#pragma unroll
                for (int i = 0; i < D; ++i) oc[i] = fsub(L.r.o[i], rec[i]);
                const float b = pdot<D>(oc, L.r.d);
                const float disc = fsub(fmul(b, b), fsub(pdot<D>(oc, oc), fmul(rec[D], rec[D])));
                if (!(disc < 0.f)) {
                  const float sq = fsqrt(disc);
                  const float roots[2] = {fsub(-b, sq), fadd(-b, sq)};
#pragma unroll
                  for (int j = 0; j < 2; ++j) {
                    const float tt = roots[j];
                    if (tt >= 0.f && tt <= L.limit) {
                      float pt[D];
                      ray_at<D>(L.r.o, L.r.d, tt, pt);
#pragma unroll
                      for (int i = 0; i < D; ++i) nrm[i] = fsub(pt[i], rec[i]);
                      normalize_or_zero<D>(nrm);
                      if (STATS) L.v_hit += 1;
                      list_insert<D>(p, L.q, L.count, tt, id, nrm);
                    }
                  }
                }
              } else if (narrow_ray<D, N>(rec, L.r, L.limit, t, nrm)) {
                if (STATS) L.v_hit += 1;
                list_insert<D>(p, L.q, L.count, t, id, nrm);
              }
            } else {
              bool listed = false;
#ifdef SQ_RTC_CROSSINGS
              if constexpr (N == kNarrowCustom) {
                if (p.crossings) {
                  // Every crossing the consumer emits is listed, as bvh.rs:309-315 pushes them.
                  auto emit = [&](float tt, const float* nn) {
                    if (STATS) L.v_hit += 1;
                    list_insert<D>(p, L.q, L.count, tt, id, nn);
                  };
                  sq_narrow_crossings(rec, id, L.r.o, L.r.d, L.limit, emit);
                  listed = true;
                }
              }
#endif
              if (!listed && narrow_ray<D, N>(rec, L.r, L.limit, t, nrm)) {
                if (STATS) L.v_hit += 1;
                list_insert<D>(p, L.q, L.count, t, id, nrm);
              }
            }
          } else {  // kCastAll
            if (narrow_cast<D, N>(rec, L.r, L.pmin, L.pmax, L.limit, t, nrm)) list_insert<D>(p, L.q, L.count, t, id, nrm);
          }
        }
      }
      if (idw & kLeafBit) break;
      ++pos;
    }
  };

  for (;;) {
    // Refill the lanes without a query.
    const bool need = !live && !exhausted && !pending;
    const uint32_t need_mask = __ballot_sync(FULL, need);
    uint32_t qs = kNoHit;
    if (need_mask) {
      const int leader = __ffs(need_mask) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(p.counter, uint32_t(__popc(need_mask)));
      base = __shfl_sync(FULL, base, leader);
      if (need) {
        const uint32_t q = base + uint32_t(__popc(need_mask & lt_mask));
        if (q < n_queries) qs = p.q_list ? p.q_list[q] : q;
        else exhausted = true;
      }
    }
    bool replay = false;
    if (INREPLAY && pending) {
      qs = pending_q;
      pending = false;
      replay = true;
    }
    if (qs != kNoHit) {
      live = start(qs, replay);
      if (!live) finish();
    }
    const uint32_t live_mask = __ballot_sync(FULL, live);
    if (!live_mask) {
      if (__all_sync(FULL, exhausted)) break;
      continue;
    }
    if constexpr (SPEC) {
      if (live) {
        // Postponed leaves (Aila and Laine's speculative traversal): a lane
        // that reaches a leaf holds it and keeps descending from the next
        // waiting node until every live lane of the warp holds a leaf or
        // has nothing left, so the leaf tests below run with the warp
        // together. The extra nodes are visited with the limit as it stood,
        // which only adds work: near-first answers are certified whatever
        // the order of the visits.
        uint32_t pend = kNoHit;
        bool empty = false;  // nothing left to walk after pend
        for (;;) {
          if (!empty) {
            if (L.code & kLeafBit) {
              if (pend == kNoHit) {
                pend = L.code;
                if (!pop()) empty = true;
              }
            } else {
              float rec[NL::vec * 4];
              load_vec<NL::vec>(p.nodes + size_t(L.code) * NL::vec, rec);
              const uint32_t ca = __float_as_uint(rec[4 * D]);
              const uint32_t cb = __float_as_uint(rec[4 * D + 1]);
              float ta, tb;
              const bool pa = test_box(rec, rec + D, ta);
              const bool pb = test_box(rec + 2 * D, rec + 3 * D, tb);
              if (pa && pb) {
                const bool a_first = (SEED && p.far_first) ? false : (ta <= tb);
                const uint32_t far_code = a_first ? cb : ca;
                const float far_t = a_first ? tb : ta;
                if constexpr (kRegTop) {
                  if (L.has_top) {  // the register entry spills below the new one
                    s_code[L.sp * kThreads + tid] = L.top_code;
                    s_t[L.sp * kThreads + tid] = L.top_t;
                    ++L.sp;
                  }
                  L.top_code = far_code;
                  L.top_t = far_t;
                  L.has_top = true;
                } else {
                  s_code[L.sp * kThreads + tid] = far_code;
                  s_t[L.sp * kThreads + tid] = far_t;
                  ++L.sp;
                }
                L.code = a_first ? ca : cb;
                L.code_t = a_first ? ta : tb;
              } else if (pa) {
                L.code = ca;
                L.code_t = ta;
              } else if (pb) {
                L.code = cb;
                L.code_t = tb;
              } else if (!pop()) {
                empty = true;
              }
            }
          }
          if (__all_sync(live_mask, pend != kNoHit || empty)) break;
        }
        if (pend != kNoHit) leaf(pend);
        // The node after the leaf was taken with the limit as it stood:
        // drop it (and what follows, as pop does) if the leaf's hit prunes it.
        if (!empty && L.code_t > L.limit && !pop()) empty = true;
        if (empty) {
          live = false;
          finish();
        }
      }
    } else if (live) {
      bool done = false;
      // Descend interior records until a leaf comes up.
      while (!(L.code & kLeafBit)) {
        if constexpr (WIDE) {
          float t4[4];
          uint32_t c4[4];
          bool exact = true;
          if constexpr (QUANT) {
            if (scene_finite) {
              // Decode each child's box (rounded outward) and test it.
              using QL = QuantLayout<D>;
              float qf[QL::vec * 4];
              load_vec<QL::vec>(p.qnodes + size_t(L.code) * QL::vec, qf);
              uint32_t qw[QL::vec * 4];
#pragma unroll
              for (int w = 0; w < QL::vec * 4; ++w) qw[w] = __float_as_uint(qf[w]);
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                c4[k] = qw[QL::o_code + k];
                float lo[D], hi[D];
#pragma unroll
                for (int i = 0; i < D; ++i) {
                  const float step = q_step(q_byte(qw + QL::o_exp, i));
                  lo[i] = q_decode(qf[i], q_byte(qw + QL::o_q, 2 * D * k + i), step);
                  hi[i] = q_decode(qf[i], q_byte(qw + QL::o_q, 2 * D * k + D + i), step);
                }
                float te = kInf;
                if (c4[k] == kNoHit || !test_box(lo, hi, te)) {
                  c4[k] = kNoHit;
                  te = kInf;
                }
                t4[k] = te;
              }
              exact = false;
            }
          }
          if (exact) {
            float rec[WL::vec * 4];
            load_vec<WL::vec>(p.wnodes + size_t(L.code) * WL::vec, rec);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              c4[i] = __float_as_uint(rec[8 * D + i]);
              float te = kInf;
              if (c4[i] == kNoHit || !test_box(rec + 2 * D * i, rec + 2 * D * i + D, te)) {
                c4[i] = kNoHit;
                te = kInf;
              }
              t4[i] = te;
            }
          }
          // Ascending entry order (a five-comparator network); misses sort last.
          auto cswap = [&](int a, int b) {
            if (t4[b] < t4[a]) {
              const float t = t4[a];
              t4[a] = t4[b];
              t4[b] = t;
              const uint32_t c = c4[a];
              c4[a] = c4[b];
              c4[b] = c;
            }
          };
          cswap(0, 1);
          cswap(2, 3);
          cswap(0, 2);
          cswap(1, 3);
          cswap(1, 2);
#pragma unroll
          for (int i = 3; i >= 1; --i) {
            if (c4[i] != kNoHit) {
              s_code[L.sp * kThreads + tid] = c4[i];
              s_t[L.sp * kThreads + tid] = t4[i];
              ++L.sp;
            }
          }
          if (c4[0] != kNoHit) {
            L.code = c4[0];
          } else if (!pop()) {
            done = true;
            break;
          }
          continue;
        }
        float rec[NL::vec * 4];
        load_vec<NL::vec>(p.nodes + size_t(L.code) * NL::vec, rec);
        const uint32_t ca = __float_as_uint(rec[4 * D]);
        const uint32_t cb = __float_as_uint(rec[4 * D + 1]);
        float ta, tb;
        const bool pa = test_box(rec, rec + D, ta);
        const bool pb = test_box(rec + 2 * D, rec + 3 * D, tb);
        if (STATS) L.v_nodes += 2;
        if constexpr (K == kOverlap) {
          // A region heavier than the budget goes to the block-per-region
          // kernel instead of holding the launch's tail on one thread.
          if (p.heavy_list && !p.fill && ++L.v_nar > p.visit_budget) {
            p.heavy_flag[L.q] = 1;
            p.heavy_list[atomicAdd(p.heavy_count, 1u)] = L.q;
            done = true;
            break;
          }
        }
        if (pa && pb) {
          // Reference order: child_a waits, child_b goes first. Near-first:
          // the smaller entry goes first.
          bool a_first = (REF || !kNearest || L.ref || (SEED && p.far_first)) ? false : (ta <= tb);
          if constexpr ((SQ_WARP_ORDER || WALK == 2) && DETECT && !WIDE) {
            const bool voter = !L.ref && !(SEED && p.far_first);
            const uint32_t voters = __ballot_sync(__activemask(), voter);
            if (voter) {
              const uint32_t same = __match_any_sync(voters, L.code);
              const uint32_t yes = __ballot_sync(voters, a_first) & same;
              a_first = 2 * __popc(yes) >= __popc(same);
            }
          }
          s_code[L.sp * kThreads + tid] = a_first ? cb : ca;
          s_t[L.sp * kThreads + tid] = a_first ? tb : ta;
          ++L.sp;
          L.code = a_first ? ca : cb;
        } else if (pa) {
          L.code = ca;
        } else if (pb) {
          L.code = cb;
        } else if (!pop()) {
          done = true;
          break;
        }
      }
      if (!done) {
        leaf(L.code);
        done = !pop();
      }
      if (done) {
        live = false;
        finish();
      }
    }
  }
  if (STATS) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      c_vis += __shfl_down_sync(FULL, c_vis, o);
      c_nar += __shfl_down_sync(FULL, c_nar, o);
      c_hit += __shfl_down_sync(FULL, c_hit, o);
    }
    if (lane == 0 && p.stats) {
      atomicAdd(p.stats + 0, c_vis);
      atomicAdd(p.stats + 1, c_vis);
      atomicAdd(p.stats + 2, c_nar);
      atomicAdd(p.stats + 3, c_hit);
    }
  }
}

// ---------------------------------------------------------------------------
// Heavy overlap regions: one block (128 threads) per region, for the regions
// the count pass gave up on (counted and filled here) and, in the fill pass,
// for those it counted with more results than it kept. The block keeps
// the region's pending nodes in one shared-memory stack and each step takes
// up to 128 of them from the top, one per thread: an interior record's
// overlapping children are pushed (block prefix sum for the slots), a leaf's
// accepted overlapping primitives are counted (count pass) or written to the
// region's CSR segment in any order (fill pass; the segmented sort that
// follows orders them). Any order of visits finds the same set of leaves as
// the crate's walk. (A warp per region left the heaviest region's walk on 32
// lanes: 339 us for the D = 6 mixture's count pass with 5% of warp slots
// busy.) Stack: each step replaces the <= 128 entries it takes with <= 256
// children one level deeper, so at most 128 entries per level stay below the
// top: it never holds more than 128 x (depth + 2) entries; it is sized
// 256 x (depth + 1) (dynamic shared memory), and a push past it is refused
// and reported through heavy_count's high bit instead of written.
// With heavy_store set, the count pass also stages a region's leaves in
// shared memory (up to kHeavyStage) and copies them to heavy_store at a
// slot taken from heavy_cursor (heavy_start[i]: the slot, kNoHit when the
// stage or the store was too small); the fill pass then copies that region's
// segment from there instead of walking it again.
// ---------------------------------------------------------------------------
constexpr int kHeavyWarps = 4;
constexpr uint32_t kHeavyStage = 2048;

template <int D, int N>
__global__ void __launch_bounds__(32 * kHeavyWarps) overlap_heavy_kernel(const QueryParams p) {
  using PL = PrimLayout<D, N>;
  using NL = NodeLayout<D>;
  constexpr uint32_t FULL = 0xffffffffu;
  constexpr int T = 32 * kHeavyWarps;
  extern __shared__ uint32_t stk[];
  __shared__ unsigned long long s_fill;
  __shared__ int s_sp;
  __shared__ int s_wsum[kHeavyWarps];
  __shared__ uint32_t s_n;      // the region's accepted leaves so far
  __shared__ uint32_t s_start;  // its slot in heavy_store (kNoHit: none)
  __shared__ uint32_t s_stage[kHeavyStage];
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int cap = p.stack;  // entries
  const uint32_t nh = *p.heavy_count & 0x7FFFFFFFu;
  for (uint32_t i = blockIdx.x; i < nh; i += gridDim.x) {
    const uint32_t q = p.heavy_list[i];
    if (!p.fill && p.heavy_flag[q] == 2) continue;  // counted by the count pass (uniform per block)
    if (p.fill && p.heavy_start) {
      const uint32_t st = p.heavy_start[i];  // uniform per block
      if (st != kNoHit) {
        // staged by the count pass: a copy, no second walk
        const unsigned long long base = p.csr_offsets[q];
        const uint32_t c = uint32_t(p.csr_offsets[q + 1] - base);
        for (uint32_t k = tid; k < c; k += T) p.csr_leaves[base + k] = p.heavy_store[st + k];
        continue;
      }
    }
    float lo[D], hi[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      lo[k] = p.queries[size_t(q) * 2 * D + k];
      hi[k] = p.queries[size_t(q) * 2 * D + D + k];
    }
    if (tid == 0) {
      s_fill = p.fill ? p.csr_offsets[q] : 0ull;
      s_n = 0;
      const bool in_root = box_overlap<D>(p.root_box, p.root_box + D, lo, hi);
      if (in_root) stk[0] = p.root_code;
      s_sp = in_root ? 1 : 0;
    }
    __syncthreads();
    for (;;) {
      const int sp = s_sp;
      if (sp == 0) break;  // uniform: every thread read the same value
      const int take = sp < T ? sp : T;
      const uint32_t code = tid < take ? stk[sp - take + tid] : kNoHit;
      __syncthreads();  // every entry taken is read before pushes overwrite it
      uint32_t push[2] = {kNoHit, kNoHit};
      if (code != kNoHit) {
        if (code & kLeafBit) {
          uint32_t pos = code & ~kLeafBit;
          for (;;) {
            float rec[PL::vec * 4];
            load_vec<PL::vec>(p.prims + size_t(pos) * PL::vec, rec);
            const uint32_t idw = __float_as_uint(rec[PL::id_word]);
            const uint32_t id = idw & ~kLeafBit;
            if (accepts(p, id) && narrow_overlap<D, N>(rec, lo, hi)) {
              if (p.fill) {
                p.csr_leaves[atomicAdd(&s_fill, 1ull)] = id;
              } else {
                const uint32_t k = atomicAdd(&s_n, 1u);
                if (k < kHeavyStage) s_stage[k] = id;
              }
            }
            if (idw & kLeafBit) break;
            ++pos;
          }
        } else {
          float rec[NL::vec * 4];
          load_vec<NL::vec>(p.nodes + size_t(code) * NL::vec, rec);
          if (box_overlap<D>(rec, rec + D, lo, hi)) push[0] = __float_as_uint(rec[4 * D]);
          if (box_overlap<D>(rec + 2 * D, rec + 3 * D, lo, hi)) push[1] = __float_as_uint(rec[4 * D + 1]);
        }
      }
      // Block prefix sum of the children to push: within each warp, then
      // across the warps' totals.
      const int mine = (push[0] != kNoHit) + (push[1] != kNoHit);
      int incl = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
      }
      if (lane == 31) s_wsum[w] = incl;
      __syncthreads();
      int before = 0, total = 0;
#pragma unroll
      for (int k = 0; k < kHeavyWarps; ++k) {
        const int ws = s_wsum[k];
        if (k < w) before += ws;
        total += ws;
      }
      const int base = sp - take;
      int at = base + before + incl - mine;
      for (int k = 0; k < 2; ++k) {
        if (push[k] == kNoHit) continue;
        if (at < cap) stk[at] = push[k];
        else atomicOr(p.heavy_count, 0x80000000u);  // refused: reported to the host
        ++at;
      }
      __syncthreads();  // pushes written and s_wsum read before the next step
      if (tid == 0) s_sp = min(base + total, cap);
      __syncthreads();
    }
    if (!p.fill) {
      // The walk's last step ended at a barrier: s_n is final.
      const uint32_t c = s_n;
      if (tid == 0) {
        p.out_count[q] = c;
        uint32_t st = kNoHit;
        if (p.heavy_start && c <= kHeavyStage) {
          const uint32_t at = atomicAdd(p.heavy_cursor, c);
          if (at <= p.heavy_cap && c <= p.heavy_cap - at) st = at;
        }
        s_start = st;
        if (p.heavy_start) p.heavy_start[i] = st;
      }
      __syncthreads();
      const uint32_t st = s_start;
      if (st != kNoHit)
        for (uint32_t k = tid; k < c; k += T) p.heavy_store[st + k] = s_stage[k];
    }
    __syncthreads();  // the region's shared state is done before the next region's
  }
}

// ---------------------------------------------------------------------------
// Device refit: tree::refit (accel/tree.rs:54-75) over the fixed topology.
//
// One thread per leaf rewrites its primitives' records from the new leaf
// parameters and unions their boxes into the leaf box, which it stores in the
// parent's child slot. It then climbs: at each interior node an arrival
// counter lets the second of the two children through, which unions the two
// slots of that node's record into its own slot in its parent, and so on to
// the root. Unions are min/max, exact in any order.
// ---------------------------------------------------------------------------

struct RefitLeaf {
  uint32_t first;   // first position in the leaf-ordered primitive array
  uint32_t count;
  uint32_t parent;  // parent interior record << 1 | slot, or kNoHit for the root
  uint32_t pad;
};

struct RefitParams {
  int* nonfinite;  // set when a refit box is not finite
  float4* nodes;
  float4* prims;
  float* root_box;
  const float* prim_data;  // new leaf parameters, indexed by leaf id
  const uint32_t* prim_ids;
  const RefitLeaf* leaves;
  const uint32_t* parents;  // per interior record: parent << 1 | slot, or kNoHit
  uint32_t* arrivals;       // per interior record, zeroed before the launch
  uint32_t n_leaves;
  uint32_t stride;          // floats per leaf parameter block
};

template <int D, int N>
__device__ __forceinline__ void prim_box(const float* v, float* lo, float* hi) {
  if constexpr (N == kNarrowAabb) {
#pragma unroll
    for (int i = 0; i < D; ++i) { lo[i] = v[i]; hi[i] = v[D + i]; }
  } else if constexpr (N == kNarrowSphere || N == kNarrowSphereNear) {
#pragma unroll
    for (int i = 0; i < D; ++i) { lo[i] = fsub(v[i], v[D]); hi[i] = fadd(v[i], v[D]); }
  } else {
    tri_aabb(v, v + 3, v + 6, lo, hi);
  }
}

// Writes a child's box into its slot of the parent's record (or the root
// box): 2D floats at an 8-byte aligned offset, as D two-float stores.
template <int D>
__device__ __forceinline__ void store_slot(const RefitParams& p, uint32_t parent, const float* lo, const float* hi) {
  float* dst;
  if (parent == kNoHit) {
    dst = p.root_box;
  } else {
    dst = reinterpret_cast<float*>(p.nodes + size_t(parent >> 1) * NodeLayout<D>::vec) + (parent & 1u) * 2 * D;
  }
  float v[2 * D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    v[i] = lo[i];
    v[D + i] = hi[i];
  }
  float2* d2 = reinterpret_cast<float2*>(dst);
#pragma unroll
  for (int i = 0; i < D; ++i) d2[i] = make_float2(v[2 * i], v[2 * i + 1]);
}

// The union of a record's two child boxes (its own box in its parent),
// read past L1 (the sibling thread wrote them) as D 16-byte loads.
template <int D>
__device__ __forceinline__ void record_union(const float4* rec, float* lo, float* hi) {
  float b[4 * D];
#pragma unroll
  for (int w = 0; w < D; ++w) {
    const float4 x = __ldcg(rec + w);
    b[4 * w] = x.x;
    b[4 * w + 1] = x.y;
    b[4 * w + 2] = x.z;
    b[4 * w + 3] = x.w;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) {
    lo[i] = fminf(b[i], b[2 * D + i]);
    hi[i] = fmaxf(b[D + i], b[3 * D + i]);
  }
}

template <int D, int N> __global__ void __launch_bounds__(256) refit_kernel(const RefitParams p) {
  const uint32_t li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= p.n_leaves) return;
  const RefitLeaf L = p.leaves[li];
  using PL = PrimLayout<D, N>;
  float lo[D], hi[D];
#pragma unroll
  for (int i = 0; i < D; ++i) { lo[i] = __int_as_float(0x7f800000); hi[i] = __int_as_float(0xff800000); }
  for (uint32_t j = 0; j < L.count; ++j) {
    const uint32_t pos = L.first + j;
    const uint32_t id = p.prim_ids[pos];
    const float* v = p.prim_data + size_t(id) * p.stride;
    float rec[PL::vec * 4];
#pragma unroll
    for (int w = 0; w < PL::vec * 4; ++w) rec[w] = 0.f;
#pragma unroll
    for (int w = 0; w < PL::payload; ++w) rec[w] = v[w];
    rec[PL::id_word] = __uint_as_float(id | (j + 1 == L.count ? kLeafBit : 0u));
    float4* dst = p.prims + size_t(pos) * PL::vec;
#pragma unroll
    for (int w = 0; w < PL::vec; ++w) dst[w] = make_float4(rec[4 * w], rec[4 * w + 1], rec[4 * w + 2], rec[4 * w + 3]);
    float plo[D], phi[D];
    prim_box<D, N>(rec, plo, phi);
#pragma unroll
    for (int i = 0; i < D; ++i) { lo[i] = fminf(lo[i], plo[i]); hi[i] = fmaxf(hi[i], phi[i]); }
  }
  bool fin = true;
#pragma unroll
  for (int i = 0; i < D; ++i) fin = fin && isfinite(lo[i]) && isfinite(hi[i]);
  if (!fin) atomicOr(p.nonfinite, 1);
  uint32_t parent = L.parent;
  store_slot<D>(p, parent, lo, hi);
  while (parent != kNoHit) {
    __threadfence();
    const uint32_t node = parent >> 1;
    if (atomicAdd(p.arrivals + node, 1u) == 0u) return;  // the sibling finishes this node
    __threadfence();
    record_union<D>(p.nodes + size_t(node) * NodeLayout<D>::vec, lo, hi);
    parent = p.parents[node];
    store_slot<D>(p, parent, lo, hi);
  }
}

// After a refit (and wide_sync_kernel): every quantised record is quantised
// again from its exact four-wide record.
template <int D>
__global__ void quant_sync_kernel(float4* qnodes, const float4* __restrict__ wnodes, uint32_t n_records) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_records) return;
  float rec[WideLayout<D>::vec * 4];
  load_vec<WideLayout<D>::vec>(wnodes + size_t(r) * WideLayout<D>::vec, rec);
  uint32_t codes[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) codes[k] = __float_as_uint(rec[8 * D + k]);
  uint32_t out[QuantLayout<D>::vec * 4];
#pragma unroll
  for (int w = 0; w < QuantLayout<D>::vec * 4; ++w) out[w] = 0u;
  quantize_record<D>(rec, codes, out);
  uint4* dst = reinterpret_cast<uint4*>(qnodes + size_t(r) * QuantLayout<D>::vec);
#pragma unroll
  for (int w = 0; w < QuantLayout<D>::vec; ++w) dst[w] = make_uint4(out[4 * w], out[4 * w + 1], out[4 * w + 2], out[4 * w + 3]);
}

// Function-pointer table entry for one (D, narrow) pair.
// After a refit: every four-wide slot copies its box from the binary record
// slot that holds the same node's box (src = record << 1 | slot).
template <int D>
__global__ void wide_sync_kernel(float4* wnodes, const float4* __restrict__ nodes, const uint32_t* __restrict__ src,
                                 uint32_t n_slots) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_slots || src[i] == kNoHit) return;
  const float* from = reinterpret_cast<const float*>(nodes + size_t(src[i] >> 1) * NodeLayout<D>::vec) +
                      (src[i] & 1u) * 2 * D;
  float* to = reinterpret_cast<float*>(wnodes + size_t(i / 4) * WideLayout<D>::vec) + (i % 4) * 2 * D;
  for (int k = 0; k < 2 * D; ++k) to[k] = from[k];
}

struct KernelSet {
  const void* ray_nearest[2][2];  // [ref][stats]
  const void* ray_nearest_wide;   // near-first over the four-wide records
  const void* ray_nearest_quant;  // near-first over the quantised four-wide records
  const void* ray_nearest_regtop; // near-first, postponed leaves, stack top in registers (WALK = 1)
  const void* ray_nearest_vote;   // near-first, child order by warp vote (WALK = 2)
  const void* wide_sync;          // refreshes four-wide boxes from the binary records
  const void* quant_sync;         // quantises the four-wide records again
  const void* ray_all[2];         // [stats]
  const void* cast_nearest[2];    // [ref]
  const void* cast_all;
  const void* overlap;
  const void* overlap_heavy;  // block-per-region overlap of the regions over the visit budget
  const void* refit_leaves;
  const void* ray_nearest_seeded[2];  // [stats]; D = 3 only
};

#ifndef __CUDACC_RTC__  // host code: not part of a run-time compiled unit
template <int D, int N> KernelSet make_kernel_set() {
  KernelSet s;
  s.ray_nearest[0][0] = (const void*)query_kernel<D, N, kRayNearest, false, false>;
  s.ray_nearest[0][1] = (const void*)query_kernel<D, N, kRayNearest, false, true>;
  s.ray_nearest[1][0] = (const void*)query_kernel<D, N, kRayNearest, true, false>;
  s.ray_nearest[1][1] = (const void*)query_kernel<D, N, kRayNearest, true, true>;
  s.ray_nearest_wide = (const void*)query_kernel<D, N, kRayNearest, false, false, false, true>;
  s.ray_nearest_quant = (const void*)query_kernel<D, N, kRayNearest, false, false, false, true, true>;
  s.ray_nearest_regtop = (const void*)query_kernel<D, N, kRayNearest, false, false, false, false, false, 1>;
  s.ray_nearest_vote = (const void*)query_kernel<D, N, kRayNearest, false, false, false, false, false, 2>;
  s.wide_sync = (const void*)wide_sync_kernel<D>;
  s.quant_sync = (const void*)quant_sync_kernel<D>;
  s.ray_all[0] = (const void*)query_kernel<D, N, kRayAll, true, false>;
  s.ray_all[1] = (const void*)query_kernel<D, N, kRayAll, true, true>;
  s.cast_nearest[0] = (const void*)query_kernel<D, N, kCastNearest, false, false>;
  s.cast_nearest[1] = (const void*)query_kernel<D, N, kCastNearest, true, false>;
  s.cast_all = (const void*)query_kernel<D, N, kCastAll, true, false>;
  s.overlap = (const void*)query_kernel<D, N, kOverlap, true, false>;
  s.overlap_heavy = (const void*)overlap_heavy_kernel<D, N>;
  s.refit_leaves = (const void*)refit_kernel<D, N>;
  s.ray_nearest_seeded[0] = nullptr;
  s.ray_nearest_seeded[1] = nullptr;
  if constexpr (D == 3) {
    s.ray_nearest_seeded[0] = (const void*)query_kernel<D, N, kRayNearest, false, false, true>;
    s.ray_nearest_seeded[1] = (const void*)query_kernel<D, N, kRayNearest, false, true, true>;
  }
  return s;
}
#endif

}  // namespace sq
