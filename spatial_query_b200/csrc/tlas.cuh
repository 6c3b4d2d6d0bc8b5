// Two-level (Tlas -> instance -> BLAS) traversal and refit for sm_100a.
//
// Restates accel/tlas.rs on the device: the top level is a child-pair tree
// over instance world AABBs; at a top-level leaf each instance maps the world
// ray into its local space (R^T (o - t), R^T d; maths/isometry.rs:70-78),
// runs its own narrow phase and lifts the hit back (toi kept, point =
// ray.at(toi), normal = R n; tlas.rs:459-481). A mesh instance's narrow phase
// is a whole nearest query in its BLAS (a triangle Bvh shared by every
// instance of that mesh) with the origin divided by the instance scale and
// max_toi / s, the toi scaled back -- the instance provider of the benchmark
// scene. The BLAS walk runs inside the same thread, on the stack entries above
// the top level's.
//
// One persistent launch serves a mixed batch: the work counter runs over
// [rays | casts | regions] and each lane handles whatever kind its index
// falls in, so rays, shape casts and overlap queries over BLASes of uneven
// size share one grid.
#pragma once

#include "traverse.cuh"

namespace sq {

enum InstKind : int { kInstMesh = 0, kInstBox = 1, kInstBall = 2 };
enum TQuery : int {
  kTRayNearest = 0,
  kTRayAll = 1,
  kTRayCross = 2,
  kTCastNearest = 3,
  kTCastAll = 4,
  kTOverlapCount = 5,
  kTOverlapFill = 6,
  kTOverlapList = 7,
};

// Instance record in top-level leaf order: R (row-major D x D), t[D],
// param (scale | half-extents[D] | radius), blas id, instance id | last flag.
template <int D, int IK> struct InstLayout {
  static constexpr int P = (IK == kInstBox) ? D : 1;
  static constexpr int rot = 0;
  static constexpr int trans = D * D;
  static constexpr int param = D * D + D;
  static constexpr int blas = D * D + D + P;
  static constexpr int id = D * D + D + P + 1;
  static constexpr int words = id + 1;
  static constexpr int vec = (words + 3) / 4;
};

struct BlasRoot {
  uint32_t code;
  uint32_t pad;
  float lo[3];
  float hi[3];
};

struct TlasParams {
  const float4* __restrict__ nodes;
  float4* insts;
  const float* root_box;
  const int* nonfinite;
  const float* local_aabbs;  // per instance position, min[D] max[D]
  float* world_aabbs;        // per instance position, min[D] max[D]
  const uint64_t* __restrict__ layers;
  const uint32_t* __restrict__ sub;
  const float4* __restrict__ bnodes;
  const float4* __restrict__ bprims;
  const BlasRoot* __restrict__ broots;
  uint32_t* counter;
  const float* rays;
  const float* ray_mt;
  const float* casts;
  const float* cast_mt;
  const float* regions;
  uint32_t* r_leaf;
  float* r_toi;
  uint32_t* r_sub;
  float* r_normal;
  float* r_point;
  uint32_t* r_count;
  uint32_t* c_leaf;
  float* c_toi;
  uint32_t* c_sub;
  float* c_normal;
  float* c_point;
  uint32_t* c_count;
  uint32_t* o_count;
  const unsigned long long* o_offsets;
  uint32_t* o_leaves;
  unsigned long long* stats;
  unsigned long long mask;
  long long exclude;
  float ray_max_toi;
  float cast_max_toi;
  uint32_t root_code;
  uint32_t n_ray, n_cast, n_region;
  uint32_t r_k, c_k, o_k;
  int ray_kind, cast_kind, region_kind;
  int stack;
  int blas_finite;  // every BLAS bound is finite
  uint32_t* replay_count;  // optional: queries answered again in the reference order
  float window;            // relative window past the limit within which near-first still visits nodes
};

__device__ __forceinline__ bool t_accepts(const TlasParams& p, uint32_t id) {
  if (!p.layers) return true;
  if (p.exclude >= 0 && (unsigned long long)p.exclude == id) return false;
  return (__ldg(p.layers + id) & p.mask) != 0ull;
}

// Isometry::rotate / rotate_transpose (maths/isometry.rs:100-123):
// accumulate from 0.0 in column order.
template <int D> __device__ __forceinline__ void rotate(const float* R, const float* v, float* out) {
#pragma unroll
  for (int i = 0; i < D; ++i) {
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < D; ++j) acc = fadd(acc, fmul(R[i * D + j], v[j]));
    out[i] = acc;
  }
}
template <int D> __device__ __forceinline__ void rotate_t(const float* R, const float* v, float* out) {
#pragma unroll
  for (int i = 0; i < D; ++i) {
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < D; ++j) acc = fadd(acc, fmul(R[j * D + i], v[j]));
    out[i] = acc;
  }
}

// Isometry::transform_aabb (maths/isometry.rs:84-97).
template <int D>
__device__ __forceinline__ void transform_aabb(const float* R, const float* t, const float* llo, const float* lhi,
                                               float* wlo, float* whi) {
  float c[D], h[D], wc[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    c[i] = fmul(fadd(llo[i], lhi[i]), 0.5f);
    h[i] = fmul(fsub(lhi[i], llo[i]), 0.5f);
  }
  rotate<D>(R, c, wc);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    wc[i] = fadd(wc[i], t[i]);
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < D; ++j) acc = fadd(acc, fmul(fabsf(R[i * D + j]), h[j]));
    wlo[i] = fsub(wc[i], acc);
    whi[i] = fadd(wc[i], acc);
  }
}

// The oriented-box instance's local test (tests/two_level.rs:70-113).
template <int D>
__device__ __forceinline__ bool ray_local_box(const float* o, const float* d, const float* h, float max_toi, float& t,
                                              float* n) {
  float t_min = 0.f, t_max = max_toi;
  int axis = -1;
  bool ok = true;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    if (fabsf(d[i]) < 1.0e-9f) {
      ok = ok && !(o[i] < -h[i] || o[i] > h[i]);
    } else {
      const float inv = fdiv(1.0f, d[i]);
      float t1 = fmul(fsub(-h[i], o[i]), inv);
      float t2 = fmul(fsub(h[i], o[i]), inv);
      if (t1 > t2) { float x = t1; t1 = t2; t2 = x; }
      if (t1 > t_min) { t_min = t1; axis = i; }
      if (t2 < t_max) t_max = t2;
    }
  }
  if (!ok || t_min > t_max) return false;
  if (!(axis >= 0 && t_min > 1.0e-6f && t_min <= max_toi)) return false;
  t = t_min;
  entry_normal<D>(d, axis, n);
  return true;
}

// A whole nearest query in BLAS b (Bvh::raycast_nearest, accel/bvh.rs:73-124)
// for a local ray, on stack entries [base, ...).
template <bool REF>
__device__ __forceinline__ bool blas_nearest(const TlasParams& p, uint32_t b, const RayPre<3>& r, bool fast,
                                             float mt, uint32_t* s_code, float* s_t, int tid, int base,
                                             float& t_out, uint32_t& leaf_out, float* n_out, uint32_t& flag,
                                             bool ref) {
  const BlasRoot R = p.broots[b];
  float limit = mt;
  float cut = mt;  // near-first prunes past a small window beyond the limit (traverse.cuh)
  const float kInf = __int_as_float(0x7f800000);
  // The slab without the limit, then the entry against the cut.
  auto test = [&](const float* lo, const float* hi, float& te) -> bool {
    int ax;
    const bool geo = fast ? slab_fast<3>(r, lo, hi, kInf, te) : slab<3>(r, lo, hi, kInf, te, ax);
    return geo && te <= cut;
  };
  float te0;
  if (!test(R.lo, R.hi, te0)) return false;
  uint32_t code = R.code;
  int sp = base;
  uint32_t best = kNoHit;
  float best_t = 0.f, best_n[3] = {0.f, 0.f, 0.f};
  for (;;) {
    bool done = false;
    while (!(code & kLeafBit)) {
      float rec[NodeLayout<3>::vec * 4];
      load_vec<NodeLayout<3>::vec>(p.bnodes + size_t(code) * NodeLayout<3>::vec, rec);
      const uint32_t ca = __float_as_uint(rec[12]);
      const uint32_t cb = __float_as_uint(rec[13]);
      float ta, tb;
      const bool pa = test(rec, rec + 3, ta);
      const bool pb = test(rec + 6, rec + 9, tb);
      if (pa && pb) {
        const bool a_first = REF ? false : (!ref && ta <= tb);
        s_code[sp * kThreads + tid] = a_first ? cb : ca;
        s_t[sp * kThreads + tid] = a_first ? tb : ta;
        ++sp;
        code = a_first ? ca : cb;
      } else if (pa) {
        code = ca;
      } else if (pb) {
        code = cb;
      } else {
        bool found = false;
        while (sp > base) {
          --sp;
          code = s_code[sp * kThreads + tid];
          const float t = s_t[sp * kThreads + tid];
          if (t <= cut) { found = true; break; }
        }
        if (!found) { done = true; break; }
      }
    }
    if (done) break;
    uint32_t pos = code & ~kLeafBit;
    for (;;) {
      float rec[12];
      load_vec<3>(p.bprims + size_t(pos) * 3, rec);
      const uint32_t idw = __float_as_uint(rec[9]);
      const uint32_t id = idw & ~kLeafBit;
      float t, nrm[3];
      if (ray_triangle(r.o, r.d, rec, rec + 3, rec + 6, t) && !(t > limit)) {
        if (best == kNoHit || hit_before(t, id, best_t, best)) {
          tri_normal(rec, rec + 3, rec + 6, nrm);
          best = id;
          best_t = t;
          limit = t;
          cut = t;
          if (!REF && !ref) {
            // certify the new best: not before its own triangle's AABB entry
            float lo[3], hi[3], te;
            int ax;
            tri_aabb(rec, rec + 3, rec + 6, lo, hi);
            if (fast) slab_fast<3>(r, lo, hi, kInf, te);
            else slab<3>(r, lo, hi, kInf, te, ax);
            flag = uint32_t(t < te);
            cut = near_limit(t, p.window);
          }
          best_n[0] = nrm[0];
          best_n[1] = nrm[1];
          best_n[2] = nrm[2];
        }
      }
      if (idw & kLeafBit) break;
      ++pos;
    }
    bool found = false;
    while (sp > base) {
      --sp;
      code = s_code[sp * kThreads + tid];
      const float t = s_t[sp * kThreads + tid];
      if (t <= cut) { found = true; break; }
    }
    if (!found) break;
  }
  if (best == kNoHit) return false;
  t_out = best_t;
  leaf_out = best;
  n_out[0] = best_n[0];
  n_out[1] = best_n[1];
  n_out[2] = best_n[2];
  return true;
}

template <int D> struct TLane {
  RayPre<D> r;  // world ray or cast path; regions keep lo in o and hi in d
  float pmin[D], pmax[D];
  float limit;
  float cut;         // nodes whose entry lies past this are pruned
  uint32_t flag;     // the best hit so far is not certified (traverse.cuh)
  bool ref;          // this pass runs in the reference order (a replay)
  uint32_t q;
  int kind;
  uint32_t code;
  int sp;
  bool fast;
  uint32_t best_leaf, best_sub;
  float best_t;
  float best_n[D];
  uint32_t count;
  unsigned long long csr_base;
  uint32_t v_nodes, v_nar, v_hit;
};

// The mesh-instance walk (the two-level benchmark's kernel) is latency-bound
// with divergent lanes, so resident warps count more than registers: it is
// held to five resident blocks per SM (96 registers, a few spilled), which
// measured 3.87 ms per two-level frame against 4.29 ms at six blocks (80
// registers) and 3.89 ms at four.
template <int D, int IK, bool REF, bool STATS>
__global__ void __launch_bounds__(kThreads, (IK == kInstMesh && !REF && !STATS) ? 5 : 1)
    tlas_kernel(const TlasParams p) {
  using IL = InstLayout<D, IK>;
  using NL = NodeLayout<D>;
  constexpr uint32_t FULL = 0xffffffffu;
  extern __shared__ uint32_t smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int S = p.stack;
  uint32_t* s_code = smem;
  float* s_t = reinterpret_cast<float*>(smem + S * kThreads);
  const uint32_t lt_mask = (1u << lane) - 1u;
  const bool scene_finite = p.nonfinite ? (*p.nonfinite == 0) : true;
  const uint32_t n_total = p.n_ray + p.n_cast + p.n_region;
  uint32_t replays = 0;
  const float kInf = __int_as_float(0x7f800000);

  unsigned long long c_vis = 0, c_nar = 0, c_hit = 0;
  TLane<D> L;
  bool live = false, exhausted = false;

  auto is_ray = [&]() { return L.kind <= kTRayCross; };
  auto is_cast = [&]() { return L.kind == kTCastNearest || L.kind == kTCastAll; };
  auto is_nearest = [&]() { return L.kind == kTRayNearest || L.kind == kTCastNearest; };

  auto test_box = [&](const float* lo, const float* hi, float& te) -> bool {
    if (L.kind >= kTOverlapCount) {
      te = 0.f;
      return box_overlap<D>(lo, hi, L.r.o, L.r.d);
    }
    int ax;
    bool geo;
    if (is_cast()) {
      geo = L.fast ? slab_grown_fast<D>(L.r, lo, hi, L.pmin, L.pmax, kInf, te)
                   : slab_grown<D>(L.r, lo, hi, L.pmin, L.pmax, kInf, te, ax);
    } else {
      geo = L.fast ? slab_fast<D>(L.r, lo, hi, kInf, te) : slab<D>(L.r, lo, hi, kInf, te, ax);
    }
    return geo && te <= L.cut;
  };

  auto pop = [&]() -> bool {
    const bool nearest = is_nearest();
    while (L.sp > 0) {
      --L.sp;
      L.code = s_code[L.sp * kThreads + tid];
      const float t = s_t[L.sp * kThreads + tid];
      if (!nearest || t <= L.cut) return true;
    }
    return false;
  };

  auto start = [&](uint32_t g) -> bool {
    L.flag = 0u;
    const float* src;
    if (g < p.n_ray) {
      L.kind = p.ray_kind;
      L.q = g;
      src = p.rays + size_t(g) * 2 * D;
      L.limit = p.ray_mt ? p.ray_mt[g] : p.ray_max_toi;
    } else if (g < p.n_ray + p.n_cast) {
      L.kind = p.cast_kind;
      L.q = g - p.n_ray;
      src = p.casts + size_t(L.q) * 4 * D;
      L.limit = p.cast_mt ? p.cast_mt[L.q] : p.cast_max_toi;
    } else {
      L.kind = p.region_kind;
      L.q = g - p.n_ray - p.n_cast;
      src = p.regions + size_t(L.q) * 2 * D;
      L.limit = 0.f;
    }
#pragma unroll
    for (int i = 0; i < D; ++i) {
      L.r.o[i] = src[i];
      L.r.d[i] = src[D + i];
    }
    if (is_cast()) {
#pragma unroll
      for (int i = 0; i < D; ++i) {
        L.pmin[i] = src[2 * D + i];
        L.pmax[i] = src[3 * D + i];
      }
    }
    L.fast = false;
    if (L.kind < kTOverlapCount) {
      ray_prep<D>(L.r);
      bool f = scene_finite && L.r.par == 0u && !isnan(L.limit);
#pragma unroll
      for (int i = 0; i < D; ++i) f = f && isfinite(L.r.o[i]) && isfinite(L.r.d[i]);
      if (is_cast()) {
#pragma unroll
        for (int i = 0; i < D; ++i) f = f && isfinite(L.pmin[i]) && isfinite(L.pmax[i]);
      }
      L.fast = f;
    }
    L.best_leaf = kNoHit;
    L.best_sub = kNoHit;
    L.best_t = 0.f;
#pragma unroll
    for (int i = 0; i < D; ++i) L.best_n[i] = 0.f;
    L.count = 0;
    L.csr_base = (L.kind == kTOverlapFill) ? p.o_offsets[L.q] : 0ull;
    L.v_nodes = STATS ? 1u : 0u;
    L.v_nar = 0;
    L.v_hit = 0;
    L.sp = 0;
    L.code = p.root_code;
    L.cut = L.limit;
    float lo[D], hi[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      lo[i] = p.root_box[i];
      hi[i] = p.root_box[D + i];
    }
    float te;
    return test_box(lo, hi, te);
  };

  auto finish = [&]() {
    const uint32_t q = L.q;
    if (L.kind == kTRayNearest || L.kind == kTCastNearest) {
      const bool ray = L.kind == kTRayNearest;
      uint32_t* o_leaf = ray ? p.r_leaf : p.c_leaf;
      float* o_toi = ray ? p.r_toi : p.c_toi;
      uint32_t* o_sub = ray ? p.r_sub : p.c_sub;
      float* o_nrm = ray ? p.r_normal : p.c_normal;
      float* o_pt = ray ? p.r_point : p.c_point;
      o_leaf[q] = L.best_leaf;
      if (o_toi) o_toi[q] = L.best_t;
      if (o_sub) o_sub[q] = L.best_sub;
      if (o_nrm)
#pragma unroll
        for (int i = 0; i < D; ++i) o_nrm[size_t(q) * D + i] = L.best_n[i];
      if (o_pt) {
        float pt[D];
        if (L.best_leaf != kNoHit) {
          ray_at<D>(L.r.o, L.r.d, L.best_t, pt);
        } else {
#pragma unroll
          for (int i = 0; i < D; ++i) pt[i] = 0.f;
        }
#pragma unroll
        for (int i = 0; i < D; ++i) o_pt[size_t(q) * D + i] = pt[i];
      }
    } else if (L.kind == kTRayAll || L.kind == kTRayCross) {
      p.r_count[q] = L.count;
    } else if (L.kind == kTCastAll) {
      p.c_count[q] = L.count;
    } else if (L.kind == kTOverlapCount || L.kind == kTOverlapList) {
      p.o_count[q] = L.count;
    }
    if (STATS) {
      c_vis += L.v_nodes;
      c_nar += L.v_nar;
      c_hit += L.v_hit;
    }
  };

  // One world-space hit of instance `id` for the lane's query.
  // The slab entry of instance `pos`'s world AABB (computed only for a hit).
  auto inst_entry = [&](uint32_t pos) -> float {
    const float* w = p.world_aabbs + size_t(pos) * 2 * D;
    float te;
    int ax;
    if (is_cast()) {
      if (L.fast) slab_grown_fast<D>(L.r, w, w + D, L.pmin, L.pmax, kInf, te);
      else slab_grown<D>(L.r, w, w + D, L.pmin, L.pmax, kInf, te, ax);
    } else {
      if (L.fast) slab_fast<D>(L.r, w, w + D, kInf, te);
      else slab<D>(L.r, w, w + D, kInf, te, ax);
    }
    return te;
  };

  // `inner` is set when the instance's own nearest hit is not certified.
  auto take = [&](float t, uint32_t id, uint32_t subv, const float* n, uint32_t pos, uint32_t inner) {
    if (is_nearest()) {
      if (L.best_leaf == kNoHit || hit_before(t, id, L.best_t, L.best_leaf)) {
        L.best_leaf = id;
        L.best_sub = subv;
        L.best_t = t;
        L.limit = t;
        L.cut = t;
        if (!REF && !L.ref) {
          L.flag = inner | uint32_t(t < inst_entry(pos));
          L.cut = near_limit(t, p.window);
        }
#pragma unroll
        for (int i = 0; i < D; ++i) L.best_n[i] = n[i];
      }
    } else if (L.kind == kTCastAll) {
      list_put<D>(p.c_k, p.c_leaf, p.c_toi, p.c_sub, p.c_normal, L.q, L.count, t, id, subv, n);
    } else {
      list_put<D>(p.r_k, p.r_leaf, p.r_toi, p.r_sub, p.r_normal, L.q, L.count, t, id, subv, n);
    }
  };

  auto leaf = [&]() {
    uint32_t pos = L.code & ~kLeafBit;
    for (;;) {
      float rec[IL::vec * 4];
      load_vec<IL::vec>(p.insts + size_t(pos) * IL::vec, rec);
      const uint32_t idw = __float_as_uint(rec[IL::id]);
      const uint32_t id = idw & ~kLeafBit;
      const uint32_t subv = p.sub ? __ldg(p.sub + id) : kNoHit;
      if (t_accepts(p, id)) {
        const float* R = rec + IL::rot;
        const float* tr = rec + IL::trans;
        if (L.kind >= kTOverlapCount) {
          bool hit;
          if constexpr (IK == kInstMesh) {
            hit = box_overlap<D>(p.world_aabbs + size_t(pos) * 2 * D, p.world_aabbs + size_t(pos) * 2 * D + D, L.r.o,
                                 L.r.d);
          } else if constexpr (IK == kInstBall) {
            float d2 = 0.f;
#pragma unroll
            for (int i = 0; i < D; ++i) {
              const float c = tr[i];
              const float v = (c < L.r.o[i]) ? fsub(L.r.o[i], c) : ((c > L.r.d[i]) ? fsub(c, L.r.d[i]) : 0.f);
              d2 = fadd(d2, fmul(v, v));
            }
            hit = fsqrt(d2) <= rec[IL::param];
          } else {
            hit = true;  // instance.rs:280-282 default
          }
          if (hit) {
            if (L.kind == kTOverlapFill) {
              // appended in walk order; the host call sorts each segment afterwards
              p.o_leaves[L.csr_base + L.count] = id;
            } else if (L.kind == kTOverlapList) {
              // the first k leaves in ascending order
              const uint32_t k = p.o_k;
              const size_t base = size_t(L.q) * k;
              uint32_t m = L.count < k ? L.count : k;
              if (k && (m < k || id < p.o_leaves[base + k - 1])) {
                uint32_t j = (m < k) ? m : k - 1;
                while (j > 0 && p.o_leaves[base + j - 1] > id) {
                  p.o_leaves[base + j] = p.o_leaves[base + j - 1];
                  --j;
                }
                p.o_leaves[base + j] = id;
              }
            }
            ++L.count;
          }
        } else if (is_cast()) {
          float t, n[D];
          bool hit = false;
          if constexpr (IK == kInstMesh) {
            int axis;
            hit = slab_grown<D>(L.r, p.world_aabbs + size_t(pos) * 2 * D, p.world_aabbs + size_t(pos) * 2 * D + D,
                                L.pmin, L.pmax, L.limit, t, axis);
            if (hit) entry_normal<D>(L.r.d, axis, n);
          } else if constexpr (IK == kInstBall) {
            hit = ray_ball<D, true>(L.r.o, L.r.d, tr, fadd(rec[IL::param], L.pmax[0]), L.limit, t, n);
          }
          if (hit) take(t, id, IK == kInstMesh ? kNoHit : subv, n, pos, 0u);
        } else {
          if (STATS) L.v_nar += 1;
          // World ray -> instance space (tlas.rs:465-471).
          float v[D], lo[D], ld[D];
#pragma unroll
          for (int i = 0; i < D; ++i) v[i] = fsub(L.r.o[i], tr[i]);
          rotate_t<D>(R, v, lo);
          rotate_t<D>(R, L.r.d, ld);
          if constexpr (IK == kInstMesh) {
            const float s = rec[IL::param];
            RayPre<3> lr;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
              lr.o[i] = fdiv(lo[i], s);
              lr.d[i] = ld[i];
            }
            ray_prep<3>(lr);
            bool f = p.blas_finite && lr.par == 0u && isfinite(s);
#pragma unroll
            for (int i = 0; i < 3; ++i) f = f && isfinite(lr.o[i]) && isfinite(lr.d[i]);
            float ts, nl[3];
            uint32_t face;
            const float mts = fdiv(L.limit, s);
            uint32_t bflag = 0u;
            // Only nearest queries are answered again when an instance's hit
            // is not certified, so the others walk the BLAS in the crate's
            // own order, whose answer needs no certificate.
            const bool bh = blas_nearest<REF>(p, __float_as_uint(rec[IL::blas]), lr, f && !isnan(mts), mts, s_code,
                                              s_t, tid, L.sp, ts, face, nl, bflag, L.ref || !is_nearest());
            if (bh) {
              const float toi = fmul(ts, s);
              if (!(toi > L.limit)) {
                float nw[3];
                rotate<3>(R, nl, nw);
                if (STATS) L.v_hit += 1;
                take(toi, id, face, nw, pos, bflag);
              }
            }
          } else if constexpr (IK == kInstBox) {
            float t, nl[D], nw[D];
            if (ray_local_box<D>(lo, ld, rec + IL::param, L.limit, t, nl)) {
              rotate<D>(R, nl, nw);
              if (STATS) L.v_hit += 1;
              take(t, id, subv, nw, pos, 0u);
            }
          } else {
            const float rr = rec[IL::param];
            if (L.kind == kTRayCross) {
              // Both roots at the local origin (tests/crossings.rs:679-694).
              const float b = pdot<D>(lo, ld);
              const float disc = fsub(fmul(b, b), fsub(pdot<D>(lo, lo), fmul(rr, rr)));
              if (!(disc < 0.f)) {
                const float sq = fsqrt(disc);
                const float roots[2] = {fsub(-b, sq), fadd(-b, sq)};
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                  const float tt = roots[j];
                  if (tt >= 0.f && tt <= L.limit) {
                    float nl[D], nw[D];
                    ray_at<D>(lo, ld, tt, nl);
                    normalize_or_zero<D>(nl);
                    rotate<D>(R, nl, nw);
                    if (STATS) L.v_hit += 1;
                    take(tt, id, subv, nw, pos, 0u);
                  }
                }
              }
            } else {
              float zero[D], t, nl[D], nw[D];
#pragma unroll
              for (int i = 0; i < D; ++i) zero[i] = 0.f;
              if (ray_ball<D, true>(lo, ld, zero, rr, L.limit, t, nl)) {
                rotate<D>(R, nl, nw);
                if (STATS) L.v_hit += 1;
                take(t, id, subv, nw, pos, 0u);
              }
            }
          }
        }
      }
      if (idw & kLeafBit) break;
      ++pos;
    }
  };

  // Mesh instances, rays (nearest, all hits, crossings): a lane walks its
  // instances' BLASes inside the same descent loop as the top level, one
  // leaf per pass, so that lanes in different levels and instances share
  // the node-test instructions instead of each lane finishing a whole BLAS
  // walk (blas_nearest) while the rest of its warp waits. Same visits, same
  // order, same answers: nearest rays walk a BLAS near-first with the
  // certificate, list rays walk it in the crate's own order (their
  // instance hits are never answered again, so they need none) and list the
  // instance's hit.
  bool in_blas = false;
  bool b_last = false;    // the instance is the last of its top-level leaf
  uint32_t b_pos = 0;     // instance record whose BLAS is walked
  int b_base = 0;         // stack depth at BLAS entry
  RayPre<3> b_r;          // the ray in instance space (origin divided by the scale)
  bool b_fast = false;
  float b_limit = 0.f, b_cut = 0.f, b_t = 0.f;
  uint32_t b_best = kNoHit, b_flag = 0u;
  float b_n[3] = {0.f, 0.f, 0.f};
  auto unified = [&]() { return IK == kInstMesh && L.kind <= kTRayCross; };

  // blas_nearest's box test and leaf, on the lane's BLAS state.
  auto btest = [&](const float* lo, const float* hi, float& te) -> bool {
    int ax;
    const bool geo = b_fast ? slab_fast<3>(b_r, lo, hi, kInf, te) : slab<3>(b_r, lo, hi, kInf, te, ax);
    return geo && te <= b_cut;
  };
  auto blas_leaf = [&]() {
    uint32_t pos = L.code & ~kLeafBit;
    for (;;) {
      float rec[12];
      load_vec<3>(p.bprims + size_t(pos) * 3, rec);
      const uint32_t idw = __float_as_uint(rec[9]);
      const uint32_t id = idw & ~kLeafBit;
      float t, nrm[3];
      if (ray_triangle(b_r.o, b_r.d, rec, rec + 3, rec + 6, t) && !(t > b_limit)) {
        if (b_best == kNoHit || hit_before(t, id, b_t, b_best)) {
          tri_normal(rec, rec + 3, rec + 6, nrm);
          b_best = id;
          b_t = t;
          b_limit = t;
          b_cut = t;
          if (!REF && !L.ref && L.kind == kTRayNearest) {
            // certify the new best: not before its own triangle's AABB entry
            float lo[3], hi[3], te;
            int ax;
            tri_aabb(rec, rec + 3, rec + 6, lo, hi);
            if (b_fast) slab_fast<3>(b_r, lo, hi, kInf, te);
            else slab<3>(b_r, lo, hi, kInf, te, ax);
            b_flag = uint32_t(t < te);
            b_cut = near_limit(t, p.window);
          }
          b_n[0] = nrm[0];
          b_n[1] = nrm[1];
          b_n[2] = nrm[2];
        }
      }
      if (idw & kLeafBit) break;
      ++pos;
    }
  };
  // Pops within the lane's current level: the BLAS's own entries when in
  // one (false: the BLAS is exhausted), else the top level's (pop).
  auto pop_level = [&]() -> bool {
    if (in_blas) {
      while (L.sp > b_base) {
        --L.sp;
        L.code = s_code[L.sp * kThreads + tid];
        const float t = s_t[L.sp * kThreads + tid];
        if (t <= b_cut) return true;
      }
      return false;
    }
    return pop();
  };
  // The instances of a top-level leaf from record `pos` on, as leaf() takes
  // them for a nearest ray: the first accepted one whose BLAS root the
  // instance-space ray enters starts its walk (true); false when the leaf
  // has no such instance left.
  auto enter_from = [&](uint32_t pos) -> bool {
    if constexpr (IK == kInstMesh) {
      for (;;) {
        float rec[IL::vec * 4];
        load_vec<IL::vec>(p.insts + size_t(pos) * IL::vec, rec);
        const uint32_t idw = __float_as_uint(rec[IL::id]);
        const uint32_t id = idw & ~kLeafBit;
        if (t_accepts(p, id)) {
          if (STATS) L.v_nar += 1;
          // World ray -> instance space (tlas.rs:465-471).
          const float* R = rec + IL::rot;
          const float* tr = rec + IL::trans;
          float v[3], lo[3], ld[3];
#pragma unroll
          for (int i = 0; i < 3; ++i) v[i] = fsub(L.r.o[i], tr[i]);
          rotate_t<3>(R, v, lo);
          rotate_t<3>(R, L.r.d, ld);
          const float sc = rec[IL::param];
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            b_r.o[i] = fdiv(lo[i], sc);
            b_r.d[i] = ld[i];
          }
          ray_prep<3>(b_r);
          bool f = p.blas_finite && b_r.par == 0u && isfinite(sc);
#pragma unroll
          for (int i = 0; i < 3; ++i) f = f && isfinite(b_r.o[i]) && isfinite(b_r.d[i]);
          const float mts = fdiv(L.limit, sc);
          b_fast = f && !isnan(mts);
          b_limit = mts;
          b_cut = mts;
          const BlasRoot br = p.broots[__float_as_uint(rec[IL::blas])];
          float te;
          if (btest(br.lo, br.hi, te)) {
            in_blas = true;
            b_last = (idw & kLeafBit) != 0u;
            b_pos = pos;
            b_base = L.sp;
            b_best = kNoHit;
            b_flag = 0u;
            b_t = 0.f;
            L.code = br.code;
            return true;
          }
        }
        if (idw & kLeafBit) return false;
        ++pos;
      }
    }
    return false;
  };
  // The BLAS is exhausted: its nearest hit, scaled and rotated back to
  // world space, is the instance's hit (as after blas_nearest in leaf()).
  auto blas_finish = [&]() {
    in_blas = false;
    if constexpr (IK == kInstMesh) {
      if (b_best == kNoHit) return;
      float rec[IL::vec * 4];
      load_vec<IL::vec>(p.insts + size_t(b_pos) * IL::vec, rec);
      const float toi = fmul(b_t, rec[IL::param]);
      if (!(toi > L.limit)) {
        float nw[3];
        rotate<3>(rec + IL::rot, b_n, nw);
        if (STATS) L.v_hit += 1;
        take(toi, __float_as_uint(rec[IL::id]) & ~kLeafBit, b_best, nw, b_pos, b_flag);
      }
    }
  };

  bool pending = false;  // this lane's query waits to be answered again in reference order
  uint32_t pending_g = 0;
  for (;;) {
    const bool need = !live && !exhausted && !pending;
    const uint32_t need_mask = __ballot_sync(FULL, need);
    uint32_t gs = kNoHit;
    if (need_mask) {
      const int leader = __ffs(need_mask) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(p.counter, uint32_t(__popc(need_mask)));
      base = __shfl_sync(FULL, base, leader);
      if (need) {
        const uint32_t g = base + uint32_t(__popc(need_mask & lt_mask));
        if (g < n_total) gs = g;
        else exhausted = true;
      }
    }
    bool replay = false;
    if (pending) {
      gs = pending_g;
      pending = false;
      replay = true;
    }
    if (gs != kNoHit) {
      L.ref = replay;
      in_blas = false;
      live = start(gs);
      if (!live) finish();
    }
    if (!__ballot_sync(FULL, live)) {
      if (__all_sync(FULL, exhausted)) break;
      continue;
    }
    if (live) {
      bool done = false;
      // Descend interior records until a leaf comes up: the top level's, or
      // the BLAS's for a lane inside an instance (the same record layout).
      while (!(L.code & kLeafBit)) {
        float rec[NL::vec * 4];
        load_vec<NL::vec>((in_blas ? p.bnodes : p.nodes) + size_t(L.code) * NL::vec, rec);
        const uint32_t ca = __float_as_uint(rec[4 * D]);
        const uint32_t cb = __float_as_uint(rec[4 * D + 1]);
        float ta, tb;
        bool pa, pb;
        if (IK == kInstMesh && in_blas) {
          pa = btest(rec, rec + 3, ta);
          pb = btest(rec + 6, rec + 9, tb);
        } else {
          pa = test_box(rec, rec + D, ta);
          pb = test_box(rec + 2 * D, rec + 3 * D, tb);
          if (STATS) L.v_nodes += 2;
        }
        if (pa && pb) {
          const bool a_first = (REF || !is_nearest()) ? false : (!L.ref && ta <= tb);
          s_code[L.sp * kThreads + tid] = a_first ? cb : ca;
          s_t[L.sp * kThreads + tid] = a_first ? tb : ta;
          ++L.sp;
          L.code = a_first ? ca : cb;
        } else if (pa) {
          L.code = ca;
        } else if (pb) {
          L.code = cb;
        } else if (!pop_level()) {
          done = true;
          break;
        }
      }
      if (unified()) {
        if (in_blas) {
          // `done` here: the BLAS is exhausted, not the query.
          if (!done) {
            blas_leaf();
            done = !pop_level();
          }
          if (done) {
            const bool last = b_last;
            const uint32_t next = b_pos + 1;
            blas_finish();
            done = false;
            if (last || !enter_from(next)) done = !pop();
          }
        } else if (!done && !enter_from(L.code & ~kLeafBit)) {
          done = !pop();
        }
      } else if (!done) {
        leaf();
        done = !pop();
      }
      if (done) {
        live = false;
        if (!REF && !L.ref && L.flag != 0u) {
          // answered again in the reference order at the top of the loop
          pending = true;
          pending_g = L.q + (L.kind <= kTRayCross ? 0u : (L.kind <= kTCastAll ? p.n_ray : p.n_ray + p.n_cast));
          ++replays;
        } else {
          finish();
        }
      }
    }
  }
  if (!REF && p.replay_count) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) replays += __shfl_down_sync(FULL, replays, o);
    if (lane == 0 && replays) atomicAdd(p.replay_count, replays);
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
// Tlas::refit (accel/tlas.rs:49-54): new transforms for every instance (or a
// translation step added to each), world AABB = transform_aabb(local AABB),
// then the bottom-up union over the fixed top-level topology.
// ---------------------------------------------------------------------------

struct TlasRefitParams {
  int* nonfinite;
  float4* nodes;
  float4* insts;
  float* root_box;
  const float* local_aabbs;
  float* world_aabbs;
  const float* new_rot;    // per instance id, D x D, or null
  const float* new_trans;  // per instance id, D, or null
  const float* delta;      // per instance id, added to the translation, or null
  const float* new_param;  // per instance id (scale | half-extents[D] | radius), or null
  float* local_aabbs_w;    // rewritten when new_param is given
  const BlasRoot* broots;  // mesh AABBs, for a new scale
  const RefitLeaf* leaves;
  const uint32_t* parents;
  uint32_t* arrivals;
  uint32_t n_leaves;
};

template <int D, int IK> __global__ void __launch_bounds__(256) tlas_refit_kernel(const TlasRefitParams p) {
  using IL = InstLayout<D, IK>;
  const uint32_t li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= p.n_leaves) return;
  const RefitLeaf L = p.leaves[li];
  float lo[D], hi[D];
#pragma unroll
  for (int i = 0; i < D; ++i) { lo[i] = __int_as_float(0x7f800000); hi[i] = __int_as_float(0xff800000); }
  for (uint32_t j = 0; j < L.count; ++j) {
    const uint32_t pos = L.first + j;
    float* rec = reinterpret_cast<float*>(p.insts + size_t(pos) * IL::vec);
    const uint32_t id = __float_as_uint(rec[IL::id]) & ~kLeafBit;
    if (p.new_rot)
#pragma unroll
      for (int k = 0; k < D * D; ++k) rec[IL::rot + k] = p.new_rot[size_t(id) * D * D + k];
    if (p.new_trans)
#pragma unroll
      for (int k = 0; k < D; ++k) rec[IL::trans + k] = p.new_trans[size_t(id) * D + k];
    if (p.delta)
#pragma unroll
      for (int k = 0; k < D; ++k) rec[IL::trans + k] = fadd(rec[IL::trans + k], p.delta[size_t(id) * D + k]);
    if (p.new_param) {
      // A deforming provider: new parameters give a new local AABB
      // (s * mesh AABB, [-h, h] or [-r, r]).
#pragma unroll
      for (int k = 0; k < IL::P; ++k) rec[IL::param + k] = p.new_param[size_t(id) * IL::P + k];
      float* la = p.local_aabbs_w + size_t(pos) * 2 * D;
#pragma unroll
      for (int k = 0; k < D; ++k) {
        if constexpr (IK == kInstMesh) {
          const BlasRoot& br = p.broots[__float_as_uint(rec[IL::blas])];
          la[k] = fmul(br.lo[k < 3 ? k : 0], rec[IL::param]);
          la[D + k] = fmul(br.hi[k < 3 ? k : 0], rec[IL::param]);
        } else {
          const float h = rec[IL::param + (IK == kInstBox ? k : 0)];
          la[k] = fmul(h, -1.0f);
          la[D + k] = h;
        }
      }
    }
    float R[D * D], t[D], wlo[D], whi[D];
#pragma unroll
    for (int k = 0; k < D * D; ++k) R[k] = rec[IL::rot + k];
#pragma unroll
    for (int k = 0; k < D; ++k) t[k] = rec[IL::trans + k];
    const float* la = p.local_aabbs + size_t(pos) * 2 * D;
    transform_aabb<D>(R, t, la, la + D, wlo, whi);
    float* wa = p.world_aabbs + size_t(pos) * 2 * D;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      wa[i] = wlo[i];
      wa[D + i] = whi[i];
      lo[i] = fminf(lo[i], wlo[i]);
      hi[i] = fmaxf(hi[i], whi[i]);
    }
  }
  bool fin = true;
#pragma unroll
  for (int i = 0; i < D; ++i) fin = fin && isfinite(lo[i]) && isfinite(hi[i]);
  if (!fin) atomicOr(p.nonfinite, 1);
  RefitParams rp;
  rp.nodes = p.nodes;
  rp.root_box = p.root_box;
  uint32_t parent = L.parent;
  store_slot<D>(rp, parent, lo, hi);
  while (parent != kNoHit) {
    __threadfence();
    const uint32_t node = parent >> 1;
    if (atomicAdd(p.arrivals + node, 1u) == 0u) return;
    __threadfence();
    record_union<D>(p.nodes + size_t(node) * NodeLayout<D>::vec, lo, hi);
    parent = p.parents[node];
    store_slot<D>(rp, parent, lo, hi);
  }
}

struct TlasKernelSet {
  const void* query[2][2];  // [ref][stats]
  const void* refit;
};

template <int D, int IK> TlasKernelSet make_tlas_kernel_set() {
  TlasKernelSet s;
  s.query[0][0] = (const void*)tlas_kernel<D, IK, false, false>;
  s.query[0][1] = (const void*)tlas_kernel<D, IK, false, true>;
  s.query[1][0] = (const void*)tlas_kernel<D, IK, true, false>;
  s.query[1][1] = (const void*)tlas_kernel<D, IK, true, true>;
  s.refit = (const void*)tlas_refit_kernel<D, IK>;
  return s;
}

}  // namespace sq
