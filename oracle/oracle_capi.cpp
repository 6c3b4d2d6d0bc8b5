// TEST INFRASTRUCTURE ONLY -- C entry points over the CPU oracle
// (sq_oracle.hpp) for the Python test-suite (ctypes), the smoke check and
// the CPU-baseline leg of bench.py. Not part of the product library.
//
// Layouts (all f32 unless noted, row-major, one record per query/leaf):
//   ray     = origin[D], dir[D]                      (dir already unit)
//   cast    = origin[D], dir[D], probe_min[D], probe_max[D]
//   region  = min[D], max[D]
//   leaf    = boxes: min[D], max[D]; balls: centre[D], radius; tris: v0 v1 v2
//   no hit  = leaf 0xFFFFFFFF; sub-object None = 0xFFFFFFFF
#include <chrono>
#include <memory>

#include "sq_oracle.hpp"

using namespace orc;

namespace {

constexpr uint32_t kNoHit = 0xFFFFFFFFu;

struct SceneBase {
  int dim = 0;
  int prec = 32;
  virtual ~SceneBase() = default;
};

template <int D, class S> struct SceneImpl : SceneBase {
  Scene<D, S> g;
  Bvh<D, S> bvh;
};

struct BlasSetBase {
  virtual ~BlasSetBase() = default;
};
template <class S> struct BlasSetImpl : BlasSetBase {
  std::vector<Blas<S>> v;
};

struct TlasBase {
  int dim = 0;
  int prec = 32;
  virtual ~TlasBase() = default;
};
template <int D, class S> struct TlasImpl : TlasBase {
  InstScene<D, S> sc;
  Tlas<D, S> tlas;
};

template <int D, class S> Ray<D, S> load_ray(const float* r) {
  Ray<D, S> ray;
  for (int i = 0; i < D; ++i) { ray.origin[i] = S(r[i]); ray.dir[i] = S(r[D + i]); }
  return ray;
}
template <int D, class S> ShapeCast<D, S> load_cast(const float* c) {
  ShapeCast<D, S> s;
  for (int i = 0; i < D; ++i) {
    s.origin[i] = S(c[i]); s.dir[i] = S(c[D + i]);
    s.aabb.min[i] = S(c[2 * D + i]); s.aabb.max[i] = S(c[3 * D + i]);
  }
  return s;
}
template <int D, class S> Aabb<D, S> load_box(const float* b) {
  Aabb<D, S> a;
  for (int i = 0; i < D; ++i) { a.min[i] = S(b[i]); a.max[i] = S(b[D + i]); }
  return a;
}
inline Filter make_filter(uint64_t mask, int64_t exclude) {
  Filter f;
  f.layer_mask = mask;
  f.has_exclude = exclude >= 0;
  f.exclude = exclude >= 0 ? uint64_t(exclude) : 0;
  return f;
}

// Output sink for one hit; T is float (f32 build) or double (f64 build).
template <int D, class S, class T>
void store_hit(const std::optional<Hit<D, S>>& h, size_t q, uint32_t* leaf, T* toi, float* normal, float* point,
               uint32_t* sub) {
  if (!h) {
    leaf[q] = kNoHit;
    if (toi) toi[q] = T(0);
    if (sub) sub[q] = kNoSub;
    if (normal) for (int i = 0; i < D; ++i) normal[q * D + i] = 0.f;
    if (point) for (int i = 0; i < D; ++i) point[q * D + i] = 0.f;
    return;
  }
  leaf[q] = h->leaf;
  if (toi) toi[q] = T(h->toi);
  if (sub) sub[q] = h->sub;
  if (normal) for (int i = 0; i < D; ++i) normal[q * D + i] = float(h->normal[i]);
  if (point) for (int i = 0; i < D; ++i) point[q * D + i] = float(h->point[i]);
}

template <int D, class S, class T>
void store_list(const std::vector<Hit<D, S>>& hits, size_t q, uint32_t k, uint32_t* count, uint32_t* leaf, T* toi,
                float* normal, uint32_t* sub) {
  count[q] = uint32_t(hits.size());
  for (uint32_t j = 0; j < k; ++j) {
    size_t o = q * k + j;
    if (j < hits.size()) {
      leaf[o] = hits[j].leaf;
      if (toi) toi[o] = T(hits[j].toi);
      if (sub) sub[o] = hits[j].sub;
      if (normal) for (int i = 0; i < D; ++i) normal[o * D + i] = float(hits[j].normal[i]);
    } else {
      leaf[o] = kNoHit;
      if (toi) toi[o] = T(0);
      if (sub) sub[o] = kNoSub;
      if (normal) for (int i = 0; i < D; ++i) normal[o * D + i] = 0.f;
    }
  }
}

template <int D, class S>
SceneBase* scene_new(int kind, uint32_t n, const float* data, const uint64_t* layers, const uint32_t* sub) {
  auto* s = new SceneImpl<D, S>();
  s->dim = D;
  s->prec = sizeof(S) * 8;
  s->g.kind = kind;
  s->g.n = n;
  uint32_t st = s->g.stride();
  s->g.data.assign(size_t(n) * st, S(0));
  for (size_t i = 0; i < size_t(n) * st; ++i) s->g.data[i] = S(data[i]);
  if (layers) { s->g.layers.assign(layers, layers + n); s->g.acc.layers = s->g.layers.data(); }
  if (sub) s->g.sub.assign(sub, sub + n);
  s->bvh.build(s->g);
  return s;
}

#define DISPATCH_D(D, ...)                              \
  switch (D) {                                          \
    case 2: { constexpr int DD = 2; __VA_ARGS__; } break; \
    case 3: { constexpr int DD = 3; __VA_ARGS__; } break; \
    case 4: { constexpr int DD = 4; __VA_ARGS__; } break; \
    case 5: { constexpr int DD = 5; __VA_ARGS__; } break; \
    case 6: { constexpr int DD = 6; __VA_ARGS__; } break; \
    case 8: { constexpr int DD = 8; __VA_ARGS__; } break; \
    default: return -1;                                 \
  }

}  // namespace

extern "C" {

int orc_version() { return 1; }

// -- single-level scenes ---------------------------------------------------

// Builds the provider and its Bvh (bvh.rs:31-38). prec = 32 or 64 (the
// crate's f64 feature); layers/sub may be NULL.
void* orc_scene_new(int D, int prec, int kind, uint32_t n, const float* data, const uint64_t* layers,
                    const uint32_t* sub) {
  if (kind == kTris && D != 3) return nullptr;
  SceneBase* out = nullptr;
  auto make = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(D, out = scene_new<DD, S>(kind, n, data, layers, sub));
    return 0;
  };
  if (prec == 64) make(double{}); else make(float{});
  return out;
}

void orc_scene_free(void* h) { delete static_cast<SceneBase*>(h); }

// Replaces the leaf parameters and refits (bvh.rs:45-48).
int orc_scene_refit(void* h, const float* data) {
  auto* b = static_cast<SceneBase*>(h);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* s = static_cast<SceneImpl<DD, S>*>(b);
      for (size_t i = 0; i < s->g.data.size(); ++i) s->g.data[i] = S(data[i]);
      s->bvh.refit(s->g);
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

uint32_t orc_scene_node_count(void* h) {
  auto* b = static_cast<SceneBase*>(h);
  uint32_t n = 0;
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, n = uint32_t(static_cast<SceneImpl<DD, S>*>(b)->bvh.nodes.size()));
    return 0;
  };
  b->prec == 64 ? run(double{}) : run(float{});
  return n;
}

// Exports the tree (tree.rs:21-26): bounds as min[D], max[D] per node.
int orc_scene_tree(void* h, float* bounds, uint32_t* child_a, uint32_t* child_b, uint32_t* prim_count,
                   uint32_t* prim_indices) {
  auto* b = static_cast<SceneBase*>(h);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* s = static_cast<SceneImpl<DD, S>*>(b);
      for (size_t i = 0; i < s->bvh.nodes.size(); ++i) {
        const auto& nd = s->bvh.nodes[i];
        for (int k = 0; k < DD; ++k) {
          bounds[i * 2 * DD + k] = float(nd.bounds.min[k]);
          bounds[i * 2 * DD + DD + k] = float(nd.bounds.max[k]);
        }
        child_a[i] = nd.child_a; child_b[i] = nd.child_b; prim_count[i] = nd.prim_count;
      }
      for (size_t i = 0; i < s->bvh.prim_indices.size(); ++i) prim_indices[i] = s->bvh.prim_indices[i];
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// TreeStats (bvh.rs:478-489): out = node_count, leaf_count, prim_count, max_depth; quality separately.
int orc_scene_stats(void* h, uint64_t* out4, double* quality) {
  auto* b = static_cast<SceneBase*>(h);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* s = static_cast<SceneImpl<DD, S>*>(b);
      size_t l, p, d;
      tree_structural(s->bvh.nodes, &l, &p, &d);
      out4[0] = s->bvh.nodes.size(); out4[1] = l; out4[2] = p; out4[3] = d;
      *quality = double(interior_surface_sum(s->bvh.nodes));
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// Nearest ray hits. mode 0 = Bvh (bvh.rs:73-124), 1 = naive scan (naive.rs:34-62).
// max_toi_arr (per query) overrides max_toi when non-NULL. toi is f32 for a
// 32-bit scene; for a 64-bit scene pass toi64 instead.
int orc_nearest(void* h, int mode, uint32_t nq, const float* rays, const float* max_toi_arr, float max_toi,
                uint64_t mask, int64_t exclude, int threads, uint32_t* leaf, float* toi, double* toi64, float* normal,
                float* point, uint32_t* sub, uint64_t* stats) {
  auto* b = static_cast<SceneBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* s = static_cast<SceneImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        for (size_t q = lo; q < hi; ++q) {
          Ray<DD, S> ray = load_ray<DD, S>(rays + q * 2 * DD);
          S mt = S(max_toi_arr ? max_toi_arr[q] : max_toi);
          QueryStats st;
          auto hit = mode == 0 ? s->bvh.nearest(s->g, ray, mt, f, stats ? &st : nullptr)
                               : naive::nearest<DD, S>(s->g, ray, mt, f);
          if (toi64) store_hit<DD, S, double>(hit, q, leaf, toi64, normal, point, sub);
          else store_hit<DD, S, float>(hit, q, leaf, toi, normal, point, sub);
          if (stats) {
            stats[q * 4 + 0] = st.nodes_visited; stats[q * 4 + 1] = st.aabb_tests;
            stats[q * 4 + 2] = st.narrow_tests; stats[q * 4 + 3] = st.hits;
          }
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// All hits (crossings = 0, bvh.rs:218-259) or all crossings (crossings = 1,
// bvh.rs:286-328), sorted by hit_ordering; the first k per query are stored
// and count[q] is the full number.
int orc_all(void* h, int mode, int crossings, uint32_t nq, const float* rays, const float* max_toi_arr, float max_toi,
            uint64_t mask, int64_t exclude, int threads, uint32_t k, uint32_t* count, uint32_t* leaf, float* toi,
            double* toi64, float* normal, uint32_t* sub, uint64_t* stats) {
  auto* b = static_cast<SceneBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* s = static_cast<SceneImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        std::vector<Hit<DD, S>> hits;
        for (size_t q = lo; q < hi; ++q) {
          Ray<DD, S> ray = load_ray<DD, S>(rays + q * 2 * DD);
          S mt = S(max_toi_arr ? max_toi_arr[q] : max_toi);
          QueryStats st;
          if (mode == 0) s->bvh.all(s->g, ray, mt, f, crossings != 0, hits, stats ? &st : nullptr);
          else naive::all<DD, S>(s->g, ray, mt, f, crossings != 0, hits);
          if (toi64) store_list<DD, S, double>(hits, q, k, count, leaf, toi64, normal, sub);
          else store_list<DD, S, float>(hits, q, k, count, leaf, toi, normal, sub);
          if (stats) {
            stats[q * 4 + 0] = st.nodes_visited; stats[q * 4 + 1] = st.aabb_tests;
            stats[q * 4 + 2] = st.narrow_tests; stats[q * 4 + 3] = st.hits;
          }
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// Nearest shape cast (bvh.rs:331-375 / naive.rs:131-158).
int orc_shapecast_nearest(void* h, int mode, uint32_t nq, const float* casts, const float* max_toi_arr, float max_toi,
                          uint64_t mask, int64_t exclude, int threads, uint32_t* leaf, float* toi, double* toi64,
                          float* normal, float* point, uint32_t* sub) {
  auto* b = static_cast<SceneBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* s = static_cast<SceneImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        for (size_t q = lo; q < hi; ++q) {
          ShapeCast<DD, S> c = load_cast<DD, S>(casts + q * 4 * DD);
          S mt = S(max_toi_arr ? max_toi_arr[q] : max_toi);
          auto hit = mode == 0 ? s->bvh.shapecast_nearest(s->g, c, mt, f) : naive::shapecast_nearest<DD, S>(s->g, c, mt, f);
          if (toi64) store_hit<DD, S, double>(hit, q, leaf, toi64, normal, point, sub);
          else store_hit<DD, S, float>(hit, q, leaf, toi, normal, point, sub);
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// All shape-cast contacts (bvh.rs:378-414 / naive.rs:161-181).
int orc_shapecast_all(void* h, int mode, uint32_t nq, const float* casts, const float* max_toi_arr, float max_toi,
                      uint64_t mask, int64_t exclude, int threads, uint32_t k, uint32_t* count, uint32_t* leaf,
                      float* toi, double* toi64, float* normal, uint32_t* sub) {
  auto* b = static_cast<SceneBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* s = static_cast<SceneImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        std::vector<Hit<DD, S>> hits;
        for (size_t q = lo; q < hi; ++q) {
          ShapeCast<DD, S> c = load_cast<DD, S>(casts + q * 4 * DD);
          S mt = S(max_toi_arr ? max_toi_arr[q] : max_toi);
          if (mode == 0) s->bvh.shapecast_all(s->g, c, mt, f, hits);
          else naive::shapecast_all<DD, S>(s->g, c, mt, f, hits);
          if (toi64) store_list<DD, S, double>(hits, q, k, count, leaf, toi64, normal, sub);
          else store_list<DD, S, float>(hits, q, k, count, leaf, toi, normal, sub);
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// Overlap (bvh.rs:418-456 / naive.rs:184-205), as CSR: call with leaves = NULL
// to get counts, then with offsets (nq + 1 entries, exclusive prefix sum) and
// leaves to fill. Each query's leaves are in ascending order.
int orc_overlap(void* h, int mode, uint32_t nq, const float* regions, uint64_t mask, int64_t exclude, int threads,
                uint32_t* counts, const uint64_t* offsets, uint32_t* leaves) {
  auto* b = static_cast<SceneBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* s = static_cast<SceneImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        std::vector<uint32_t> out;
        for (size_t q = lo; q < hi; ++q) {
          Aabb<DD, S> r = load_box<DD, S>(regions + q * 2 * DD);
          if (mode == 0) s->bvh.overlap(s->g, r, f, out);
          else naive::overlap<DD, S>(s->g, r, f, out);
          if (counts) counts[q] = uint32_t(out.size());
          if (leaves && offsets) for (size_t j = 0; j < out.size(); ++j) leaves[offsets[q] + j] = out[j];
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// The product's device layout decisions are checked against these free
// functions of the maths layer.
int orc_ray_intersect(int D, const float* box, const float* ray, float max_toi, float* t_enter, float* t_exit) {
  int ok = 0;
  DISPATCH_D(D, {
    Aabb<DD, float> a = load_box<DD, float>(box);
    Ray<DD, float> r = load_ray<DD, float>(ray);
    ok = a.ray_intersect(r, max_toi, t_enter, t_exit) ? 1 : 0;
  });
  return ok;
}

// Ray::new (ray.rs:18-23): normalises n directions in place (point.rs:82-89).
int orc_normalize(int D, uint32_t n, float* vecs) {
  DISPATCH_D(D, {
    for (size_t q = 0; q < n; ++q) {
      Point<DD, float> p;
      for (int i = 0; i < DD; ++i) p[i] = vecs[q * DD + i];
      p = p.normalize_or_zero();
      for (int i = 0; i < DD; ++i) vecs[q * DD + i] = p[i];
    }
  });
  return 0;
}

// -- two-level scenes --------------------------------------------------------

// A set of triangle-mesh BLASes: tri_offsets has n_blas + 1 entries (in
// triangles); tris holds 9 floats per triangle. Each mesh gets its own Bvh.
void* orc_blas_set_new(int prec, uint32_t n_blas, const uint64_t* tri_offsets, const float* tris) {
  auto build = [&](auto tag) -> BlasSetBase* {
    using S = decltype(tag);
    auto* set = new BlasSetImpl<S>();
    set->v.resize(n_blas);
    for (uint32_t b = 0; b < n_blas; ++b) {
      Blas<S>& bl = set->v[b];
      uint64_t t0 = tri_offsets[b], t1 = tri_offsets[b + 1];
      bl.soup.kind = kTris;
      bl.soup.n = uint32_t(t1 - t0);
      bl.soup.data.resize(size_t(t1 - t0) * 9);
      for (size_t i = 0; i < bl.soup.data.size(); ++i) bl.soup.data[i] = S(tris[t0 * 9 + i]);
      bl.bvh.build(bl.soup);
      bl.aabb = bl.bvh.nodes.empty() ? Aabb<3, S>::empty() : bl.bvh.nodes[0].bounds;
    }
    return set;
  };
  return prec == 64 ? build(double{}) : build(float{});
}

void orc_blas_set_free(void* h) { delete static_cast<BlasSetBase*>(h); }

// Instances: rot = n*D*D row-major, trans = n*D, param = scale (mesh, n),
// half-extents (box, n*D) or radius (ball, n). blas may be NULL for box/ball.
void* orc_tlas_new(int D, int prec, int kind, uint32_t n, const float* rot, const float* trans, const float* param,
                   const uint32_t* blas_id, void* blas, const uint64_t* layers, const uint32_t* sub) {
  if (kind == kInstMesh && (D != 3 || !blas)) return nullptr;
  TlasBase* out = nullptr;
  auto make = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(D, {
      auto* t = new TlasImpl<DD, S>();
      t->dim = DD;
      t->prec = sizeof(S) * 8;
      t->sc.kind = kind;
      t->sc.iso.resize(n);
      for (size_t i = 0; i < n; ++i) {
        for (int r = 0; r < DD; ++r) for (int c = 0; c < DD; ++c) t->sc.iso[i].rot[r][c] = S(rot[i * DD * DD + r * DD + c]);
        for (int r = 0; r < DD; ++r) t->sc.iso[i].translation[r] = S(trans[i * DD + r]);
      }
      size_t np = kind == kInstBox ? size_t(n) * DD : size_t(n);
      t->sc.param.resize(np);
      for (size_t i = 0; i < np; ++i) t->sc.param[i] = S(param[i]);
      if (blas_id) t->sc.blas_id.assign(blas_id, blas_id + n);
      if (blas) t->sc.blas = &static_cast<BlasSetImpl<S>*>(static_cast<BlasSetBase*>(blas))->v;
      if (layers) { t->sc.layers.assign(layers, layers + n); t->sc.acc.layers = t->sc.layers.data(); }
      if (sub) t->sc.sub.assign(sub, sub + n);
      t->tlas.build(t->sc);
      out = t;
    });
    return 0;
  };
  if (prec == 64) make(double{}); else make(float{});
  return out;
}

void orc_tlas_free(void* h) { delete static_cast<TlasBase*>(h); }

// New transforms (and optionally new per-instance parameters: a deforming
// provider) for every instance, then Tlas::refit (tlas.rs:49-54). rot and
// param may be NULL to keep them.
int orc_tlas_refit(void* h, const float* rot, const float* trans, const float* param) {
  auto* b = static_cast<TlasBase*>(h);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* t = static_cast<TlasImpl<DD, S>*>(b);
      for (size_t i = 0; i < t->sc.iso.size(); ++i) {
        if (rot) for (int r = 0; r < DD; ++r) for (int c = 0; c < DD; ++c) t->sc.iso[i].rot[r][c] = S(rot[i * DD * DD + r * DD + c]);
        for (int r = 0; r < DD; ++r) t->sc.iso[i].translation[r] = S(trans[i * DD + r]);
      }
      if (param) for (size_t i = 0; i < t->sc.param.size(); ++i) t->sc.param[i] = S(param[i]);
      t->tlas.refit(t->sc);
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// Rebuilds the tree from the current transforms (Tlas::build).
int orc_tlas_rebuild(void* h) {
  auto* b = static_cast<TlasBase*>(h);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, { auto* t = static_cast<TlasImpl<DD, S>*>(b); t->tlas.build(t->sc); });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

int orc_tlas_needs_rebuild(void* h, float factor) {
  auto* b = static_cast<TlasBase*>(h);
  int r = 0;
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, r = static_cast<TlasImpl<DD, S>*>(b)->tlas.needs_rebuild(S(factor)) ? 1 : 0);
    return 0;
  };
  b->prec == 64 ? run(double{}) : run(float{});
  return r;
}

uint32_t orc_tlas_node_count(void* h) {
  auto* b = static_cast<TlasBase*>(h);
  uint32_t n = 0;
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, n = uint32_t(static_cast<TlasImpl<DD, S>*>(b)->tlas.nodes.size()));
    return 0;
  };
  b->prec == 64 ? run(double{}) : run(float{});
  return n;
}

int orc_tlas_tree(void* h, float* bounds, uint32_t* child_a, uint32_t* child_b, uint32_t* prim_count,
                  uint32_t* indices, float* world_aabbs) {
  auto* b = static_cast<TlasBase*>(h);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* t = static_cast<TlasImpl<DD, S>*>(b);
      for (size_t i = 0; i < t->tlas.nodes.size(); ++i) {
        const auto& nd = t->tlas.nodes[i];
        for (int k = 0; k < DD; ++k) {
          bounds[i * 2 * DD + k] = float(nd.bounds.min[k]);
          bounds[i * 2 * DD + DD + k] = float(nd.bounds.max[k]);
        }
        child_a[i] = nd.child_a; child_b[i] = nd.child_b; prim_count[i] = nd.prim_count;
      }
      for (size_t i = 0; i < t->tlas.indices.size(); ++i) indices[i] = t->tlas.indices[i];
      if (world_aabbs)
        for (size_t i = 0; i < t->tlas.world.size(); ++i)
          for (int k = 0; k < DD; ++k) {
            world_aabbs[i * 2 * DD + k] = float(t->tlas.world[i].min[k]);
            world_aabbs[i * 2 * DD + DD + k] = float(t->tlas.world[i].max[k]);
          }
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// mode 0 = Tlas (tlas.rs:104-154), 1 = naive instance scan (tests/two_level.rs:134-154).
int orc_tlas_nearest(void* h, int mode, uint32_t nq, const float* rays, const float* max_toi_arr, float max_toi,
                     uint64_t mask, int64_t exclude, int threads, uint32_t* leaf, float* toi, double* toi64,
                     float* normal, float* point, uint32_t* sub, uint64_t* stats) {
  auto* b = static_cast<TlasBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* t = static_cast<TlasImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        for (size_t q = lo; q < hi; ++q) {
          Ray<DD, S> ray = load_ray<DD, S>(rays + q * 2 * DD);
          S mt = S(max_toi_arr ? max_toi_arr[q] : max_toi);
          QueryStats st;
          auto hit = mode == 0 ? t->tlas.nearest(t->sc, ray, mt, f, stats ? &st : nullptr)
                               : inst_naive_nearest<DD, S>(t->sc, ray, mt, f);
          if (toi64) store_hit<DD, S, double>(hit, q, leaf, toi64, normal, point, sub);
          else store_hit<DD, S, float>(hit, q, leaf, toi, normal, point, sub);
          if (stats) {
            stats[q * 4 + 0] = st.nodes_visited; stats[q * 4 + 1] = st.aabb_tests;
            stats[q * 4 + 2] = st.narrow_tests; stats[q * 4 + 3] = st.hits;
          }
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

int orc_tlas_all(void* h, int crossings, uint32_t nq, const float* rays, const float* max_toi_arr, float max_toi,
                 uint64_t mask, int64_t exclude, int threads, uint32_t k, uint32_t* count, uint32_t* leaf, float* toi,
                 float* normal, uint32_t* sub) {
  auto* b = static_cast<TlasBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* t = static_cast<TlasImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        std::vector<Hit<DD, S>> hits;
        for (size_t q = lo; q < hi; ++q) {
          Ray<DD, S> ray = load_ray<DD, S>(rays + q * 2 * DD);
          S mt = S(max_toi_arr ? max_toi_arr[q] : max_toi);
          t->tlas.all(t->sc, ray, mt, f, crossings != 0, hits, nullptr);
          store_list<DD, S, float>(hits, q, k, count, leaf, toi, normal, sub);
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

int orc_tlas_shapecast_nearest(void* h, uint32_t nq, const float* casts, const float* max_toi_arr, float max_toi,
                               uint64_t mask, int64_t exclude, int threads, uint32_t* leaf, float* toi, float* normal,
                               float* point, uint32_t* sub) {
  auto* b = static_cast<TlasBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* t = static_cast<TlasImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        for (size_t q = lo; q < hi; ++q) {
          ShapeCast<DD, S> c = load_cast<DD, S>(casts + q * 4 * DD);
          S mt = S(max_toi_arr ? max_toi_arr[q] : max_toi);
          store_hit<DD, S, float>(t->tlas.shapecast_nearest(t->sc, c, mt, f), q, leaf, toi, normal, point, sub);
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

int orc_tlas_shapecast_all(void* h, uint32_t nq, const float* casts, const float* max_toi_arr, float max_toi,
                           uint64_t mask, int64_t exclude, int threads, uint32_t k, uint32_t* count, uint32_t* leaf,
                           float* toi, float* normal, uint32_t* sub) {
  auto* b = static_cast<TlasBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* t = static_cast<TlasImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        std::vector<Hit<DD, S>> hits;
        for (size_t q = lo; q < hi; ++q) {
          ShapeCast<DD, S> c = load_cast<DD, S>(casts + q * 4 * DD);
          S mt = S(max_toi_arr ? max_toi_arr[q] : max_toi);
          t->tlas.shapecast_all(t->sc, c, mt, f, hits);
          store_list<DD, S, float>(hits, q, k, count, leaf, toi, normal, sub);
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

int orc_tlas_overlap(void* h, uint32_t nq, const float* regions, uint64_t mask, int64_t exclude, int threads,
                     uint32_t* counts, const uint64_t* offsets, uint32_t* leaves) {
  auto* b = static_cast<TlasBase*>(h);
  Filter f = make_filter(mask, exclude);
  auto run = [&](auto tag) -> int {
    using S = decltype(tag);
    DISPATCH_D(b->dim, {
      auto* t = static_cast<TlasImpl<DD, S>*>(b);
      parallel_chunks(nq, threads, [&](size_t lo, size_t hi) {
        std::vector<uint32_t> out;
        for (size_t q = lo; q < hi; ++q) {
          Aabb<DD, S> r = load_box<DD, S>(regions + q * 2 * DD);
          t->tlas.overlap(t->sc, r, f, out);
          if (counts) counts[q] = uint32_t(out.size());
          if (leaves && offsets) for (size_t j = 0; j < out.size(); ++j) leaves[offsets[q] + j] = out[j];
        }
      });
    });
    return 0;
  };
  return b->prec == 64 ? run(double{}) : run(float{});
}

// Isometry helpers for tests (isometry.rs:58-97): op 0 transform_vector,
// 1 inverse_transform_vector, 2 transform_point, 3 inverse_transform_point.
int orc_iso_apply(int D, const float* rot, const float* trans, int op, const float* in, float* out) {
  DISPATCH_D(D, {
    Isometry<DD, float> iso;
    for (int r = 0; r < DD; ++r) for (int c = 0; c < DD; ++c) iso.rot[r][c] = rot[r * DD + c];
    for (int r = 0; r < DD; ++r) iso.translation[r] = trans[r];
    Point<DD, float> p; for (int i = 0; i < DD; ++i) p[i] = in[i];
    Point<DD, float> q = op == 0 ? iso.transform_vector(p) : op == 1 ? iso.inverse_transform_vector(p)
                       : op == 2 ? iso.transform_point(p) : iso.inverse_transform_point(p);
    for (int i = 0; i < DD; ++i) out[i] = q[i];
  });
  return 0;
}

int orc_iso_transform_aabb(int D, const float* rot, const float* trans, const float* box, float* out) {
  DISPATCH_D(D, {
    Isometry<DD, float> iso;
    for (int r = 0; r < DD; ++r) for (int c = 0; c < DD; ++c) iso.rot[r][c] = rot[r * DD + c];
    for (int r = 0; r < DD; ++r) iso.translation[r] = trans[r];
    Aabb<DD, float> a = iso.transform_aabb(load_box<DD, float>(box));
    for (int i = 0; i < DD; ++i) { out[i] = a.min[i]; out[DD + i] = a.max[i]; }
  });
  return 0;
}

}  // extern "C"
