/*
 * sq.h -- C ABI of the B200 batched-query library (libsqcuda.so).
 *
 * This is the boundary a host binding links against in place of the
 * spatial-query crate's `gpu` feature (crates/spatial-query/src/gpu/mod.rs).
 * Every entry point takes plain pointers and sizes; none takes or returns a
 * Rust, C++ or torch type. Entry points return an int32 status (SQ_OK = 0);
 * the message of the last failure on a context is sq_ctx_last_error(). No
 * entry point unwinds or aborts across the boundary.
 *
 * Conventions shared by every query:
 *   D        the dimension of the uploaded tree (2, 3, 4 or 6).
 *   ray      origin[D], dir[D] as floats (dir unit length: the crate's
 *            `Ray::new` normalises on the host, maths/ray.rs:18-23).
 *   cast     origin[D], dir[D], probe_min[D], probe_max[D]
 *            (query/shapecast.rs:26-40: the probe box as offsets).
 *   region   min[D], max[D] (maths/aabb.rs:8-12).
 *   leaf     the provider leaf index 0..leaf_count; SQ_NO_HIT when none.
 *   results  bit-identical to the reference CPU path (accel/bvh.rs,
 *            accel/tlas.rs): the same leaf, the same f32 time of impact, the
 *            same (toi, leaf) total order (query/hit.rs:77-84).
 *
 * Host-buffer entry points copy inputs in and results out on the context's
 * stream and return when the results are in host memory. Nearest calls of
 * 524,288 queries or more (sq_raycast_nearest, sq_shapecast_nearest,
 * sq_raycast_nearest_guided) without stats run in two or four chunks: rays
 * copied in and hits copied out on two internal copy streams while chunks
 * are walked, alternately on the context's stream and on a second internal
 * context (its own stream and scratch, same settings); all of them have
 * settled when the call returns. Host buffers in page-locked memory let the
 * copies overlap. The `_d` variants take device pointers, enqueue on the
 * context's stream and return at once.
 *
 * Threading: a context is used by one host thread at a time; uploaded scenes
 * may be shared by contexts on the same device.
 */
#ifndef SQ_H
#define SQ_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define SQ_OK 0
#define SQ_ERR_INVALID 1      /* a bad argument: size, pointer, dimension, tree shape */
#define SQ_ERR_CUDA 2         /* a CUDA runtime failure (message in sq_ctx_last_error) */
#define SQ_ERR_NO_DEVICE 3    /* no CUDA device (the `headless` -> None case, gpu/mod.rs:308-324) */
#define SQ_ERR_UNSUPPORTED 4  /* a dimension / narrow-phase pair this build has no kernel for */
#define SQ_ERR_DEPTH 5        /* the tree is deeper than the traversal stack */
#define SQ_ERR_CAPACITY 6     /* an output buffer is too small; the needed size is reported */
#define SQ_ERR_COMPILE 7      /* a consumer narrow phase failed to compile */

#define SQ_NO_HIT 0xFFFFFFFFu /* leaf of a query with no hit */
#define SQ_NO_SUB 0xFFFFFFFFu /* sub-object `None` (query/hit.rs:36-40) */

/* Built-in narrow phases (the providers' QueryGeometry::test_ray etc.). */
#define SQ_NARROW_AABB 0        /* leaf = box min[D],max[D]; hit = slab entry (maths/aabb.rs:118-148) */
#define SQ_NARROW_SPHERE 1      /* leaf = centre[D],radius; near root, far root from inside (tests/differential.rs:61-82) */
#define SQ_NARROW_SPHERE_NEAR 2 /* leaf = centre[D],radius; near root only (tests/gpu.rs:92-106) */
#define SQ_NARROW_TRIANGLE 3    /* leaf = v0,v1,v2 (D = 3); Moeller-Trumbore (viewport-lib-query/src/lib.rs:281-306) */
#define SQ_NARROW_CUSTOM 4      /* a consumer narrow phase compiled at run time (sq_bvh_upload_custom) */

/* Traversal order of nearest queries (sq_ctx_set_order). */
#define SQ_ORDER_NEAR_FIRST 0   /* the default: visit the child with the smaller slab entry first; an answer
                                   that is not certified order-independent is recomputed in the reference
                                   order by a second launch */
#define SQ_ORDER_REFERENCE 1    /* the crate's own order (accel/bvh.rs:119-120), replaying the CPU's
                                   decisions step for step (QueryStats counters included) */

/* Node records walked by near-first nearest rays (sq_ctx_set_layout); both
 * give the reference's answers. */
#define SQ_LAYOUT_BINARY 0      /* the default: child-pair records, both children of a node in one record */
#define SQ_LAYOUT_WIDE 1        /* four-wide records (the binary tree with every other level folded into
                                   its parent): half the dependent fetches per ray, twice the boxes per
                                   fetch; the autotuner picks it where it is faster */
#define SQ_LAYOUT_QUANT 2       /* the four-wide records quantised: each child box as 8-bit steps from
                                   the record's corner, rounded outward (64 B per record at D = 3, as a
                                   child-pair record); the exact records serve scenes with non-finite
                                   bounds */
#define SQ_LAYOUT_BINARY_REGTOP 3 /* child-pair records walked with postponed leaves (a lane that reaches a
                                   leaf keeps descending until its warp holds leaves) and the stack's top
                                   entry in registers, older entries spilling to the shared-memory stack */
#define SQ_LAYOUT_BINARY_VOTE 4 /* child-pair records, child order by warp vote: the lanes opening the same
                                   record with both children hit take the order most of them prefer */

typedef struct sq_ctx sq_ctx;
typedef struct sq_bvh sq_bvh;

/* QueryFilter (query/filter.rs:12-29). Honoured when the scene was uploaded
 * with per-leaf layers: a leaf is accepted when layers[leaf] & layer_mask is
 * non-zero and leaf != exclude. Without layers every leaf is accepted (the
 * QueryGeometry::accepts default, query/geometry.rs:95-97). NULL = default. */
typedef struct sq_filter {
  uint64_t layer_mask; /* default: all bits */
  int64_t exclude;     /* a leaf index, or -1 for none */
} sq_filter;

/* One result per query (GpuHit, gpu/mod.rs:104-114, plus the sub-object).
 * Any pointer but `leaf` may be NULL to skip that output. */
typedef struct sq_hits {
  uint32_t* leaf;       /* [n] SQ_NO_HIT when nothing was hit */
  float* toi;           /* [n] */
  uint32_t* sub_object; /* [n] the per-leaf sub-object given at upload, SQ_NO_SUB if none */
  float* normal;        /* [n*D] */
  float* point;         /* [n*D] origin + dir * toi, no FMA (maths/ray.rs:33-35) */
} sq_hits;

/* Bounded sorted hit lists (raycast_all / shapecast_all): count[q] is the full
 * number of hits, the first min(count[q], k) entries of query q are stored in
 * hit order at [q*k ...]; entries past that are left untouched. */
typedef struct sq_hit_lists {
  uint32_t k;
  uint32_t* count;      /* [n] */
  uint32_t* leaf;       /* [n*k] */
  float* toi;           /* [n*k] */
  uint32_t* sub_object; /* [n*k] or NULL */
  float* normal;        /* [n*k*D] or NULL */
} sq_hit_lists;

/* QueryStats (accel/stats.rs:41-50), summed over the batch. */
typedef struct sq_query_stats {
  uint64_t nodes_visited;
  uint64_t aabb_tests;
  uint64_t narrow_tests;
  uint64_t hits;
} sq_query_stats;

typedef struct sq_bvh_info {
  int32_t dim;
  int32_t narrow;
  uint32_t n_nodes;      /* nodes of the uploaded host tree */
  uint32_t n_prims;
  uint32_t max_depth;    /* in nodes (tree.rs:81-99) */
  uint32_t n_interior;
  uint64_t device_bytes; /* node records + primitive records + tables */
  uint32_t node_record_bytes;
  uint32_t prim_record_bytes;
} sq_bvh_info;

/* ---- context ---------------------------------------------------------------
 * Replaces GpuRaycaster::headless / new's device acquisition
 * (gpu/mod.rs:252-324): returns SQ_ERR_NO_DEVICE when there is no GPU.
 * A context owns a stream, a scratch arena and a memory pool; the stream-
 * ordered scratch of the device tree build, the overlap sort and the f64
 * host-buffer overlap comes from that pool, which keeps its memory for the
 * next call until sq_ctx_destroy. */
int32_t sq_version(void);
int32_t sq_ctx_create(int32_t device, sq_ctx** out);
int32_t sq_ctx_destroy(sq_ctx* ctx);
const char* sq_ctx_last_error(const sq_ctx* ctx);
/* The context's stream (a cudaStream_t); `stream` NULL restores its own. */
void* sq_ctx_stream(sq_ctx* ctx);
int32_t sq_ctx_set_stream(sq_ctx* ctx, void* stream);
int32_t sq_ctx_synchronize(sq_ctx* ctx);
/* Nearest-query order (SQ_ORDER_*, default SQ_ORDER_NEAR_FIRST) and
 * persistent-grid blocks per SM (0 = occupancy). */
int32_t sq_ctx_set_order(sq_ctx* ctx, int32_t order);
int32_t sq_ctx_set_layout(sq_ctx* ctx, int32_t layout);
int32_t sq_ctx_set_blocks_per_sm(sq_ctx* ctx, int32_t blocks);
/* Near-first nearest queries prune a node only when its slab entry lies more
 * than `window` (relative, default 2^-16) past the current limit, and are
 * answered again in the reference order when their answer comes before the
 * slab entry of its own primitive's AABB (the one case where the reference's
 * walk could miss it). */
int32_t sq_ctx_set_replay_window(sq_ctx* ctx, float window);
/* Keeps a scene's node records in L2 across calls: marks them as persisting
 * for kernels on the context's stream (and its internal second lane) through
 * an access-policy window (persisting on a hit, streaming on a miss), with
 * up to `bytes` of the L2 set aside for persisting lines (capped at the
 * device's maximum; hit ratio = set-aside bytes / window bytes). The
 * set-aside belongs to this process's CUDA context and ends with it. `bvh`
 * NULL or `bytes` 0 clears the window and returns persisting lines to
 * normal. Answers are unchanged; only where the records live changes. */
int32_t sq_ctx_set_l2_persist(sq_ctx* ctx, const sq_bvh* bvh, uint64_t bytes);
/* Autotuner for nearest rays on one scene: times every candidate launch
 * configuration on a sample of device-resident rays (CUDA events, best of
 * `reps`), keeps the fastest in the context and reports the table. The knobs
 * are the traversal order (near-first, certified / the reference's order,
 * both give the reference's hits), the node records and walk of near-first
 * rays (child-pair, four-wide, quantised four-wide, child-pair with the
 * register-held stack top, child-pair with the warp-vote child order) and
 * the persistent grid's resident blocks per SM (0 = the occupancy limit):
 * up to 48 entries. No counterpart in the reference, whose
 * WGSL path has a fixed 64-thread workgroup (gpu/mod.rs:119-227). */
typedef struct sq_tune_entry {
  int32_t order;
  int32_t blocks_per_sm;
  float ms;
  int32_t layout;  /* SQ_LAYOUT_* (near-first entries) */
} sq_tune_entry;
typedef struct sq_tune_result {
  uint32_t n_entries;
  sq_tune_entry entries[48];
  int32_t best;  /* index into entries */
} sq_tune_result;
int32_t sq_autotune_nearest_d(sq_ctx* ctx, const sq_bvh* bvh, const float* d_rays, uint32_t n, float max_toi,
                              uint32_t reps, sq_tune_result* out);
/* Kernels this context has launched so far. */
uint64_t sq_ctx_launch_count(const sq_ctx* ctx);
/* How many queries of the last near-first launch were answered again, in the
 * same launch, in the reference order because their answer could depend on
 * the visiting order (waits for the context's stream). */
int32_t sq_ctx_last_replay_count(sq_ctx* ctx, uint32_t* out);

/* ---- host tree build -------------------------------------------------------
 * tree::build (accel/tree.rs:39-49, 112-163): the median-split tree the
 * crate's Bvh::build / Tlas::build make, for callers without the Rust crate.
 * prim_aabbs is n * 2D floats (min, max); outputs need capacity for
 * max(2n - 1, 0) nodes; node_bounds is n_nodes * 2D. threads <= 0: all cores. */
int32_t sq_tree_build(int32_t dim, uint32_t n, const float* prim_aabbs, int32_t threads, uint32_t node_capacity,
                      uint32_t* n_nodes_out, float* node_bounds, uint32_t* child_a, uint32_t* child_b,
                      uint32_t* prim_count, uint32_t* prim_indices);

/* The same tree built on the device: d_prim_aabbs and every output are device
 * pointers (same layouts and capacity rule as sq_tree_build), the arrays equal
 * sq_tree_build's (bounds compare equal; a zero bound may differ in sign,
 * which f32::min / max leave unspecified). Runs on the context's stream and
 * returns once the tree is complete; *n_nodes_out is the node count. A
 * per-frame rebuild (Tlas::needs_rebuild, accel/tlas.rs:58-60) no longer
 * needs the host. */
int32_t sq_tree_build_d(sq_ctx* ctx, int32_t dim, uint32_t n, const float* d_prim_aabbs, uint32_t node_capacity,
                        uint32_t* n_nodes_out, float* d_node_bounds, uint32_t* d_child_a, uint32_t* d_child_b,
                        uint32_t* d_prim_count, uint32_t* d_prim_indices);

/* The world AABB of each built-in leaf (the providers' world_aabb). */
int32_t sq_prim_aabbs(int32_t dim, int32_t narrow, uint32_t n, const float* prim_data, float* out_aabbs);

/* ---- the crate's f64 feature (Scalar = f64, maths/point.rs:14-18) ---------
 * The same tree and leaf AABBs in double precision (centroids, EPSILON and
 * total_cmp of f64), for scenes uploaded with sq_bvh_upload_f64. */
int32_t sq_tree_build_f64(int32_t dim, uint32_t n, const double* prim_aabbs, int32_t threads, uint32_t node_capacity,
                          uint32_t* n_nodes_out, double* node_bounds, uint32_t* child_a, uint32_t* child_b,
                          uint32_t* prim_count, uint32_t* prim_indices);
int32_t sq_prim_aabbs_f64(int32_t dim, int32_t narrow, uint32_t n, const double* prim_data, double* out_aabbs);
/* An f64 scene: the host tree (tree::Node arrays with double bounds) and
 * double leaf parameters (built-in narrow phases, same layouts as
 * sq_bvh_upload); layers optional. It answers only the _f64 queries; the f32
 * entry points return SQ_ERR_UNSUPPORTED for it. */
int32_t sq_bvh_upload_f64(sq_ctx* ctx, int32_t dim, int32_t narrow, uint32_t n_nodes, const double* node_bounds,
                          const uint32_t* child_a, const uint32_t* child_b, const uint32_t* prim_count,
                          uint32_t n_prims, const uint32_t* prim_indices, const double* prim_data,
                          uint32_t prim_stride, const uint64_t* layers, sq_bvh** out);
/* Bvh::raycast_nearest with Scalar = f64 (accel/bvh.rs:73-124), walked in the
 * crate's own order: leaf, toi and normal (D doubles) equal the f64 CPU
 * path's, and so do the QueryStats counters (stats may be NULL). A miss gives
 * SQ_NO_HIT, toi 0 and a zero normal. toi / normal may be NULL. */
int32_t sq_raycast_nearest_f64(sq_ctx* ctx, const sq_bvh* bvh, const double* rays, uint32_t n, double max_toi,
                               const double* max_toi_per_query, const sq_filter* filter, uint32_t* leaf,
                               double* toi, double* normal, sq_query_stats* stats);
int32_t sq_raycast_nearest_f64_d(sq_ctx* ctx, const sq_bvh* bvh, const double* d_rays, uint32_t n, double max_toi,
                                 const double* d_max_toi_per_query, const sq_filter* filter, uint32_t* d_leaf,
                                 double* d_toi, double* d_normal, sq_query_stats* stats);

/* Bounded sorted hit lists of an f64 scene (as sq_hit_lists, with double
 * toi and normals; no sub-objects: f64 scenes carry none). */
typedef struct sq_hit_lists_f64 {
  uint32_t k;
  uint32_t* count;  /* [n] full number of hits */
  uint32_t* leaf;   /* [n*k] */
  double* toi;      /* [n*k] */
  double* normal;   /* [n*k*D] or NULL */
} sq_hit_lists_f64;

/* raycast_all / raycast_crossings (accel/bvh.rs:196-328) with Scalar = f64,
 * walked in the crate's own order; crossings != 0 lists both roots of sphere
 * leaves (tests/crossings.rs:505-521), one crossing per hit otherwise. The
 * first min(count, k) entries per ray equal the f64 CPU path's sorted list. */
int32_t sq_raycast_all_f64(sq_ctx* ctx, const sq_bvh* bvh, const double* rays, uint32_t n, double max_toi,
                           const double* max_toi_per_query, const sq_filter* filter, int32_t crossings,
                           const sq_hit_lists_f64* out);
int32_t sq_raycast_all_f64_d(sq_ctx* ctx, const sq_bvh* bvh, const double* d_rays, uint32_t n, double max_toi,
                             const double* d_max_toi_per_query, const sq_filter* filter, int32_t crossings,
                             const sq_hit_lists_f64* d_out);
/* shapecast_nearest / shapecast_all (accel/bvh.rs:330-414) with Scalar = f64:
 * casts are origin[D], dir[D], probe.min[D], probe.max[D] (doubles); the same
 * narrow phases as sq_shapecast_*. */
int32_t sq_shapecast_nearest_f64(sq_ctx* ctx, const sq_bvh* bvh, const double* casts, uint32_t n, double max_toi,
                                 const double* max_toi_per_query, const sq_filter* filter, uint32_t* leaf, double* toi,
                                 double* normal);
int32_t sq_shapecast_nearest_f64_d(sq_ctx* ctx, const sq_bvh* bvh, const double* d_casts, uint32_t n, double max_toi,
                                   const double* d_max_toi_per_query, const sq_filter* filter, uint32_t* d_leaf,
                                   double* d_toi, double* d_normal);
int32_t sq_shapecast_all_f64(sq_ctx* ctx, const sq_bvh* bvh, const double* casts, uint32_t n, double max_toi,
                             const double* max_toi_per_query, const sq_filter* filter, const sq_hit_lists_f64* out);
int32_t sq_shapecast_all_f64_d(sq_ctx* ctx, const sq_bvh* bvh, const double* d_casts, uint32_t n, double max_toi,
                               const double* d_max_toi_per_query, const sq_filter* filter,
                               const sq_hit_lists_f64* d_out);
/* overlap (accel/bvh.rs:416-456) of double regions lo[D], hi[D] as CSR, as
 * sq_overlap / sq_overlap_d. */
int32_t sq_overlap_f64(sq_ctx* ctx, const sq_bvh* bvh, const double* regions, uint32_t n, const sq_filter* filter,
                       uint64_t* offsets, uint32_t* leaves, uint64_t leaf_capacity, uint64_t* total);
int32_t sq_overlap_f64_d(sq_ctx* ctx, const sq_bvh* bvh, const double* d_regions, uint32_t n, const sq_filter* filter,
                         uint64_t* d_offsets, uint32_t* d_leaves, uint64_t leaf_capacity, uint64_t* total);

/* ---- scene upload (GpuRaycaster::new, gpu/mod.rs:252-303) -------------------
 * Takes the host tree as tree::Node arrays (accel/tree.rs:21-26; Bvh::nodes
 * and Bvh::prim_indices, accel/bvh.rs:463-475) and the leaf parameters indexed
 * by leaf id (prim_stride floats each: 2D boxes, D+1 balls, 9 triangles;
 * GpuGeometry::prim_data, gpu/mod.rs:86-99). layers (u64 per leaf) and
 * sub_objects (u32 per leaf) are optional. */
int32_t sq_bvh_upload(sq_ctx* ctx, int32_t dim, int32_t narrow, uint32_t n_nodes, const float* node_bounds,
                      const uint32_t* child_a, const uint32_t* child_b, const uint32_t* prim_count, uint32_t n_prims,
                      const uint32_t* prim_indices, const float* prim_data, uint32_t prim_stride,
                      const uint64_t* layers, const uint32_t* sub_objects, sq_bvh** out);

/* A D = 3 scene whose narrow phase is the caller's own CUDA source, compiled
 * at upload time with NVRTC into the traversal kernels (the GpuGeometry
 * contract, gpu/mod.rs:69-99, where the consumer hands a WGSL `narrow`). The
 * source defines, in the library's namespace (it is wrapped in one):
 *   __device__ bool sq_narrow(const float* prim, uint32_t leaf, const float* ro,
 *                             const float* rd, float max_toi, float* toi,
 *                             float* normal);
 * prim: the leaf's prim_stride floats (1..32); return true with *toi (not
 * past max_toi) and normal[3] for a hit. The library's exact maths
 * (fadd, fmul, ray_at, ...) are in scope. prim_aabbs (min[3], max[3] per
 * leaf) are the boxes the tree was built from; each must contain its
 * leaf's hits (near-first answers are certified against them). The source
 * may also define every crossing of a leaf (QueryGeometry::
 * test_ray_crossings, query/geometry.rs), which raycast_crossings then lists:
 *   template <class Emit>
 *   __device__ void sq_narrow_crossings(const float* prim, uint32_t leaf,
 *       const float* ro, const float* rd, float max_toi, Emit& emit);
 * calling emit(toi, normal) per crossing. Ray nearest, all-hits and
 * crossings queries are supported; casts, overlaps and refit return
 * SQ_ERR_UNSUPPORTED. A source that does not compile returns SQ_ERR_COMPILE
 * with the compiler log in sq_ctx_last_error. Kernels are cached per source
 * and stride for the process. */
int32_t sq_bvh_upload_custom(sq_ctx* ctx, uint32_t n_nodes, const float* node_bounds, const uint32_t* child_a,
                             const uint32_t* child_b, const uint32_t* prim_count, uint32_t n_prims,
                             const uint32_t* prim_indices, const float* prim_data, uint32_t prim_stride,
                             const float* prim_aabbs, const char* narrow_src, sq_bvh** out);
int32_t sq_bvh_destroy(sq_bvh* bvh);
int32_t sq_bvh_info_get(const sq_bvh* bvh, sq_bvh_info* out);

/* GpuRaycaster::refit (gpu/mod.rs:333-341) with the refit itself on the
 * device: new leaf parameters (same layout as at upload), then a bottom-up
 * pass over the fixed topology (tree::refit, accel/tree.rs:54-75). */
int32_t sq_bvh_refit(sq_ctx* ctx, sq_bvh* bvh, const float* prim_data);
int32_t sq_bvh_refit_d(sq_ctx* ctx, sq_bvh* bvh, const float* d_prim_data);
/* Node bounds back in host-tree node order (n_nodes * 2D floats). */
int32_t sq_bvh_read_bounds(sq_ctx* ctx, const sq_bvh* bvh, float* node_bounds);

/* ---- queries ------------------------------------------------------------------
 * raycast_nearest: GpuRaycaster::raycast_nearest_batch (gpu/mod.rs:348-463)
 * and Bvh::raycast_nearest_batch (accel/bvh.rs:134-144). max_toi_per_query
 * (may be NULL) overrides max_toi per query. stats may be NULL. */
int32_t sq_raycast_nearest(sq_ctx* ctx, const sq_bvh* bvh, const float* rays, uint32_t n, float max_toi,
                           const float* max_toi_per_query, const sq_filter* filter, const sq_hits* out,
                           sq_query_stats* stats);
int32_t sq_raycast_nearest_d(sq_ctx* ctx, const sq_bvh* bvh, const float* d_rays, uint32_t n, float max_toi,
                             const float* d_max_toi_per_query, const sq_filter* filter, const sq_hits* d_out,
                             sq_query_stats* stats);

/* raycast_all (accel/bvh.rs:196-259), bounded to k hits per query. */
int32_t sq_raycast_all(sq_ctx* ctx, const sq_bvh* bvh, const float* rays, uint32_t n, float max_toi,
                       const float* max_toi_per_query, const sq_filter* filter, const sq_hit_lists* out,
                       sq_query_stats* stats);
int32_t sq_raycast_all_d(sq_ctx* ctx, const sq_bvh* bvh, const float* d_rays, uint32_t n, float max_toi,
                         const float* d_max_toi_per_query, const sq_filter* filter, const sq_hit_lists* d_out,
                         sq_query_stats* stats);

/* raycast_crossings (accel/bvh.rs:261-328): every entry and exit of sphere
 * leaves; every crossing a consumer narrow phase emits when its source also
 * defines sq_narrow_crossings (see sq_bvh_upload_custom); one crossing per
 * hit for the other narrow phases. */
int32_t sq_raycast_crossings(sq_ctx* ctx, const sq_bvh* bvh, const float* rays, uint32_t n, float max_toi,
                             const float* max_toi_per_query, const sq_filter* filter, const sq_hit_lists* out);
int32_t sq_raycast_crossings_d(sq_ctx* ctx, const sq_bvh* bvh, const float* d_rays, uint32_t n, float max_toi,
                               const float* d_max_toi_per_query, const sq_filter* filter, const sq_hit_lists* d_out);

/* shapecast_nearest / shapecast_all (accel/bvh.rs:330-414). The point of a
 * cast hit is cast.at(toi) (query/shapecast.rs:61-63). Narrow phases: boxes
 * are the exact swept-box test (the slab against the leaf box grown by the
 * probe, ShapeCast::broadphase, shapecast.rs:70-73); balls sweep the probe's
 * max[0] as a radius (tests/shape_overlap.rs:96-110). The reference defines
 * no swept box against a triangle, so a triangle leaf answers the swept box
 * against the triangle's AABB (the same broadphase slab, the normal of the
 * AABB face entered): a conservative time of impact, never later than the
 * exact swept-box-vs-triangle one. Mesh instances of a Tlas likewise answer
 * a cast against the instance's world AABB. */
int32_t sq_shapecast_nearest(sq_ctx* ctx, const sq_bvh* bvh, const float* casts, uint32_t n, float max_toi,
                             const float* max_toi_per_query, const sq_filter* filter, const sq_hits* out);
int32_t sq_shapecast_nearest_d(sq_ctx* ctx, const sq_bvh* bvh, const float* d_casts, uint32_t n, float max_toi,
                               const float* d_max_toi_per_query, const sq_filter* filter, const sq_hits* d_out);
int32_t sq_shapecast_all(sq_ctx* ctx, const sq_bvh* bvh, const float* casts, uint32_t n, float max_toi,
                         const float* max_toi_per_query, const sq_filter* filter, const sq_hit_lists* out);
int32_t sq_shapecast_all_d(sq_ctx* ctx, const sq_bvh* bvh, const float* d_casts, uint32_t n, float max_toi,
                           const float* d_max_toi_per_query, const sq_filter* filter, const sq_hit_lists* d_out);

/* overlap (accel/bvh.rs:416-456) as CSR: offsets[n + 1] (u64, exclusive
 * prefix) and the leaves of query q at [offsets[q], offsets[q+1]) in ascending
 * leaf order. When the total exceeds leaf_capacity the call returns
 * SQ_ERR_CAPACITY with *total and offsets filled and no leaves written. */
int32_t sq_overlap(sq_ctx* ctx, const sq_bvh* bvh, const float* regions, uint32_t n, const sq_filter* filter,
                   uint64_t* offsets, uint32_t* leaves, uint64_t leaf_capacity, uint64_t* total);
int32_t sq_overlap_d(sq_ctx* ctx, const sq_bvh* bvh, const float* d_regions, uint32_t n, const sq_filter* filter,
                     uint64_t* d_offsets, uint32_t* d_leaves, uint64_t leaf_capacity, uint64_t* total);

/* Overlap (as sq_overlap_d) without any device allocation. No counterpart in
 * the reference. For callers that may not allocate device memory at query
 * time -- an engine that owns a fixed device-memory budget and forbids
 * driver allocations, a real-time loop that cannot take an allocation's
 * latency, code with no sq_ctx to hold scratch -- it keeps its scratch (the
 * per-region counts and work counters) in one static device array of the
 * library, sized for at most 1,048,576 regions (about 4 MiB per GPU that
 * loads the library, held until the process exits). n beyond that returns
 * SQ_ERR_CAPACITY, as does a result larger than leaf_capacity (*total is then
 * set). Device pointers; runs on `stream` (a cudaStream_t, NULL = the legacy
 * default stream) and returns when the results are written: every call reads
 * the total back and waits for its stream, so it blocks the calling thread
 * and must never be called on a stream that is being captured. The first
 * call on a device also looks up the array's address on that device. Every
 * call shares the one array, so calls that overlap on the GPU (from several
 * threads or streams) race. With no
 * sort scratch, each region's leaves are kept ascending by insertion as they
 * are found: a region with k results costs O(k^2) writes (sq_overlap and
 * sq_overlap_d append, then sort every segment at once). */
int32_t sq_overlap_noalloc(const sq_bvh* bvh, const float* d_regions, uint32_t n, const sq_filter* filter,
                           uint64_t* d_offsets, uint32_t* d_leaves, uint64_t leaf_capacity, uint64_t* total,
                           void* stream);

/* ---- two-level scenes (accel/tlas.rs) -------------------------------------
 * A Tlas over instances of one kind. Mesh instances (D = 3) reference a BLAS
 * of a shared BLAS set and carry a uniform scale: the instance's local test is
 * a nearest query in the mesh tree with the origin divided by the scale and
 * max_toi / scale, the toi scaled back (the provider of the benchmark's
 * instanced scene; Isometry itself is rigid, maths/isometry.rs:14-25). Box
 * instances are the oriented boxes of tests/two_level.rs:42-113; ball
 * instances the balls of tests/shape_overlap.rs:289-342. Rays are world-space;
 * each instance maps them to local space (tlas.rs:459-481). */
#define SQ_INSTANCE_MESH 0 /* param: scale; blas_id per instance */
#define SQ_INSTANCE_BOX 1  /* param: half-extents[D] */
#define SQ_INSTANCE_BALL 2 /* param: radius */

typedef struct sq_blas_set sq_blas_set;
typedef struct sq_tlas sq_tlas;
typedef struct sq_graph sq_graph;

/* Triangle meshes, each with its host tree (Bvh::build per mesh). Trees are
 * concatenated: mesh b owns nodes [node_offsets[b], node_offsets[b+1]) with
 * child indices local to the mesh, and triangles [tri_offsets[b],
 * tri_offsets[b+1]) of `tris` (9 floats each, in mesh leaf order) with
 * prim_indices local to the mesh. A hit's sub-object is the mesh-local
 * triangle index. */
int32_t sq_blas_set_upload(sq_ctx* ctx, uint32_t n_blas, const uint32_t* node_offsets, const float* node_bounds,
                           const uint32_t* child_a, const uint32_t* child_b, const uint32_t* prim_count,
                           const uint32_t* tri_offsets, const uint32_t* prim_indices, const float* tris,
                           sq_blas_set** out);
int32_t sq_blas_set_destroy(sq_blas_set* blas);

/* World AABBs of instances (Isometry::transform_aabb of the local AABB,
 * maths/isometry.rs:84-97): the boxes Tlas::build's tree is built over
 * (tlas.rs:483-487). rot is n*D*D row-major, trans n*D. */
int32_t sq_instance_world_aabbs(int32_t dim, int32_t kind, uint32_t n, const float* rot, const float* trans,
                                const float* param, const uint32_t* blas_id, const sq_blas_set* blas,
                                float* out_aabbs);

/* Tlas::build's result uploaded (tlas.rs:35-45): the tree over the instance
 * world AABBs as tree::Node arrays and its instance order. */
int32_t sq_tlas_upload(sq_ctx* ctx, int32_t dim, int32_t kind, uint32_t n_inst, const float* rot,
                       const float* trans, const float* param, const uint32_t* blas_id, const sq_blas_set* blas,
                       uint32_t n_nodes, const float* node_bounds, const uint32_t* child_a,
                       const uint32_t* child_b, const uint32_t* prim_count, const uint32_t* inst_indices,
                       const uint64_t* layers, const uint32_t* sub_objects, sq_tlas** out);
int32_t sq_tlas_destroy(sq_tlas* tlas);

/* Tlas::refit (tlas.rs:49-54) on the device: new rotations (may be NULL),
 * translations and instance parameters (may be NULL: a deforming provider's
 * new local AABBs) per instance id, then the bottom-up pass. The _d form takes
 * device pointers, any of them NULL, and per-instance translation steps
 * (delta) added in place. */
int32_t sq_tlas_refit(sq_ctx* ctx, sq_tlas* tlas, const float* rot, const float* trans, const float* param);
int32_t sq_tlas_refit_d(sq_ctx* ctx, sq_tlas* tlas, const float* d_rot, const float* d_trans, const float* d_delta,
                        const float* d_param);
/* Node bounds in host-tree order and instance world AABBs in id order (either may be NULL). */
int32_t sq_tlas_read_bounds(sq_ctx* ctx, const sq_tlas* tlas, float* node_bounds, float* world_aabbs);
/* Tlas::needs_rebuild (tlas.rs:58-60). */
int32_t sq_tlas_needs_rebuild(sq_ctx* ctx, const sq_tlas* tlas, float factor, int32_t* out);

/* Tlas queries (tlas.rs:82-431): same layouts and semantics as the
 * single-level ones; leaf = instance index. */
int32_t sq_tlas_raycast_nearest(sq_ctx* ctx, const sq_tlas* tlas, const float* rays, uint32_t n, float max_toi,
                                const float* max_toi_per_query, const sq_filter* filter, const sq_hits* out,
                                sq_query_stats* stats);
int32_t sq_tlas_raycast_all(sq_ctx* ctx, const sq_tlas* tlas, const float* rays, uint32_t n, float max_toi,
                            const float* max_toi_per_query, const sq_filter* filter, const sq_hit_lists* out);
int32_t sq_tlas_raycast_crossings(sq_ctx* ctx, const sq_tlas* tlas, const float* rays, uint32_t n, float max_toi,
                                  const float* max_toi_per_query, const sq_filter* filter, const sq_hit_lists* out);
int32_t sq_tlas_shapecast_nearest(sq_ctx* ctx, const sq_tlas* tlas, const float* casts, uint32_t n, float max_toi,
                                  const float* max_toi_per_query, const sq_filter* filter, const sq_hits* out);
int32_t sq_tlas_shapecast_all(sq_ctx* ctx, const sq_tlas* tlas, const float* casts, uint32_t n, float max_toi,
                              const float* max_toi_per_query, const sq_filter* filter, const sq_hit_lists* out);
int32_t sq_tlas_overlap(sq_ctx* ctx, const sq_tlas* tlas, const float* regions, uint32_t n, const sq_filter* filter,
                        uint64_t* offsets, uint32_t* leaves, uint64_t leaf_capacity, uint64_t* total);

/* One persistent launch over a mixed batch (device pointers): nearest rays,
 * nearest shape casts and overlap regions. Overlaps report the full count
 * and the first region_k instances in ascending order. */
typedef struct sq_mixed_batch {
  const float* rays;
  uint32_t n_rays;
  float ray_max_toi;
  const float* ray_max_toi_per_query;
  sq_hits ray_hits;
  const float* casts;
  uint32_t n_casts;
  float cast_max_toi;
  const float* cast_max_toi_per_query;
  sq_hits cast_hits;
  const float* regions;
  uint32_t n_regions;
  uint32_t region_k;
  uint32_t* region_count;
  uint32_t* region_leaves;
} sq_mixed_batch;
int32_t sq_tlas_mixed_d(sq_ctx* ctx, const sq_tlas* tlas, const sq_mixed_batch* batch, const sq_filter* filter);

/* ---- CUDA graphs -------------------------------------------------------------
 * Records the device-pointer calls made on the context's stream between
 * begin and end (e.g. one frame: sq_tlas_refit_d + sq_tlas_mixed_d) and
 * replays them with one launch. Host-buffer calls cannot be recorded. */
int32_t sq_graph_begin(sq_ctx* ctx);
int32_t sq_graph_end(sq_ctx* ctx, sq_graph** out);
int32_t sq_graph_launch(sq_ctx* ctx, const sq_graph* graph);
int32_t sq_graph_destroy(sq_graph* graph);

#ifdef __cplusplus
}
#endif

#endif /* SQ_H */
