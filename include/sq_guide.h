/* Learned guide for nearest-ray queries: C ABI.
 *
 * No counterpart exists in the reference crate. Its one batched GPU call,
 * GpuRaycaster::raycast_nearest_batch (crates/spatial-query/src/gpu/mod.rs:348),
 * walks every ray from the root. Here a small MLP (ray origin normalised to
 * the scene box and direction in, 3 hidden layers of 128 with ReLU, bf16
 * weights with f32 accumulation, one logit per bucket out) predicts, per
 * ray, the bucket (a subtree at a fixed depth of the crate's tree) that holds
 * its nearest hit. The seeded query searches that subtree first; its nearest
 * hit becomes the limit for the walk from the root, which skips the subtree.
 * The answer is certified as in SQ_ORDER_NEAR_FIRST (include/sq.h) and
 * replayed in the reference order when it is not, so the hits are the
 * crate's own (Bvh::raycast_nearest, accel/bvh.rs:73-124) whatever the
 * network predicts. The network trains on the GPU with tcgen05 kernels on
 * rays labelled by the plain traversal (AdamW).
 *
 * Scope: D = 3 scenes, nearest rays, the default filter.
 */
#ifndef SQ_GUIDE_H
#define SQ_GUIDE_H

#include <stddef.h>
#include <stdint.h>

#include "sq.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sq_guide sq_guide;

typedef struct sq_guide_config {
  uint32_t depth;      /* bucket depth in the tree (root = 0); 12 gives 4,096 buckets on 2^20 primitives */
  uint32_t batch;      /* training batch (multiple of 128) */
  float lr;            /* AdamW learning rate */
  float weight_decay;  /* AdamW decoupled weight decay */
  float beta1, beta2, eps;
  uint64_t seed;       /* weight initialisation (uniform +-1/sqrt(fan_in), as torch.nn.Linear) */
} sq_guide_config;

/* Defaults: depth 12, batch 8192, lr 1e-3, weight decay 0.01, betas 0.9 / 0.999, eps 1e-8, seed 0. */
void sq_guide_config_default(sq_guide_config* cfg);

/* Builds the bucket table of `bvh` (D = 3) and a freshly initialised
 * network on the context's device. `bvh` must outlive the guide. The
 * output layer has one logit per bucket, rounded up to a multiple of 128. */
int32_t sq_guide_create(sq_ctx* ctx, const sq_bvh* bvh, const sq_guide_config* cfg, sq_guide** out);
int32_t sq_guide_destroy(sq_guide* g);

typedef struct sq_guide_info {
  uint32_t n_buckets;  /* subtrees at the bucket depth (plus shallower leaves) */
  uint32_t n_out;      /* output logits (n_buckets rounded up to 128) */
  uint32_t hidden;     /* 128 */
  uint32_t inputs;     /* 6 */
  uint64_t n_params;   /* weights and biases */
  uint32_t steps;      /* optimiser steps taken */
} sq_guide_info;
int32_t sq_guide_get_info(const sq_guide* g, sq_guide_info* info);

/* Training labels: the bucket of each ray's nearest hit under the plain
 * traversal, -1 for a miss (device pointers, enqueued on the context's stream). */
int32_t sq_guide_label_d(sq_guide* g, const float* d_rays, uint32_t n, float max_toi, int32_t* d_labels);

/* One AdamW step on rays [0, cfg.batch) of d_rays with their labels
 * (label -1 rows are ignored). *loss (optional) receives the batch's mean
 * cross-entropy (waits for the stream). */
int32_t sq_guide_train_step_d(sq_guide* g, const float* d_rays, const int32_t* d_labels, float* loss);

/* `epochs` passes over n rays in batches of cfg.batch (a trailing partial
 * batch is dropped); loss_per_epoch (optional, `epochs` floats) receives
 * each epoch's mean loss. */
int32_t sq_guide_train_d(sq_guide* g, const float* d_rays, const int32_t* d_labels, uint32_t n, uint32_t epochs,
                         float* loss_per_epoch);

/* Forward and backward on one batch without the optimiser step; gradients
 * are kept for sq_guide_get_grads. For gradient checks. */
int32_t sq_guide_forward_backward_d(sq_guide* g, const float* d_rays, const int32_t* d_labels, float* loss);

/* Parameters (host, f32), in this order and layout:
 *   W1 [128 x 6], b1 [128], W2 [128 x 128], b2 [128], W3 [128 x 128], b3 [128],
 *   W4 [n_out x 128], b4 [n_out]   (row-major [out x in]).
 * `count` must equal sq_guide_info.n_params. */
int32_t sq_guide_get_params(sq_guide* g, float* host, uint64_t count);
int32_t sq_guide_set_params(sq_guide* g, const float* host, uint64_t count);
/* Gradients of the last forward/backward, same layout. */
int32_t sq_guide_get_grads(sq_guide* g, float* host, uint64_t count);

/* Top-1 bucket per ray from the fused tcgen05 inference kernel (device pointers). */
int32_t sq_guide_predict_d(sq_guide* g, const float* d_rays, uint32_t n, int32_t* d_bucket);

/* Learned-seeded nearest rays (device pointers): same outputs, same hits as
 * sq_raycast_nearest_d. `d_bucket` NULL runs the network first (into the
 * context's arena); otherwise the given predictions seed the queries. With
 * `d_bucket` NULL, no stats and 524,288 rays or more, the two halves are
 * predicted and walked on the context's stream and on its internal second
 * lane (own stream and scratch, joined back to the context's stream before
 * the call returns); the first such call of a batch size sizes that lane's
 * scratch, so it belongs outside a stream capture. After the predicted
 * bucket the walk follows the context's order (sq_ctx_set_order): near-first,
 * or the crate's child order (push a, push b); either way each answer is
 * certified and equals the reference's. */
int32_t sq_raycast_nearest_guided_d(sq_ctx* ctx, const sq_bvh* bvh, const sq_guide* g, const float* d_rays,
                                    uint32_t n, float max_toi, const int32_t* d_bucket, const sq_hits* out,
                                    sq_query_stats* stats);

/* The same through host buffers (rays and outputs in host memory). */
int32_t sq_raycast_nearest_guided(sq_ctx* ctx, const sq_bvh* bvh, const sq_guide* g, const float* rays, uint32_t n,
                                  float max_toi, const sq_hits* out, sq_query_stats* stats);

/* Serialised network (config, step, parameters and optimiser moments). */
int32_t sq_guide_save(const sq_guide* g, void* buf, size_t cap, size_t* size);
int32_t sq_guide_load(sq_guide* g, const void* buf, size_t size);

/* The tensor-core GEMM the guide trains with, exposed for testing:
 * C[M x N] (f32, row stride ldc) = A[M x K] * B[N x K]^T with bf16 A and B
 * (row strides lda, ldb elements; K, lda and ldb multiples of 8). */
int32_t sq_gemm_bf16_tn_d(sq_ctx* ctx, const uint16_t* d_a, const uint16_t* d_b, float* d_c, uint32_t m, uint32_t n,
                          uint32_t k, uint32_t lda, uint32_t ldb, uint32_t ldc);

#ifdef __cplusplus
}
#endif

#endif /* SQ_GUIDE_H */
