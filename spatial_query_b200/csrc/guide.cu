// The learned guide (include/sq_guide.h): bucket table, training on the
// GPU with tcgen05 GEMMs, fused tcgen05 inference, and the seeded query.
//
// Network: x = (origin normalised to the scene box in [-1, 1], unit
// direction) -> 128 -> 128 -> 128 (ReLU) -> one logit per bucket. Weights are
// bf16 for the tensor cores with f32 master copies for AdamW; every product
// accumulates in f32. Activations feeding a GEMM are rounded to bf16.
//
// Training step on a batch of B rays (B a multiple of 128), as GEMMs
// C = A * B^T on K-major bf16 operands (guide_gemm.cuh):
//   Z1 = X W1^T, H1 = relu(Z1 + b1), ..., Z4 = H3 W4^T, softmax cross-entropy
//   dZ4 = (softmax - onehot) / n_labelled, dW4 = dZ4^T H3, dH3 = dZ4 W4, ...
// The transposed operands (dZ^T, H^T, W^T) are written by the kernels that
// produce them.
//
// Inference (guide_infer_kernel): one persistent CTA per SM runs the whole
// network for 256 rays at a time: warp 0 streams pre-swizzled weight chunks
// (W2, W3, then W4 in 128-row chunks) with bulk copies into a 3-slot ring,
// warps 1 and 10 issue tcgen05.mma (one thread each, one 128-ray half each)
// into double-buffered TMEM accumulators, eight
// epilogue warps apply bias + ReLU and write the next layer's bf16 operand
// back to shared memory, and for the last layer fold each 128-logit chunk
// into a running argmax. Logits never leave the SM.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sq_guide.h"
#include "guide_gemm.cuh"
#include "sq_internal.cuh"

using namespace sq;
using namespace sqi;
using bf16 = __nv_bfloat16;

namespace {

constexpr uint32_t kHidden = 128;
constexpr uint32_t kInputs = 6;
constexpr uint32_t kInPad = 64;  // layer-1 K padded to one 128-byte panel for the training GEMM

// ---------------------------------------------------------------------------
// Feature map, shared by training and inference: origin to [-1, 1] over the
// scene box, direction as is. Explicit roundings keep both paths bitwise equal.
// ---------------------------------------------------------------------------
struct Features {
  float lo[3], inv[3];
};

__device__ __forceinline__ void ray_features(const float* ray, const Features& f, float* x) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    x[i] = __fsub_rn(__fmul_rn(__fmul_rn(__fsub_rn(ray[i], f.lo[i]), f.inv[i]), 2.0f), 1.0f);
    x[3 + i] = ray[3 + i];
  }
}

// X [B x 64] bf16 (zero past the 6 features) and X^T [128 x B] (zero rows past 6).
__global__ void features_kernel(const float* __restrict__ rays, uint32_t n, uint32_t B, Features f, bf16* X,
                                bf16* XT) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  float x[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (r < n) ray_features(rays + size_t(r) * 6, f, x);
  for (uint32_t k = 0; k < kInPad; ++k) X[size_t(r) * kInPad + k] = __float2bfloat16_rn(k < 6 ? x[k] : 0.f);
  for (uint32_t k = 0; k < 6; ++k) XT[size_t(k) * B + r] = __float2bfloat16_rn(x[k]);
}

// H = bf16(relu(Z + b)) and H^T, for Z [R x 128] f32.
__global__ void bias_relu_kernel(const float* __restrict__ Z, const float* __restrict__ b, bf16* H, bf16* HT,
                                 uint32_t R) {
  __shared__ bf16 tile[32][33];
  const uint32_t r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
    const uint32_t r = r0 + i, c = c0 + threadIdx.x;
    bf16 h = __float2bfloat16_rn(0.f);
    if (r < R) {
      h = __float2bfloat16_rn(fmaxf(Z[size_t(r) * kHidden + c] + b[c], 0.f));
      H[size_t(r) * kHidden + c] = h;
    }
    tile[i][threadIdx.x] = h;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
    const uint32_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < R) HT[size_t(c) * R + r] = tile[threadIdx.x][i];
  }
}

__global__ void count_labels_kernel(const int32_t* __restrict__ labels, uint32_t B, uint32_t n_buckets,
                                    uint32_t* count) {
  uint32_t c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x)
    c += (labels[i] >= 0 && uint32_t(labels[i]) < n_buckets) ? 1u : 0u;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// One row of logits per block: softmax cross-entropy against the label
// (-1: ignored), dZ = (softmax - onehot) / n_labelled as bf16.
__global__ void softmax_ce_kernel(const float* __restrict__ Z, const float* __restrict__ b,
                                  const int32_t* __restrict__ labels, uint32_t n_out, uint32_t n_buckets,
                                  const uint32_t* count, bf16* dZ, float* loss_sum) {
  const uint32_t row = blockIdx.x;
  const float* z = Z + size_t(row) * n_out;
  bf16* dz = dZ + size_t(row) * n_out;
  const int32_t y = labels[row];
  __shared__ float red[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (y < 0 || uint32_t(y) >= n_buckets) {
    for (uint32_t j = threadIdx.x; j < n_out; j += blockDim.x) dz[j] = __float2bfloat16_rn(0.f);
    return;
  }
  float m = -INFINITY;
  for (uint32_t j = threadIdx.x; j < n_buckets; j += blockDim.x) m = fmaxf(m, z[j] + b[j]);
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) red[warp] = m;
  __syncthreads();
  m = red[0];
  for (int w = 1; w < nw; ++w) m = fmaxf(m, red[w]);
  __syncthreads();
  float s = 0.f;
  for (uint32_t j = threadIdx.x; j < n_buckets; j += blockDim.x) s += expf(z[j] + b[j] - m);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  s = 0.f;
  for (int w = 0; w < nw; ++w) s += red[w];
  const float inv_n = 1.0f / float(max(*count, 1u));
  const float inv_s = 1.0f / s;
  for (uint32_t j = threadIdx.x; j < n_out; j += blockDim.x) {
    float g = 0.f;
    if (j < n_buckets) g = expf(z[j] + b[j] - m) * inv_s - (j == uint32_t(y) ? 1.f : 0.f);
    dz[j] = __float2bfloat16_rn(g * inv_n);
  }
  if (threadIdx.x == 0) atomicAdd(loss_sum, logf(s) + m - (z[y] + b[y]));
}

// out[C x R] = in[R x C]^T (bf16), and colsum[c] += sum over rows of in[., c].
__global__ void transpose_colsum_kernel(const bf16* __restrict__ in, bf16* out, float* colsum, uint32_t R,
                                        uint32_t C) {
  __shared__ bf16 tile[32][33];
  __shared__ float part[8][32];
  const uint32_t r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  float acc = 0.f;
  for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
    const uint32_t r = r0 + i, c = c0 + threadIdx.x;
    bf16 v = __float2bfloat16_rn(0.f);
    if (r < R && c < C) v = in[size_t(r) * C + c];
    tile[i][threadIdx.x] = v;
    acc += __bfloat162float(v);
  }
  part[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (colsum && threadIdx.y == 0 && c0 + threadIdx.x < C) {
    float t = 0.f;
    for (uint32_t k = 0; k < blockDim.y; ++k) t += part[k][threadIdx.x];
    atomicAdd(colsum + c0 + threadIdx.x, t);
  }
  for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
    const uint32_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < R && c < C) out[size_t(c) * R + r] = tile[threadIdx.x][i];
  }
}

// dZ = bf16(dH * (H > 0)), dZ^T, and db += column sums of dZ.
__global__ void relu_back_kernel(const float* __restrict__ dH, const bf16* __restrict__ H, bf16* dZ, bf16* dZT,
                                 float* db, uint32_t R) {
  __shared__ bf16 tile[32][33];
  __shared__ float part[8][32];
  const uint32_t r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  float acc = 0.f;
  for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
    const uint32_t r = r0 + i, c = c0 + threadIdx.x;
    bf16 v = __float2bfloat16_rn(0.f);
    if (r < R) {
      const size_t k = size_t(r) * kHidden + c;
      v = __float2bfloat16_rn(__bfloat162float(H[k]) > 0.f ? dH[k] : 0.f);
      dZ[k] = v;
    }
    tile[i][threadIdx.x] = v;
    acc += __bfloat162float(v);
  }
  part[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.y == 0) {
    float t = 0.f;
    for (uint32_t k = 0; k < blockDim.y; ++k) t += part[k][threadIdx.x];
    atomicAdd(db + c0 + threadIdx.x, t);
  }
  for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
    const uint32_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < R) dZT[size_t(c) * R + r] = tile[threadIdx.x][i];
  }
}

// AdamW (decoupled weight decay), as torch.optim.AdamW.
__global__ void adamw_kernel(float* P, const float* __restrict__ G, float* M, float* V, size_t n, float lr, float b1,
                             float b2, float eps, float wd, float bc1, float bc2) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    const float g = G[i];
    float p = P[i] * (1.f - lr * wd);
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    p -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
    P[i] = p;
  }
}

// bf16 copy of W [rows x cols] and, optionally, its transpose [cols x rows].
__global__ void to_bf16_kernel(const float* __restrict__ W, bf16* Wb, bf16* WbT, uint32_t rows, uint32_t cols) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < size_t(rows) * cols;
       i += size_t(gridDim.x) * blockDim.x) {
    const bf16 v = __float2bfloat16_rn(W[i]);
    Wb[i] = v;
    if (WbT) WbT[(i % cols) * rows + i / cols] = v;
  }
}

// Shared-memory images of K-major weight rows, 128-byte swizzled: rows
// [c*128, c*128+128) of Wb [rows x K] become chunk c, made of K/64 panels of
// 128 rows x 128 B (K = 64 or 128). One bulk copy lands a chunk as is.
__global__ void swizzle_image_kernel(const bf16* __restrict__ Wb, uint8_t* img, uint32_t rows, uint32_t K) {
  const uint32_t panels = K / 64;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < size_t(rows) * (K / 8);
       i += size_t(gridDim.x) * blockDim.x) {
    const uint32_t r = uint32_t(i / (K / 8)), k8 = uint32_t(i % (K / 8)) * 8;
    const uint32_t c = r / 128, rr = r % 128, panel = k8 / 64;
    uint8_t* dst = img + size_t(c) * panels * 16384 + panel * 16384 + umma::sw128_offset(rr, k8 % 64);
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(Wb + size_t(r) * K + k8);
  }
}

__global__ void bucket_of_id_kernel(const uint32_t* __restrict__ prim_ids, const uint32_t* __restrict__ starts,
                                    uint32_t nb, int32_t* out, uint32_t n_prims) {
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n_prims) return;
  uint32_t lo = 0, hi = nb;  // last bucket with start <= pos
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (starts[mid] <= pos) lo = mid;
    else hi = mid;
  }
  out[prim_ids[pos]] = int32_t(lo);
}

// Batch gather for shuffled epochs: rays and labels of perm[0 .. B).
__global__ void gather_batch_kernel(const float* __restrict__ rays, const int32_t* __restrict__ labels,
                                    const uint32_t* __restrict__ perm, uint32_t B, float* b_rays, int32_t* b_labels) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B) return;
  const size_t r = perm[i];
#pragma unroll
  for (int k = 0; k < 6; ++k) b_rays[size_t(i) * 6 + k] = rays[r * 6 + k];
  b_labels[i] = labels[r];
}

__global__ void labels_kernel(const uint32_t* __restrict__ leaf, const int32_t* __restrict__ bucket_of_id,
                              int32_t* labels, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) labels[i] = leaf[i] == kNoHit ? -1 : bucket_of_id[leaf[i]];
}

// ---------------------------------------------------------------------------
// Fused inference.
// ---------------------------------------------------------------------------
constexpr int kInferThreads = 352;  // warp 0 loads, warps 1 and 10 issue MMAs (half 0 / half 1), warps 2..9 epilogue
constexpr int kRing = 3;
constexpr uint32_t kChunkBytes = 32768;  // 128 rows x 128 bf16, two swizzled panels

struct InferParams {
  const float* rays;
  uint32_t n;
  Features f;
  const uint8_t* w1_img;   // 16 KB: W1 [128 x 64] as one panel
  const uint8_t* w23_img;  // 2 chunks: W2, W3
  const uint8_t* w4_img;   // n_chunks chunks
  const float* bias;       // b1, b2, b3 (128 each), b4 (n_chunks * 128)
  uint32_t n_chunks;
  uint32_t n_buckets;
  int32_t* out;
  int* err;
};

struct InferSmem {
  static constexpr uint32_t act = 0;                       // 2 halves x 32 KB
  static constexpr uint32_t w1 = 65536;                    // 16 KB
  static constexpr uint32_t ring = w1 + 16384;             // 3 x 32 KB
  static constexpr uint32_t bias = ring + kRing * kChunkBytes;  // (384 + 4096) floats max
  static constexpr uint32_t bars = bias + (384 + 4096) * 4;
  static constexpr uint32_t bytes = bars + 256 + 1024;
};

// A logit with the index i (0..127) of its column in the low 7 mantissa bits,
// as 127 - i: (x | 0x7F) ^ i. Written as one LOP3 whose mask comes from a
// register the compiler cannot fold (r7f is read from shared memory), so i
// is the instruction's only immediate: one ALU operation per logit, where
// the two-immediate form costs two.
__device__ __forceinline__ float tag7(float x, uint32_t r7f, uint32_t i) {
  uint32_t r;
  asm("lop3.b32 %0, %1, %2, %3, 0x56;" : "=r"(r) : "r"(__float_as_uint(x)), "r"(r7f), "r"(i));
  return __uint_as_float(r);
}

// max of two (PTX max.f32 with two sources); kept as written, not merged
// into three-source maxima.
__device__ __forceinline__ float fmax2(float a, float b) {
  float r;
  asm("max.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// a0 += b0, a1 += b1 in one packed instruction (add.rn.f32x2, sm_100), each
// sum rounded to nearest as a scalar f32 add would be.
__device__ __forceinline__ void add2(float& a0, float& a1, float b0, float b1) {
  asm("{.reg .b64 pa, pb, pd;\n\t"
      "mov.b64 pa, {%0, %1};\n\t"
      "mov.b64 pb, {%2, %3};\n\t"
      "add.rn.f32x2 pd, pa, pb;\n\t"
      "mov.b64 {%0, %1}, pd;}"
      : "+f"(a0), "+f"(a1)
      : "f"(b0), "f"(b1));
}

__global__ void __launch_bounds__(kInferThreads, 1) guide_infer_kernel(const InferParams p) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = umma::smem_u32(smem_raw);
  uint8_t* base = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + InferSmem::bars);
  uint64_t* w_full = bars + 0;
  uint64_t* ring_full = bars + 1;            // [3]
  uint64_t* ring_empty = bars + 4;           // [3]
  // The two 128-ray halves of a tile run as independent pipelines that
  // share the weight ring: per stage and half an accumulator-full and an
  // accumulator-empty barrier, per half an operand-ready barrier.
  uint64_t* acc_full = bars + 7;             // [stage * 2 + half]
  uint64_t* acc_empty = bars + 11;           // [stage * 2 + half]
  uint64_t* act_ready = bars + 15;           // [half]
  uint64_t* fin = bars + 17;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 18);
  int* s_err = reinterpret_cast<int*>(bars + 19);
  uint32_t* s_r7f = reinterpret_cast<uint32_t*>(bars + 20);  // 0x7F, for tag7
  const float* s_bias = reinterpret_cast<const float*>(base + InferSmem::bias);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t n_tiles = (p.n + 255) / 256;
  const uint32_t bias_bytes = (384 + p.n_chunks * 128) * 4;
  constexpr uint32_t idesc = umma::idesc_bf16(128, 128);

  if (threadIdx.x == 0) {
    umma::mbar_init(w_full, 1);
    for (int s = 0; s < kRing; ++s) {
      umma::mbar_init(&ring_full[s], 1);
      umma::mbar_init(&ring_empty[s], 2);  // released by both halves' MMAs
    }
    for (int k = 0; k < 4; ++k) {
      umma::mbar_init(&acc_full[k], 1);
      umma::mbar_init(&acc_empty[k], 4);
    }
    umma::mbar_init(&act_ready[0], 4);
    umma::mbar_init(&act_ready[1], 4);
    umma::mbar_init(fin, 2);
    *s_err = 0;
    *s_r7f = 0x7Fu;
    umma::fence_barrier_init();
  }
  __syncwarp();
  if (warp == 1) umma::tmem_alloc(tslot, 512);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  auto failed = [&]() { return *(volatile int*)s_err != 0; };
  auto set_err = [&](int code) { atomicCAS(s_err, 0, code); };

  if (warp == 0) {
    if (lane == 0) {
      // Producer: W1 + biases once, then per tile W2, W3, W4 chunks.
      umma::mbar_arrive_expect_tx(w_full, 16384 + bias_bytes);
      umma::bulk_load(base + InferSmem::w1, p.w1_img, 16384, w_full);
      umma::bulk_load(base + InferSmem::bias, p.bias, bias_bytes, w_full);
      uint32_t G = 0;
      for (uint32_t t = blockIdx.x; t < n_tiles && !failed(); t += gridDim.x) {
        for (uint32_t j = 0; j < 2 + p.n_chunks; ++j, ++G) {
          const uint32_t slot = G % kRing;
          if (G >= kRing && !umma::mbar_wait(&ring_empty[slot], ((G / kRing) + 1) & 1)) {
            set_err(1);
            break;
          }
          const uint8_t* src = j < 2 ? p.w23_img + size_t(j) * kChunkBytes : p.w4_img + size_t(j - 2) * kChunkBytes;
          umma::mbar_arrive_expect_tx(&ring_full[slot], kChunkBytes);
          umma::bulk_load(base + InferSmem::ring + slot * kChunkBytes, src, kChunkBytes, &ring_full[slot]);
        }
      }
      // Let every copy issued land before shared memory is released.
      for (uint32_t k = (G > kRing ? G - kRing : 0); k < G; ++k)
        umma::mbar_wait(&ring_full[k % kRing], (k / kRing) & 1, 100000000ull);
      umma::mbar_wait(w_full, 0, 100000000ull);
    }
  } else if (warp == 1 || warp == 10) {
    if (lane == 0) {
      // MMA issuers, one per half (warp 1: half 0, warp 10: half 1). With
      // one issuing thread for both halves the tensor pipe drained while that
      // thread waited on the next weight slot and accumulator; two threads
      // keep one half's MMAs queued while the other half's issuer waits.
      const uint32_t h = warp == 1 ? 0u : 1u;
      if (!umma::mbar_wait(w_full, 0)) set_err(2);
      uint32_t G = 0, J = 0, A = 0;
      const uint32_t w1d = umma::smem_u32(base + InferSmem::w1);
      const uint32_t a = umma::smem_u32(base + InferSmem::act + h * 32768);
      // Every descriptor of the K-steps, made once: this half's operand rows
      // and each weight slot. The epilogue warps keep the ALU pipe busy with
      // the argmax; descriptor arithmetic between the MMAs would queue behind
      // it and slow their issue.
      static_assert(kRing == 3, "the issue below names each slot's descriptors");
      uint64_t ad[8], bd[kRing][8];
#pragma unroll
      for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t off = (k >> 2) * 16384;
        ad[k] = umma::desc_sw128(a + off) + 2 * (k & 3);
#pragma unroll
        for (int sl = 0; sl < kRing; ++sl)
          bd[sl][k] = umma::desc_sw128(umma::smem_u32(base + InferSmem::ring + sl * kChunkBytes) + off) + 2 * (k & 3);
      }
      bool ok = true;
      for (uint32_t t = blockIdx.x; ok && t < n_tiles && !failed(); t += gridDim.x) {
        for (uint32_t j = 0; ok && j < 3 + p.n_chunks && !failed(); ++j, ++J) {
          const uint32_t s = J & 1;
          uint32_t slot = 0;
          if (j >= 1) {
            slot = G % kRing;
            if (!umma::mbar_wait(&ring_full[slot], (G / kRing) & 1)) { set_err(5); ok = false; break; }
          }
          // Layers 1-3 and the first W4 chunk wait for this half's operand rows.
          if (j <= 3) {
            if (!umma::mbar_wait(&act_ready[h], A & 1)) { set_err(3); ok = false; break; }
            ++A;
          }
          if (J >= 2 && !umma::mbar_wait(&acc_empty[s * 2 + h], ((J / 2) + 1) & 1)) {
            set_err(4);
            ok = false;
            break;
          }
          umma::tc_fence_after();
          const uint32_t d = tbase + s * 256 + h * 128;
          if (j == 0) {
            umma::mma_bf16(d, umma::desc_sw128(a), umma::desc_sw128(w1d), idesc, 0);
          } else if (slot == 0) {
            umma::mma_bf16_x8(d, ad, bd[0], idesc);
          } else if (slot == 1) {
            umma::mma_bf16_x8(d, ad, bd[1], idesc);
          } else {
            umma::mma_bf16_x8(d, ad, bd[2], idesc);
          }
          umma::mma_commit(&acc_full[s * 2 + h]);
          if (j >= 1) {
            umma::mma_commit(&ring_empty[slot]);
            ++G;
          }
        }
      }
      umma::mma_commit(fin);
    }
  } else {
    // Epilogue warps: half h of the 256-ray tile, TMEM lanes of quarter q.
    const uint32_t e = warp - 2, h = e / 4, q = warp & 3;
    const uint32_t row = q * 32 + lane;
    uint8_t* act = base + InferSmem::act + h * 32768;
    const uint32_t lane_base = (q * 32u) << 16;
    uint32_t J = 0;
    // Every lane waits; the warp proceeds only if all of them saw the phase
    // (tcgen05.ld below is warp-collective).
    auto warp_wait = [&](uint64_t* bar, uint32_t parity) {
      return __all_sync(0xffffffffu, umma::mbar_wait(bar, parity)) != 0;
    };
    if (!warp_wait(w_full, 0)) set_err(6);
    for (uint32_t t = blockIdx.x; t < n_tiles && !failed(); t += gridDim.x) {
      const uint32_t ray = t * 256 + h * 128 + row;
      // Layer-1 operand: the 6 features (K = 16, rest zero) in panel 0.
      {
        float x[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (ray < p.n) ray_features(p.rays + size_t(ray) * 6, p.f, x);
        __align__(16) bf16 v[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = __float2bfloat16_rn(k < 6 ? x[k] : 0.f);
        *reinterpret_cast<uint4*>(act + umma::sw128_offset(row, 0)) = *reinterpret_cast<const uint4*>(v);
        *reinterpret_cast<uint4*>(act + umma::sw128_offset(row, 8)) = *reinterpret_cast<const uint4*>(v + 8);
      }
      umma::fence_proxy_async();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(&act_ready[h]);
      float best = -INFINITY;
      uint32_t best_idx = 0;
      for (uint32_t j = 0; j < 3 + p.n_chunks; ++j, ++J) {
        const uint32_t s = J & 1;
        if (!warp_wait(&acc_full[s * 2 + h], (J / 2) & 1)) { set_err(7); break; }
        umma::tc_fence_after();
        const uint32_t tcol = tbase + lane_base + s * 256 + h * 128;
        if (j < 3) {
          // bias + ReLU -> bf16 -> next layer's operand rows
          const float* b = s_bias + j * 128;
          float v[128];
          umma::tmem_ld128(tcol, v);  // the whole row in one load and one wait
#pragma unroll
          for (uint32_t c = 0; c < 128; c += 32) {
            __align__(16) __nv_bfloat162 o[16];
#pragma unroll
            for (int i = 0; i < 16; ++i)
              o[i] = __floats2bfloat162_rn(fmaxf(v[c + 2 * i] + b[c + 2 * i], 0.f),
                                           fmaxf(v[c + 2 * i + 1] + b[c + 2 * i + 1], 0.f));
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const uint32_t k = c + 8 * i;
              *reinterpret_cast<uint4*>(act + (k >> 6) * 16384 + umma::sw128_offset(row, k & 63)) =
                  *reinterpret_cast<const uint4*>(o + 4 * i);
            }
          }
          umma::tc_fence_before();
          umma::fence_proxy_async();
          __syncwarp();
          if (lane == 0) {
            umma::mbar_arrive(&acc_empty[s * 2 + h]);
            umma::mbar_arrive(&act_ready[h]);
          }
        } else {
          float v[128];
          umma::tmem_ld128(tcol, v);  // the chunk's 128 logits of this row in one load and one wait
          // The logits are in registers: the accumulator goes back to the MMA
          // issuer now and the argmax below runs beside the next chunks'
          // MMAs, adding the bias from registers (handing it back after the
          // argmax, with the bias stored into TMEM first, measured the same:
          // 1.032 against 1.035 ms per 1,048,576 rays).
          umma::tc_fence_before();
          __syncwarp();
          if (lane == 0) umma::mbar_arrive(&acc_empty[s * 2 + h]);
          // Running argmax over this chunk's 128 logits plus their bias. The
          // chunk-local index rides in the low mantissa bits, so one max per
          // logit suffices (ties within 2^-16 relative go either way).
          const uint32_t c0 = (j - 3) * 128;
          const float* bb = s_bias + 384 + c0;
          const uint32_t r7f = *reinterpret_cast<volatile uint32_t*>(s_r7f);
          float m = -INFINITY;
          if (c0 + 128 <= p.n_buckets) {
            // Four independent chains of two-input maxima: measured 0.999
            // against 1.035 ms per 1,048,576 rays for two chains of
            // three-input maxima.
            float m1 = -INFINITY, m2 = -INFINITY, m3 = -INFINITY;
#pragma unroll
            for (uint32_t i = 0; i < 128; i += 4) {
              const float4 b4 = *reinterpret_cast<const float4*>(bb + i);
              add2(v[i], v[i + 1], b4.x, b4.y);
              add2(v[i + 2], v[i + 3], b4.z, b4.w);
              m = fmax2(m, tag7(v[i], r7f, i));
              m1 = fmax2(m1, tag7(v[i + 1], r7f, i + 1));
              m2 = fmax2(m2, tag7(v[i + 2], r7f, i + 2));
              m3 = fmax2(m3, tag7(v[i + 3], r7f, i + 3));
            }
            m = fmaxf(fmaxf(m, m1), fmaxf(m2, m3));
          } else {
#pragma unroll
            for (uint32_t i = 0; i < 128; ++i) {
              const float l = (c0 + i < p.n_buckets) ? v[i] + bb[i] : -INFINITY;
              m = fmaxf(m, tag7(l, r7f, i));
            }
          }
          if (m > best) {
            best = m;
            best_idx = c0 + (127u - (__float_as_uint(m) & 0x7Fu));
          }
        }
      }
      if (ray < p.n && !failed()) p.out[ray] = int32_t(best_idx);
    }
  }
  __syncwarp();
  if (threadIdx.x == 32) {
    if (!umma::mbar_wait(fin, 0)) set_err(8);
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  __syncwarp();
  if (warp == 1) umma::tmem_dealloc(tbase, 512);
  if (threadIdx.x == 0 && *s_err) atomicCAS(p.err, 0, *s_err);
}

// ---------------------------------------------------------------------------
// TMA tensor maps (driver entry point fetched through the runtime).
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

// Row-major bf16 [rows x cols] (row stride ld elements), boxes of box_rows x 64.
bool make_map(CUtensorMap* m, const void* ptr, uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {ld * 2};
  cuuint32_t box[2] = {64, box_rows};
  cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int* g_err_slot(sq_ctx* ctx);

// C[M x N] = A[M x K] * B[N x K]^T. a_rows / b_rows: allocated rows of A and B
// (at least M and N; at least one box of 128 rows).
int32_t gemm(sq_ctx* ctx, const bf16* A, uint64_t a_rows, uint32_t lda, const bf16* B, uint64_t b_rows, uint32_t ldb,
             float* C, uint32_t M, uint32_t N, uint32_t K, uint32_t ldc) {
  if (M == 0 || N == 0) return SQ_OK;
  if (K == 0) {
    for (uint32_t r = 0; r < M; ++r) CK(cudaMemsetAsync(C + size_t(r) * ldc, 0, size_t(N) * 4, ctx->stream));
    return SQ_OK;
  }
  if ((K & 7) || (lda & 7) || (ldb & 7) || (uintptr_t(A) & 15) || (uintptr_t(B) & 15) || a_rows < 128 ||
      b_rows < 128 || K < 64)
    return fail(ctx, SQ_ERR_INVALID, "gemm: K and row strides must be multiples of 8 (K >= 64, >= 128 rows), 16-byte aligned");
  CUtensorMap ta, tb;
  if (!make_map(&ta, A, a_rows, K, lda, 128) || !make_map(&tb, B, b_rows, K, ldb, 128))
    return fail(ctx, SQ_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  constexpr int BN = 128;
  const int smem = guide::GemmSmem<BN>::bytes;
  static std::once_flag attr;
  std::call_once(attr, [&] {
    cudaFuncSetAttribute(guide::gemm_tn_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  });
  int* err = g_err_slot(ctx);
  if (!err) return fail(ctx, SQ_ERR_CUDA, "error slot");
  dim3 grid((M + 127) / 128, (N + BN - 1) / BN);
  guide::gemm_tn_kernel<BN><<<grid, guide::kGemmThreads, smem, ctx->stream>>>(ta, tb, C, int(M), int(N), int(K),
                                                                                int(ldc), guide::kEpiStore, err);
  ctx->launches++;
  CK(cudaGetLastError());
  return SQ_OK;
}

// One device int per context for kernel error codes (timeouts).
std::mutex g_err_mu;
std::vector<std::pair<sq_ctx*, int*>> g_err_slots;
int* g_err_slot(sq_ctx* ctx) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  for (auto& e : g_err_slots)
    if (e.first == ctx) return e.second;
  int* p = nullptr;
  if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
  if (cudaMemset(p, 0, sizeof(int)) != cudaSuccess) return nullptr;
  g_err_slots.emplace_back(ctx, p);
  return p;
}

}  // namespace

// The context's error slot goes with the context (a later context at the
// same address, possibly on another device, must not inherit it).
void sqi::release_err_slot(sq_ctx* ctx) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  for (auto it = g_err_slots.begin(); it != g_err_slots.end(); ++it) {
    if (it->first == ctx) {
      cudaFree(it->second);
      g_err_slots.erase(it);
      return;
    }
  }
}

namespace {

int32_t check_err(sq_ctx* ctx, int* err) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (h) {
    CK(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    return fail(ctx, SQ_ERR_CUDA, "tensor-core kernel timed out waiting (code " + std::to_string(h) + ")");
  }
  return SQ_OK;
}

uint32_t blocks_for(size_t n, uint32_t threads) { return uint32_t(std::min<size_t>((n + threads - 1) / threads, 1u << 20)); }

}  // namespace

// ============================================================================
// the guide object
// ============================================================================

struct sq_guide {
  sq_ctx* ctx = nullptr;
  int device = 0;  // destroy needs no context: it may outlive it
  const sq_bvh* bvh = nullptr;
  sq_guide_config cfg{};
  uint32_t n_buckets = 0, n_out = 0, steps = 0;
  Features feat{};
  // parameters: f32 master, gradients, AdamW moments (same layout)
  size_t n_p = 0;
  size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0, oW4 = 0, ob4 = 0;
  float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
  // bf16 weights and transposes
  bf16 *W1b = nullptr, *W2b = nullptr, *W3b = nullptr, *W4b = nullptr;
  bf16 *W2bT = nullptr, *W3bT = nullptr, *W4bT = nullptr;
  // inference images and bias
  uint8_t *w1_img = nullptr, *w23_img = nullptr, *w4_img = nullptr;
  float* infer_bias = nullptr;
  bool images_fresh = false;
  // buckets
  uint2* d_buckets = nullptr;
  uint32_t* d_bucket_sibs = nullptr;  // per bucket, sib_stride ancestor-sibling slots
  uint32_t sib_stride = 0;
  int32_t* d_bucket_of_id = nullptr;
  // batch scratch
  uint32_t B = 0;
  bf16 *X = nullptr, *XT = nullptr, *H[3] = {}, *HT[3] = {}, *dZ4 = nullptr, *dZ4T = nullptr, *dZ = nullptr,
       *dZT = nullptr;
  float *Z = nullptr, *dH = nullptr, *loss = nullptr;
  uint32_t* count = nullptr;
  std::vector<void*> allocs;
  // label scratch
  uint32_t* d_leaf = nullptr;
  uint32_t leaf_cap = 0;
  // shuffled training: permutation of the epoch and the gathered batch
  uint32_t* d_perm = nullptr;
  uint32_t perm_cap = 0;
  float* b_rays = nullptr;
  int32_t* b_labels = nullptr;
};

namespace {

int32_t galloc(sq_guide* g, void** p, size_t bytes) {
  sq_ctx* ctx = g->ctx;
  CK(cudaMalloc(p, std::max<size_t>(bytes, 256)));
  g->allocs.push_back(*p);
  return SQ_OK;
}

// Buckets: the nodes at cfg.depth (and leaves above it), in preorder. Per
// bucket also the slots (record << 1 | slot) of its ancestors' other
// children, root level first, `stride` = depth entries (kNoHit past the
// bucket's own depth): with the bucket they partition the tree, so a walk
// that starts in the bucket and then takes them covers every leaf once.
void build_buckets(const sq_bvh* b, uint32_t depth, std::vector<uint2>& table, std::vector<uint32_t>& starts,
                   std::vector<uint32_t>& sibs, uint32_t stride) {
  table.clear();
  starts.clear();
  sibs.clear();
  if (b->n_nodes == 0) return;
  struct Item { uint32_t node, depth, parent_slot; };
  std::vector<Item> stack{{0u, 0u, kNoHit}};
  std::vector<uint32_t> path;  // sibling slot per level of the current item's ancestors
  while (!stack.empty()) {
    const Item it = stack.back();
    stack.pop_back();
    const uint32_t i = it.node;
    path.resize(it.depth);
    if (it.depth > 0) path[it.depth - 1] = it.parent_slot ^ 1u;  // the other child of the same record
    const bool leaf = b->h_count[i] != 0;
    if (leaf || it.depth == depth) {
      const uint32_t code = leaf ? (kLeafBit | b->h_child_a[i]) : b->h_iidx[i];
      table.push_back(make_uint2(code, it.parent_slot));
      uint32_t k = i;
      while (b->h_count[k] == 0) k = b->h_child_a[k];
      starts.push_back(b->h_child_a[k]);
      for (uint32_t s = 0; s < stride; ++s) sibs.push_back(s < path.size() ? path[s] : kNoHit);
      continue;
    }
    const uint32_t rec = b->h_iidx[i];
    stack.push_back({b->h_child_b[i], it.depth + 1, (rec << 1) | 1u});
    stack.push_back({b->h_child_a[i], it.depth + 1, (rec << 1) | 0u});
  }
}

int32_t refresh_bf16(sq_guide* g) {
  sq_ctx* ctx = g->ctx;
  const uint32_t T = 256;
  to_bf16_kernel<<<blocks_for(kHidden * kInPad, T), T, 0, ctx->stream>>>(g->P + g->oW1, g->W1b, nullptr, kHidden, kInPad);
  to_bf16_kernel<<<blocks_for(kHidden * kHidden, T), T, 0, ctx->stream>>>(g->P + g->oW2, g->W2b, g->W2bT, kHidden, kHidden);
  to_bf16_kernel<<<blocks_for(kHidden * kHidden, T), T, 0, ctx->stream>>>(g->P + g->oW3, g->W3b, g->W3bT, kHidden, kHidden);
  to_bf16_kernel<<<blocks_for(size_t(g->n_out) * kHidden, T), T, 0, ctx->stream>>>(g->P + g->oW4, g->W4b, g->W4bT,
                                                                                      g->n_out, kHidden);
  ctx->launches += 4;
  CK(cudaGetLastError());
  g->images_fresh = false;
  return SQ_OK;
}

int32_t refresh_images(sq_guide* g) {
  if (g->images_fresh) return SQ_OK;
  sq_ctx* ctx = g->ctx;
  const uint32_t T = 256;
  swizzle_image_kernel<<<blocks_for(kHidden * kInPad / 8, T), T, 0, ctx->stream>>>(g->W1b, g->w1_img, kHidden, kInPad);
  swizzle_image_kernel<<<blocks_for(kHidden * kHidden / 8, T), T, 0, ctx->stream>>>(g->W2b, g->w23_img, kHidden, kHidden);
  swizzle_image_kernel<<<blocks_for(kHidden * kHidden / 8, T), T, 0, ctx->stream>>>(g->W3b, g->w23_img + kChunkBytes,
                                                                                     kHidden, kHidden);
  swizzle_image_kernel<<<blocks_for(size_t(g->n_out) * kHidden / 8, T), T, 0, ctx->stream>>>(g->W4b, g->w4_img,
                                                                                              g->n_out, kHidden);
  CK(cudaMemcpyAsync(g->infer_bias, g->P + g->ob1, kHidden * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(g->infer_bias + 128, g->P + g->ob2, kHidden * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(g->infer_bias + 256, g->P + g->ob3, kHidden * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(g->infer_bias + 384, g->P + g->ob4, size_t(g->n_out) * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  ctx->launches += 4;
  CK(cudaGetLastError());
  g->images_fresh = true;
  return SQ_OK;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Host (unpadded) parameter layout <-> device (W1 padded to 64 columns).
size_t host_count(const sq_guide* g) { return size_t(kHidden) * kInputs + 3 * kHidden + 2 * size_t(kHidden) * kHidden + size_t(g->n_out) * kHidden + g->n_out; }

void host_to_dev(const sq_guide* g, const float* h, std::vector<float>& d) {
  d.assign(g->n_p, 0.f);
  size_t o = 0;
  for (uint32_t r = 0; r < kHidden; ++r)
    for (uint32_t c = 0; c < kInputs; ++c) d[g->oW1 + r * kInPad + c] = h[o++];
  auto copy = [&](size_t dst, size_t n) { std::memcpy(d.data() + dst, h + o, n * 4); o += n; };
  copy(g->ob1, kHidden);
  copy(g->oW2, size_t(kHidden) * kHidden);
  copy(g->ob2, kHidden);
  copy(g->oW3, size_t(kHidden) * kHidden);
  copy(g->ob3, kHidden);
  copy(g->oW4, size_t(g->n_out) * kHidden);
  copy(g->ob4, g->n_out);
}

void dev_to_host(const sq_guide* g, const std::vector<float>& d, float* h) {
  size_t o = 0;
  for (uint32_t r = 0; r < kHidden; ++r)
    for (uint32_t c = 0; c < kInputs; ++c) h[o++] = d[g->oW1 + r * kInPad + c];
  auto copy = [&](size_t src, size_t n) { std::memcpy(h + o, d.data() + src, n * 4); o += n; };
  copy(g->ob1, kHidden);
  copy(g->oW2, size_t(kHidden) * kHidden);
  copy(g->ob2, kHidden);
  copy(g->oW3, size_t(kHidden) * kHidden);
  copy(g->ob3, kHidden);
  copy(g->oW4, size_t(g->n_out) * kHidden);
  copy(g->ob4, g->n_out);
}

// Forward + backward of one batch into g->G; the mean loss stays on the device.
int32_t forward_backward(sq_guide* g, const float* d_rays, const int32_t* d_labels) {
  sq_ctx* ctx = g->ctx;
  const uint32_t B = g->B, NO = g->n_out;
  int32_t rc;
  CK(cudaMemsetAsync(g->G, 0, g->n_p * 4, ctx->stream));
  CK(cudaMemsetAsync(g->loss, 0, 4, ctx->stream));
  CK(cudaMemsetAsync(g->count, 0, 4, ctx->stream));
  features_kernel<<<blocks_for(B, 256), 256, 0, ctx->stream>>>(d_rays, B, B, g->feat, g->X, g->XT);
  count_labels_kernel<<<std::min<uint32_t>(blocks_for(B, 256), 64), 256, 0, ctx->stream>>>(d_labels, B, g->n_buckets,
                                                                                            g->count);
  ctx->launches += 2;
  const dim3 tb(32, 8);
  const dim3 tgrid(B / 32, kHidden / 32);
  // forward
  const bf16* in = g->X;
  uint32_t in_k = kInPad;
  const bf16* W[3] = {g->W1b, g->W2b, g->W3b};
  const size_t ob[3] = {g->ob1, g->ob2, g->ob3};
  for (int l = 0; l < 3; ++l) {
    if ((rc = gemm(ctx, in, B, in_k, W[l], kHidden, in_k, g->Z, B, kHidden, in_k, kHidden))) return rc;
    bias_relu_kernel<<<tgrid, tb, 0, ctx->stream>>>(g->Z, g->P + ob[l], g->H[l], g->HT[l], B);
    ctx->launches++;
    in = g->H[l];
    in_k = kHidden;
  }
  if ((rc = gemm(ctx, g->H[2], B, kHidden, g->W4b, NO, kHidden, g->Z, B, NO, kHidden, NO))) return rc;
  softmax_ce_kernel<<<B, 256, 0, ctx->stream>>>(g->Z, g->P + g->ob4, d_labels, NO, g->n_buckets, g->count, g->dZ4,
                                                g->loss);
  transpose_colsum_kernel<<<dim3(B / 32, NO / 32), tb, 0, ctx->stream>>>(g->dZ4, g->dZ4T, g->G + g->ob4, B, NO);
  ctx->launches += 2;
  // backward
  if ((rc = gemm(ctx, g->dZ4T, NO, B, g->HT[2], kHidden, B, g->G + g->oW4, NO, kHidden, B, kHidden))) return rc;
  if ((rc = gemm(ctx, g->dZ4, B, NO, g->W4bT, kHidden, NO, g->dH, B, kHidden, NO, kHidden))) return rc;
  const bf16* WT[3] = {nullptr, g->W2bT, g->W3bT};
  const size_t oW[3] = {g->oW1, g->oW2, g->oW3};
  for (int l = 2; l >= 0; --l) {
    relu_back_kernel<<<tgrid, tb, 0, ctx->stream>>>(g->dH, g->H[l], g->dZ, g->dZT, g->G + ob[l], B);
    ctx->launches++;
    // dW_l = dZ^T [128 x B] * (input of layer l)^T [K x B]^T
    const bf16* inT = l == 0 ? g->XT : g->HT[l - 1];
    const uint32_t K_l = l == 0 ? kInPad : kHidden;
    if ((rc = gemm(ctx, g->dZT, kHidden, B, inT, kHidden, B, g->G + oW[l], kHidden, K_l, B, K_l))) return rc;
    if (l > 0) {
      if ((rc = gemm(ctx, g->dZ, B, kHidden, WT[l], kHidden, kHidden, g->dH, B, kHidden, kHidden, kHidden))) return rc;
    }
  }
  CK(cudaGetLastError());
  return SQ_OK;
}

int32_t read_loss(sq_guide* g, float* loss) {
  sq_ctx* ctx = g->ctx;
  float s = 0.f;
  uint32_t c = 0;
  CK(cudaMemcpyAsync(&s, g->loss, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&c, g->count, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *loss = c ? s / float(c) : 0.f;
  return SQ_OK;
}

int32_t adam_step(sq_guide* g) {
  sq_ctx* ctx = g->ctx;
  g->steps++;
  const double bc1 = 1.0 - std::pow(double(g->cfg.beta1), double(g->steps));
  const double bc2 = 1.0 - std::pow(double(g->cfg.beta2), double(g->steps));
  adamw_kernel<<<std::min<uint32_t>(blocks_for(g->n_p, 256), 4096), 256, 0, ctx->stream>>>(
      g->P, g->G, g->M, g->V, g->n_p, g->cfg.lr, g->cfg.beta1, g->cfg.beta2, g->cfg.eps, g->cfg.weight_decay,
      float(bc1), float(bc2));
  ctx->launches++;
  CK(cudaGetLastError());
  return refresh_bf16(g);
}

sqi::SeedTable seed_table(const sq_guide* g) {
  sqi::SeedTable t;
  t.buckets = g->d_buckets;
  t.sibs = g->d_bucket_sibs;
  t.n_buckets = g->n_buckets;
  t.sib_stride = g->sib_stride;
  return t;
}

int32_t predict(sq_guide* g, const float* d_rays, uint32_t n, int32_t* d_bucket) {
  sq_ctx* ctx = g->ctx;
  if (n == 0) return SQ_OK;
  int32_t rc = refresh_images(g);
  if (rc) return rc;
  int* err = g_err_slot(ctx);
  if (!err) return fail(ctx, SQ_ERR_CUDA, "error slot");
  InferParams p;
  p.rays = d_rays;
  p.n = n;
  p.f = g->feat;
  p.w1_img = g->w1_img;
  p.w23_img = g->w23_img;
  p.w4_img = g->w4_img;
  p.bias = g->infer_bias;
  p.n_chunks = g->n_out / 128;
  p.n_buckets = g->n_buckets;
  p.out = d_bucket;
  p.err = err;
  static std::once_flag attr;
  std::call_once(attr, [] {
    cudaFuncSetAttribute(guide_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(InferSmem::bytes));
  });
  const uint32_t tiles = (n + 255) / 256;
  const uint32_t grid = std::min<uint32_t>(tiles, uint32_t(ctx->sm_count));
  guide_infer_kernel<<<grid, kInferThreads, InferSmem::bytes, ctx->stream>>>(p);
  ctx->launches++;
  CK(cudaGetLastError());
  return SQ_OK;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================

extern "C" void sq_guide_config_default(sq_guide_config* c) {
  if (!c) return;
  c->depth = 12;
  c->batch = 8192;
  c->lr = 1e-3f;
  c->weight_decay = 0.01f;
  c->beta1 = 0.9f;
  c->beta2 = 0.999f;
  c->eps = 1e-8f;
  c->seed = 0;
}

extern "C" int32_t sq_guide_destroy(sq_guide* g) {
  if (!g) return SQ_OK;
  cudaSetDevice(g->device);
  for (void* p : g->allocs) cudaFree(p);  // cudaFree waits for work using the memory
  if (g->d_leaf) cudaFree(g->d_leaf);
  if (g->d_perm) cudaFree(g->d_perm);
  delete g;
  return SQ_OK;
}

extern "C" int32_t sq_guide_create(sq_ctx* ctx, const sq_bvh* b, const sq_guide_config* cfg, sq_guide** out) {
  if (!ctx || !b || !out) return SQ_ERR_INVALID;
  *out = nullptr;
  if (b->dim != 3 || b->prec != 32) return fail(ctx, SQ_ERR_UNSUPPORTED, "the learned guide needs a D = 3 f32 scene");
  if (b->n_nodes == 0) return fail(ctx, SQ_ERR_INVALID, "the learned guide needs a non-empty scene");
  sq_guide_config c;
  sq_guide_config_default(&c);
  if (cfg) c = *cfg;
  if (c.batch == 0 || c.batch % 128 || c.depth > 24) return fail(ctx, SQ_ERR_INVALID, "batch must be a positive multiple of 128, depth <= 24");
  CK(cudaSetDevice(ctx->device));
  auto g = std::make_unique<sq_guide>();
  g->ctx = ctx;
  g->device = ctx->device;
  g->bvh = b;
  g->cfg = c;
  g->B = c.batch;
  std::vector<uint2> table;
  std::vector<uint32_t> starts, sibs;
  g->sib_stride = std::max<uint32_t>(c.depth, 1u);
  build_buckets(b, c.depth, table, starts, sibs, g->sib_stride);
  g->n_buckets = uint32_t(table.size());
  g->n_out = (g->n_buckets + 127) / 128 * 128;
  if (g->n_out > 4096) return fail(ctx, SQ_ERR_INVALID, "more than 4096 buckets: lower the depth");
  // scene box for the features
  float root[6];
  CK(cudaMemcpy(root, b->d_root, sizeof(root), cudaMemcpyDeviceToHost));
  for (int i = 0; i < 3; ++i) {
    g->feat.lo[i] = root[i];
    const float ext = root[3 + i] - root[i];
    g->feat.inv[i] = ext > 0.f ? 1.0f / ext : 0.f;
  }
  // parameter layout
  size_t o = 0;
  auto take = [&](size_t n) { size_t r = o; o += (n + 3) / 4 * 4; return r; };
  g->oW1 = take(size_t(kHidden) * kInPad);
  g->ob1 = take(kHidden);
  g->oW2 = take(size_t(kHidden) * kHidden);
  g->ob2 = take(kHidden);
  g->oW3 = take(size_t(kHidden) * kHidden);
  g->ob3 = take(kHidden);
  g->oW4 = take(size_t(g->n_out) * kHidden);
  g->ob4 = take(g->n_out);
  g->n_p = o;
  sq_guide* gp = g.get();
  int32_t rc;
  auto A = [&](auto** p, size_t bytes) { return galloc(gp, reinterpret_cast<void**>(p), bytes); };
  const size_t NO = g->n_out, B = g->B;
  if ((rc = A(&g->P, g->n_p * 4)) || (rc = A(&g->G, g->n_p * 4)) || (rc = A(&g->M, g->n_p * 4)) ||
      (rc = A(&g->V, g->n_p * 4)) || (rc = A(&g->W1b, kHidden * kInPad * 2)) ||
      (rc = A(&g->W2b, kHidden * kHidden * 2)) || (rc = A(&g->W3b, kHidden * kHidden * 2)) ||
      (rc = A(&g->W4b, NO * kHidden * 2)) || (rc = A(&g->W2bT, kHidden * kHidden * 2)) ||
      (rc = A(&g->W3bT, kHidden * kHidden * 2)) || (rc = A(&g->W4bT, NO * kHidden * 2)) ||
      (rc = A(&g->w1_img, 16384)) || (rc = A(&g->w23_img, 2 * kChunkBytes)) ||
      (rc = A(&g->w4_img, NO / 128 * kChunkBytes)) || (rc = A(&g->infer_bias, (384 + NO) * 4)) ||
      (rc = A(&g->d_buckets, table.size() * sizeof(uint2))) || (rc = A(&g->d_bucket_sibs, sibs.size() * 4)) ||
      (rc = A(&g->d_bucket_of_id, size_t(b->n_prims) * 4)) ||
      (rc = A(&g->X, B * kInPad * 2)) || (rc = A(&g->XT, size_t(kHidden) * B * 2)) ||
      (rc = A(&g->Z, B * std::max<size_t>(NO, kHidden) * 4)) || (rc = A(&g->dZ4, B * NO * 2)) ||
      (rc = A(&g->dZ4T, B * NO * 2)) || (rc = A(&g->dZ, B * kHidden * 2)) || (rc = A(&g->dZT, B * kHidden * 2)) ||
      (rc = A(&g->dH, B * kHidden * 4)) || (rc = A(&g->loss, 16)) || (rc = A(&g->count, 16)) ||
      (rc = A(&g->b_rays, B * 6 * 4)) || (rc = A(&g->b_labels, B * 4))) {
    sq_guide_destroy(g.release());
    return rc;
  }
  for (int l = 0; l < 3; ++l)
    if ((rc = A(&g->H[l], B * kHidden * 2)) || (rc = A(&g->HT[l], B * kHidden * 2))) {
      sq_guide_destroy(g.release());
      return rc;
    }
  // zero: moments, X^T (rows past the features stay zero), padded W1 columns
  CK(cudaMemset(g->M, 0, g->n_p * 4));
  CK(cudaMemset(g->V, 0, g->n_p * 4));
  CK(cudaMemset(g->XT, 0, size_t(kHidden) * B * 2));
  // bucket table and per-primitive buckets
  CK(cudaMemcpy(g->d_buckets, table.data(), table.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g->d_bucket_sibs, sibs.data(), sibs.size() * 4, cudaMemcpyHostToDevice));
  {
    uint32_t* d_starts = nullptr;
    CK(cudaMalloc(&d_starts, starts.size() * 4));
    CK(cudaMemcpy(d_starts, starts.data(), starts.size() * 4, cudaMemcpyHostToDevice));
    bucket_of_id_kernel<<<blocks_for(b->n_prims, 256), 256, 0, ctx->stream>>>(b->d_prim_ids, d_starts,
                                                                              uint32_t(starts.size()),
                                                                              g->d_bucket_of_id, b->n_prims);
    ctx->launches++;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(d_starts));
  }
  // initial weights: uniform +-1/sqrt(fan_in) (torch.nn.Linear's default bounds)
  std::vector<float> h(host_count(gp));
  uint64_t s = c.seed;
  size_t k = 0;
  auto fill = [&](size_t n, uint32_t fan_in) {
    const double bound = 1.0 / std::sqrt(double(fan_in));
    for (size_t i = 0; i < n; ++i) {
      const double u = double(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
      h[k++] = float((2.0 * u - 1.0) * bound);
    }
  };
  fill(size_t(kHidden) * kInputs, kInputs);
  fill(kHidden, kInputs);
  fill(size_t(kHidden) * kHidden, kHidden);
  fill(kHidden, kHidden);
  fill(size_t(kHidden) * kHidden, kHidden);
  fill(kHidden, kHidden);
  fill(NO * kHidden, kHidden);
  fill(NO, kHidden);
  *out = g.release();
  if ((rc = sq_guide_set_params(*out, h.data(), h.size()))) {
    sq_guide_destroy(*out);
    *out = nullptr;
    return rc;
  }
  return SQ_OK;
}

extern "C" int32_t sq_guide_get_info(const sq_guide* g, sq_guide_info* info) {
  if (!g || !info) return SQ_ERR_INVALID;
  info->n_buckets = g->n_buckets;
  info->n_out = g->n_out;
  info->hidden = kHidden;
  info->inputs = kInputs;
  info->n_params = host_count(g);
  info->steps = g->steps;
  return SQ_OK;
}

extern "C" int32_t sq_guide_set_params(sq_guide* g, const float* host, uint64_t count) {
  if (!g || !host) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  if (count != host_count(g)) return fail(ctx, SQ_ERR_INVALID, "parameter count mismatch");
  std::vector<float> d;
  host_to_dev(g, host, d);
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(g->P, d.data(), g->n_p * 4, cudaMemcpyHostToDevice, ctx->stream));
  int32_t rc = refresh_bf16(g);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

static int32_t get_vec(sq_guide* g, const float* dsrc, float* host, uint64_t count) {
  if (!g || !host) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  if (count != host_count(g)) return fail(ctx, SQ_ERR_INVALID, "parameter count mismatch");
  std::vector<float> d(g->n_p);
  CK(cudaMemcpyAsync(d.data(), dsrc, g->n_p * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  dev_to_host(g, d, host);
  return SQ_OK;
}

extern "C" int32_t sq_guide_get_params(sq_guide* g, float* host, uint64_t count) {
  return g ? get_vec(g, g->P, host, count) : SQ_ERR_INVALID;
}

extern "C" int32_t sq_guide_get_grads(sq_guide* g, float* host, uint64_t count) {
  return g ? get_vec(g, g->G, host, count) : SQ_ERR_INVALID;
}

extern "C" int32_t sq_guide_label_d(sq_guide* g, const float* d_rays, uint32_t n, float max_toi, int32_t* d_labels) {
  if (!g || (n && (!d_rays || !d_labels))) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  if (n == 0) return SQ_OK;
  if (g->leaf_cap < n) {
    CK(cudaStreamSynchronize(ctx->stream));
    if (g->d_leaf) CK(cudaFree(g->d_leaf));
    g->d_leaf = nullptr;
    g->leaf_cap = 0;
    CK(cudaMalloc(&g->d_leaf, size_t(n) * 4));
    g->leaf_cap = n;
  }
  sq_hits o{};
  o.leaf = g->d_leaf;
  int32_t rc = sq_raycast_nearest_d(ctx, g->bvh, d_rays, n, max_toi, nullptr, nullptr, &o, nullptr);
  if (rc) return rc;
  labels_kernel<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(g->d_leaf, g->d_bucket_of_id, d_labels, n);
  ctx->launches++;
  CK(cudaGetLastError());
  return SQ_OK;
}

extern "C" int32_t sq_guide_forward_backward_d(sq_guide* g, const float* d_rays, const int32_t* d_labels,
                                               float* loss) {
  if (!g || !d_rays || !d_labels) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  CK(cudaSetDevice(ctx->device));
  int32_t rc = forward_backward(g, d_rays, d_labels);
  if (rc) return rc;
  if ((rc = check_err(ctx, g_err_slot(ctx)))) return rc;
  return loss ? read_loss(g, loss) : SQ_OK;
}

extern "C" int32_t sq_guide_train_step_d(sq_guide* g, const float* d_rays, const int32_t* d_labels, float* loss) {
  if (!g || !d_rays || !d_labels) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  CK(cudaSetDevice(ctx->device));
  int32_t rc = forward_backward(g, d_rays, d_labels);
  if (rc) return rc;
  if (loss && (rc = read_loss(g, loss))) return rc;
  return adam_step(g);
}

extern "C" int32_t sq_guide_train_d(sq_guide* g, const float* d_rays, const int32_t* d_labels, uint32_t n,
                                    uint32_t epochs, float* loss_per_epoch) {
  if (!g || (n && (!d_rays || !d_labels))) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  CK(cudaSetDevice(ctx->device));
  const uint32_t steps = n / g->B;
  int32_t rc;
  if (g->perm_cap < n) {
    CK(cudaStreamSynchronize(ctx->stream));
    if (g->d_perm) CK(cudaFree(g->d_perm));
    g->d_perm = nullptr;
    g->perm_cap = 0;
    CK(cudaMalloc(&g->d_perm, size_t(n) * 4));
    g->perm_cap = n;
  }
  std::vector<uint32_t> perm(n);
  for (uint32_t e = 0; e < epochs; ++e) {
    // A fresh shuffle per epoch (Fisher-Yates on SplitMix64, seeded by the
    // config seed and the optimiser step), so batches mix both ray kinds.
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    uint64_t st = g->cfg.seed ^ (0x5851F42D4C957F2Dull * (g->steps + 1));
    for (uint32_t i = n; i > 1; --i) {
      const uint32_t j = uint32_t(splitmix(st) % i);
      std::swap(perm[i - 1], perm[j]);
    }
    CK(cudaMemcpyAsync(g->d_perm, perm.data(), size_t(n) * 4, cudaMemcpyHostToDevice, ctx->stream));
    double sum = 0.0;
    for (uint32_t s = 0; s < steps; ++s) {
      gather_batch_kernel<<<blocks_for(g->B, 256), 256, 0, ctx->stream>>>(d_rays, d_labels, g->d_perm + size_t(s) * g->B,
                                                                          g->B, g->b_rays, g->b_labels);
      ctx->launches++;
      if ((rc = forward_backward(g, g->b_rays, g->b_labels))) return rc;
      if (loss_per_epoch) {
        float l = 0.f;
        if ((rc = read_loss(g, &l))) return rc;
        sum += l;
      }
      if ((rc = adam_step(g))) return rc;
    }
    if (loss_per_epoch) loss_per_epoch[e] = steps ? float(sum / steps) : 0.f;
  }
  return check_err(ctx, g_err_slot(ctx));
}

extern "C" int32_t sq_guide_predict_d(sq_guide* g, const float* d_rays, uint32_t n, int32_t* d_bucket) {
  if (!g || (n && (!d_rays || !d_bucket))) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  CK(cudaSetDevice(ctx->device));
  return predict(g, d_rays, n, d_bucket);
}

extern "C" int32_t sq_raycast_nearest_guided_d(sq_ctx* ctx, const sq_bvh* b, const sq_guide* gc, const float* d_rays,
                                               uint32_t n, float max_toi, const int32_t* d_bucket, const sq_hits* out,
                                               sq_query_stats* stats) {
  if (!ctx || !b || !gc || !out) return SQ_ERR_INVALID;
  sq_guide* g = const_cast<sq_guide*>(gc);
  if (g->bvh != b) return fail(ctx, SQ_ERR_INVALID, "the guide was built for another scene");
  int32_t rc;
  const int32_t* seeds = d_bucket;
  if (!seeds && !stats && n >= (1u << 19)) {
    // Two halves, one on the context's stream and one on its second lane:
    // the second half's inference fills the SMs that the first half's
    // traversal tail leaves idle. Seeds and hits land where one launch
    // would put them.
    if ((rc = arena_reserve(ctx, size_t(n) * 4))) return rc;
    int32_t* d = static_cast<int32_t*>(ctx->arena.p);
    sq_ctx* lane = nullptr;
    if ((rc = sqi::second_lane(ctx, &lane))) return rc;
    sq_ctx* saved = g->ctx;
    g->ctx = ctx;
    rc = refresh_images(g);  // once, before either half predicts
    g->ctx = saved;
    if (rc) return rc;
    const uint64_t lane_launches = lane->launches;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    for (auto& e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaError_t ce = cudaEventRecord(ev[0], ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(lane->stream, ev[0], 0);
    const uint32_t m0 = (n / 2 + 255) / 256 * 256;
    sq_ctx* failed = nullptr;
    for (int k = 0; k < 2 && ce == cudaSuccess && !failed; ++k) {
      sq_ctx* on = k ? lane : ctx;
      const uint32_t s0 = k ? m0 : 0, m = k ? n - m0 : m0;
      sq_hits c = *out;
      c.leaf += s0;
      if (c.toi) c.toi += s0;
      if (c.sub_object) c.sub_object += s0;
      if (c.normal) c.normal += size_t(s0) * 3;
      if (c.point) c.point += size_t(s0) * 3;
      g->ctx = on;
      rc = predict(g, d_rays + size_t(s0) * 6, m, d + s0);
      g->ctx = saved;
      if (!rc) rc = seeded_nearest(on, b, d_rays + size_t(s0) * 6, m, max_toi, d + s0, seed_table(g), c, nullptr);
      if (rc) failed = on;
    }
    // The context's stream takes the lane's half back in every case.
    if (cudaEventRecord(ev[1], lane->stream) == cudaSuccess) cudaStreamWaitEvent(ctx->stream, ev[1], 0);
    for (auto& e : ev) cudaEventDestroy(e);
    ctx->launches += lane->launches - lane_launches;
    if (failed) return failed == ctx ? rc : fail(ctx, rc, lane->err.c_str());
    if (ce != cudaSuccess) return cuda_fail(ctx, "guided halves", ce);
    return SQ_OK;
  }
  if (!seeds && n) {
    if ((rc = arena_reserve(ctx, size_t(n) * 4))) return rc;
    int32_t* d = static_cast<int32_t*>(ctx->arena.p);
    sq_ctx* saved = g->ctx;
    g->ctx = ctx;
    rc = predict(g, d_rays, n, d);
    g->ctx = saved;
    if (rc) return rc;
    seeds = d;
  }
  return seeded_nearest(ctx, b, d_rays, n, max_toi, seeds, seed_table(g), *out, stats);
}

extern "C" int32_t sq_raycast_nearest_guided(sq_ctx* ctx, const sq_bvh* b, const sq_guide* gc, const float* rays,
                                             uint32_t n, float max_toi, const sq_hits* o, sq_query_stats* st) {
  if (!ctx || !b || !gc || !o || !o->leaf || (n && !rays)) return SQ_ERR_INVALID;
  if (n == 0) {
    if (st) *st = sq_query_stats{0, 0, 0, 0};
    return SQ_OK;
  }
  CK(cudaSetDevice(ctx->device));
  Carve cv;
  const size_t o_q = cv.take(size_t(n) * 24), o_b = cv.take(size_t(n) * 4), o_leaf = cv.take(size_t(n) * 4);
  const size_t o_toi = o->toi ? cv.take(size_t(n) * 4) : 0, o_sub = o->sub_object ? cv.take(size_t(n) * 4) : 0;
  const size_t o_nrm = o->normal ? cv.take(size_t(n) * 12) : 0, o_pt = o->point ? cv.take(size_t(n) * 12) : 0;
  int32_t rc;
  if ((rc = arena_reserve(ctx, cv.off))) return rc;
  char* base = static_cast<char*>(ctx->arena.p);
  sq_guide* g = const_cast<sq_guide*>(gc);
  sq_hits dh{};
  dh.leaf = reinterpret_cast<uint32_t*>(base + o_leaf);
  dh.toi = o->toi ? reinterpret_cast<float*>(base + o_toi) : nullptr;
  dh.sub_object = o->sub_object ? reinterpret_cast<uint32_t*>(base + o_sub) : nullptr;
  dh.normal = o->normal ? reinterpret_cast<float*>(base + o_nrm) : nullptr;
  dh.point = o->point ? reinterpret_cast<float*>(base + o_pt) : nullptr;
  const float* d_q = reinterpret_cast<const float*>(base + o_q);
  int32_t* d_b = reinterpret_cast<int32_t*>(base + o_b);
  // Chunked: rays of one chunk are copied in and hits of another copied out
  // while a third is predicted and walked.
  auto in = [&](uint32_t s0, uint32_t m, cudaStream_t sm) -> int32_t {
    CK(cudaMemcpyAsync(base + o_q + size_t(s0) * 24, rays + size_t(s0) * 6, size_t(m) * 24, cudaMemcpyHostToDevice,
                       sm));
    return SQ_OK;
  };
  auto run = [&](sq_ctx* lane, uint32_t s0, uint32_t m) -> int32_t {
    sq_ctx* saved = g->ctx;
    g->ctx = lane;
    int32_t r = predict(g, d_q + size_t(s0) * 6, m, d_b + s0);
    g->ctx = saved;
    if (r) return r;
    sq_hits c = dh;
    c.leaf += s0;
    if (c.toi) c.toi += s0;
    if (c.sub_object) c.sub_object += s0;
    if (c.normal) c.normal += size_t(s0) * 3;
    if (c.point) c.point += size_t(s0) * 3;
    return seeded_nearest(lane, b, d_q + size_t(s0) * 6, m, max_toi, d_b + s0, seed_table(g), c, nullptr);
  };
  auto out = [&](uint32_t s0, uint32_t m, cudaStream_t sm) -> int32_t {
    auto cp = [&](void* dst, const void* src, size_t per) -> int32_t {
      if (dst) CK(cudaMemcpyAsync(static_cast<char*>(dst) + size_t(s0) * per,
                                  static_cast<const char*>(src) + size_t(s0) * per, size_t(m) * per,
                                  cudaMemcpyDeviceToHost, sm));
      return SQ_OK;
    };
    int32_t r;
    if ((r = cp(o->leaf, dh.leaf, 4)) || (r = cp(o->toi, dh.toi, 4)) || (r = cp(o->sub_object, dh.sub_object, 4)) ||
        (r = cp(o->normal, dh.normal, 12)) || (r = cp(o->point, dh.point, 12)))
      return r;
    return SQ_OK;
  };
  // The weight images are refreshed once, on the context's stream, before
  // either lane predicts from them.
  {
    sq_ctx* saved = g->ctx;
    g->ctx = ctx;
    rc = refresh_images(g);
    g->ctx = saved;
    if (rc) return rc;
  }
  if ((rc = sqi::pipelined(ctx, n, in, run, out))) return rc;
  if (st) *st = sq_query_stats{0, 0, 0, 0};
  return SQ_OK;
}

namespace {
constexpr uint32_t kSaveMagic = 0x47515321u;  // "!SQG"
struct SaveHeader {
  uint32_t magic, version, n_out, n_buckets, steps, depth;
  uint64_t n_p;
  sq_guide_config cfg;
};
}  // namespace

extern "C" int32_t sq_guide_save(const sq_guide* g, void* buf, size_t cap, size_t* size) {
  if (!g || !size) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  const size_t need = sizeof(SaveHeader) + 3 * g->n_p * 4;
  *size = need;
  if (!buf || cap < need) return buf ? fail(ctx, SQ_ERR_CAPACITY, "buffer too small") : SQ_OK;
  SaveHeader h{kSaveMagic, 1u, g->n_out, g->n_buckets, g->steps, g->cfg.depth, g->n_p, g->cfg};
  std::memcpy(buf, &h, sizeof(h));
  char* p = static_cast<char*>(buf) + sizeof(h);
  CK(cudaMemcpyAsync(p, g->P, g->n_p * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(p + g->n_p * 4, g->M, g->n_p * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(p + 2 * g->n_p * 4, g->V, g->n_p * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

extern "C" int32_t sq_guide_load(sq_guide* g, const void* buf, size_t size) {
  if (!g || !buf) return SQ_ERR_INVALID;
  sq_ctx* ctx = g->ctx;
  SaveHeader h;
  if (size < sizeof(h)) return fail(ctx, SQ_ERR_INVALID, "truncated guide");
  std::memcpy(&h, buf, sizeof(h));
  if (h.magic != kSaveMagic || h.version != 1u) return fail(ctx, SQ_ERR_INVALID, "not a saved guide");
  if (h.n_out != g->n_out || h.n_buckets != g->n_buckets || h.n_p != g->n_p || h.depth != g->cfg.depth)
    return fail(ctx, SQ_ERR_INVALID, "the saved guide was built for another scene or depth");
  if (size < sizeof(h) + 3 * g->n_p * 4) return fail(ctx, SQ_ERR_INVALID, "truncated guide");
  const char* p = static_cast<const char*>(buf) + sizeof(h);
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(g->P, p, g->n_p * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(g->M, p + g->n_p * 4, g->n_p * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(g->V, p + 2 * g->n_p * 4, g->n_p * 4, cudaMemcpyHostToDevice, ctx->stream));
  g->steps = h.steps;
  g->cfg = h.cfg;
  int32_t rc = refresh_bf16(g);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return SQ_OK;
}

extern "C" int32_t sq_gemm_bf16_tn_d(sq_ctx* ctx, const uint16_t* d_a, const uint16_t* d_b, float* d_c, uint32_t m,
                                     uint32_t n, uint32_t k, uint32_t lda, uint32_t ldb, uint32_t ldc) {
  if (!ctx || (m && n && (!d_a || !d_b || !d_c))) return SQ_ERR_INVALID;
  if (m < 128 || n < 128 || k < 64) return fail(ctx, SQ_ERR_INVALID, "gemm: m and n must be >= 128 and k >= 64");
  CK(cudaSetDevice(ctx->device));
  int32_t rc = gemm(ctx, reinterpret_cast<const bf16*>(d_a), m, lda, reinterpret_cast<const bf16*>(d_b), n, ldb, d_c,
                    m, n, k, ldc);
  if (rc) return rc;
  return check_err(ctx, g_err_slot(ctx));
}
