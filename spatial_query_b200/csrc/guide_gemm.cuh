// The tcgen05 GEMM the learned guide trains with:
//   C[M, N] (f32, row-major, ldc) = A[M, K] * B[N, K]^T
// with A and B bf16, row-major (K contiguous), loaded by TMA as 128-byte
// swizzled tiles, multiplied by tcgen05.mma (M = 128, N = BN, K = 16 per
// instruction) into a TMEM accumulator, and written back by four epilogue
// warps through tcgen05.ld.
//
// One CTA per 128 x BN output tile; a 4-stage TMA -> MMA pipeline over K in
// 64-element panels: warp 0 lane 0 issues the loads, warp 1 lane 0 issues the
// MMAs and frees each stage with tcgen05.commit, all four warps drain TMEM.
// Rows and columns past M, N and K are zero-filled by TMA and masked at the
// store, so any M, N and any K that is a multiple of 8 (16-byte rows) work.
#pragma once

#include "umma.cuh"

namespace sq {
namespace guide {

constexpr int kGemmStages = 4;
constexpr int kGemmThreads = 128;

template <int BN> struct GemmSmem {
  static constexpr int a_bytes = 128 * 128;  // 128 rows x 64 bf16
  static constexpr int b_bytes = BN * 128;
  static constexpr int stage = a_bytes + b_bytes;
  static constexpr int bytes = kGemmStages * stage + 1024 /* barriers */ + 1024 /* alignment slack */;
};

// Epilogue modes: plain store, or add into C.
enum GemmEpi : int { kEpiStore = 0, kEpiAccumulate = 1 };

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
    gemm_tn_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, float* __restrict__ C,
                   int M, int N, int K, int ldc, int epi, int* err) {
  using S = GemmSmem<BN>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = umma::smem_u32(smem_raw);
  uint8_t* base = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kGemmStages * S::stage);
  uint64_t* empty = full + kGemmStages;
  uint64_t* done = empty + kGemmStages;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  int* s_err = reinterpret_cast<int*>(tslot + 1);
  int* s_issued = s_err + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
  const int kt_n = (K + 63) / 64;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kGemmStages; ++s) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    umma::mbar_init(done, 1);
    *s_err = 0;
    *s_issued = 0;
    umma::fence_barrier_init();
  }
  __syncwarp();
  if (warp == 0) umma::tmem_alloc(tslot, BN);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;

  if (warp == 0 && lane == 0) {
    int kt = 0;
    for (; kt < kt_n; ++kt) {
      const int s = kt % kGemmStages;
      if (kt >= kGemmStages && !umma::mbar_wait(&empty[s], ((kt / kGemmStages) + 1) & 1)) {
        atomicExch(s_err, 1);
        break;
      }
      if (*(volatile int*)s_err) break;
      uint8_t* sa = base + s * S::stage;
      umma::mbar_arrive_expect_tx(&full[s], S::stage);
      umma::tma_load_2d(sa, &ta, &full[s], kt * 64, m0);
      umma::tma_load_2d(sa + S::a_bytes, &tb, &full[s], kt * 64, n0);
    }
    *s_issued = kt;
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc = umma::idesc_bf16(128, BN);
    for (int kt = 0; kt < kt_n; ++kt) {
      const int s = kt % kGemmStages;
      if (!umma::mbar_wait(&full[s], (kt / kGemmStages) & 1)) {
        atomicExch(s_err, 2);
        break;
      }
      umma::tc_fence_after();
      const uint8_t* sa = base + s * S::stage;
      const uint64_t ad = umma::desc_sw128(umma::smem_u32(sa));
      const uint64_t bd = umma::desc_sw128(umma::smem_u32(sa + S::a_bytes));
#pragma unroll
      for (int k = 0; k < 4; ++k) umma::mma_bf16(tbase, ad + 2 * k, bd + 2 * k, idesc, (kt | k) != 0);
      umma::mma_commit(&empty[s]);
    }
    umma::mma_commit(done);
  }
  __syncwarp();

  const bool ok = umma::mbar_wait(done, 0);
  umma::tc_fence_after();
  if (!ok) atomicExch(s_err, 3);
  __syncthreads();
  const bool good = (*(volatile int*)s_err) == 0 && kt_n > 0;
  const int row = m0 + warp * 32 + lane;
  if (good) {
#pragma unroll 1
    for (int c = 0; c < BN; c += 32) {
      float v[32];
      umma::tmem_ld32(tbase + (uint32_t(warp * 32) << 16) + uint32_t(c), v);
      if (row < M) {
        float* dst = C + size_t(row) * ldc + n0 + c;
        const int lim = N - (n0 + c);
        if (epi == kEpiAccumulate) {
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (j < lim) dst[j] += v[j];
        } else if (lim >= 32 && (ldc & 3) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0) {
#pragma unroll
          for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(dst + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (j < lim) dst[j] = v[j];
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, *s_err ? *s_err : 4);
    // Let loads still in flight land before the CTA's shared memory goes away.
    const int issued = *s_issued;
    for (int kt = issued - kGemmStages; kt < issued; ++kt)
      if (kt >= 0) umma::mbar_wait(&full[kt % kGemmStages], (kt / kGemmStages) & 1, 100000000ull);
  }
  umma::tc_fence_before();
  __syncthreads();
  __syncwarp();
  if (warp == 0) umma::tmem_dealloc(tbase, BN);
}

}  // namespace guide
}  // namespace sq
