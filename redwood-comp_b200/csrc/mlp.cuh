// Inference of the boundary MLP (16 -> 64 -> 64 -> 1, ReLU) on the tensor
// cores, shared by rw_tree_mlp_forward (k_mlp.cu) and the learned sort's
// boundary kernel (k_learned.cu).
//
// Numerics: the inputs, W1, W2 and the hidden activations are rounded to BF16
// (round to nearest even); both 64-wide layers are tcgen05 MMAs with FP32
// accumulation in tensor memory, the biases are added in FP32 after the
// products; the last layer (64 -> 1, W3 rounded to BF16) is an FP32 dot product
// per row on the CUDA cores, b3 first, then units 0..63 in order.  The
// training kernel (k_mlp_grad) keeps its activations in FP32.
#pragma once

#include <cuda_bf16.h>

#include "internal.hpp"
#include "tcgen05.cuh"

namespace rwt {

// parameter layout (FP32): W1 [64][16], b1 [64], W2 [64][64], b2 [64], W3 [64], b3
constexpr int kMlpOffW1 = 0, kMlpOffB1 = kMlpOffW1 + kMlpHidden * kMlpIn,
              kMlpOffW2 = kMlpOffB1 + kMlpHidden,
              kMlpOffB2 = kMlpOffW2 + kMlpHidden * kMlpHidden,
              kMlpOffW3 = kMlpOffB2 + kMlpHidden, kMlpOffB3 = kMlpOffW3 + kMlpHidden;
static_assert(kMlpOffB3 + 1 == kMlpParams, "parameter layout");

// One tile: 128 rows, 128 threads (thread t: row t), one CTA.
constexpr int kMlpTcRows = 128, kMlpTcThreads = 128;
constexpr uint32_t kMlpTcCols = 128;  // TMEM columns: layer 1 in [0, 64), layer 2 in [64, 128)

struct MlpTcSmem {
  alignas(1024) unsigned char a1[kMlpTcRows * kMlpIn * 2];        // inputs, K-major
  alignas(128) unsigned char b1[kMlpHidden * kMlpIn * 2];         // W1 (rows: units)
  alignas(128) unsigned char a2[kMlpTcRows * kMlpHidden * 2];     // hidden layer 1
  alignas(128) unsigned char b2[kMlpHidden * kMlpHidden * 2];     // W2
  float bias1[kMlpHidden], bias2[kMlpHidden], w3[kMlpHidden];
  uint64_t bar[2];  // completion of layer 1's and layer 2's MMAs
  uint32_t tmem;    // TMEM base address
};

// 8 floats -> 8 BF16 in one 16-byte unit (element i at bytes 2i, 2i + 1)
__device__ __forceinline__ uint4 pack_bf16x8(const float* v) {
  uint32_t w[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<const uint32_t*>(&p);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// Evaluates the network for the CTA's 128 rows.  feat(t, x) fills row t's 16
// inputs and returns whether the row is live (a dead row's inputs are zeros);
// out(t, y, ok) receives row t's output, ok false when a wait on the tensor
// core ran out (then *err |= 1 and y is meaningless).  Every thread of the CTA
// must call it, once.
template <typename Feat, typename Out>
__device__ __forceinline__ void mlp_tile_tc(const float* __restrict__ params, Feat feat, Out out,
                                            uint32_t* __restrict__ err) {
  __shared__ MlpTcSmem sm;
  const int tid = int(threadIdx.x), warp = tid >> 5;
  if (warp == 0) {
    tc::tmem_alloc(&sm.tmem, kMlpTcCols);
    tc::fence_before_sync();
  }
  if (tid == 32) {
    bulk_barrier_init(&sm.bar[0]);
    bulk_barrier_init(&sm.bar[1]);
  }
  // weights rounded to BF16, output units as the MMA's B rows
  for (int i = tid; i < kMlpHidden * kMlpIn; i += kMlpTcThreads)
    *reinterpret_cast<__nv_bfloat16*>(sm.b1 + tc::kmajor_offset<kMlpIn>(i / kMlpIn, i % kMlpIn)) =
        __float2bfloat16_rn(params[kMlpOffW1 + i]);
  for (int i = tid; i < kMlpHidden * kMlpHidden; i += kMlpTcThreads)
    *reinterpret_cast<__nv_bfloat16*>(
        sm.b2 + tc::kmajor_offset<kMlpHidden>(i / kMlpHidden, i % kMlpHidden)) =
        __float2bfloat16_rn(params[kMlpOffW2 + i]);
  if (tid < kMlpHidden) {
    sm.bias1[tid] = params[kMlpOffB1 + tid];
    sm.bias2[tid] = params[kMlpOffB2 + tid];
    sm.w3[tid] = __bfloat162float(__float2bfloat16_rn(params[kMlpOffW3 + tid]));
  }
  const float b3 = params[kMlpOffB3];
  float x[kMlpIn];
  const bool live = feat(tid, x);
  if (!live) {
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) x[k] = 0.0f;
  }
#pragma unroll
  for (int c = 0; c < kMlpIn / 8; ++c)
    *reinterpret_cast<uint4*>(sm.a1 + tc::kmajor_offset<kMlpIn>(tid, 8 * c)) = pack_bf16x8(x + 8 * c);
  tc::fence_smem_for_mma();
  __syncthreads();
  tc::fence_after_sync();

  const uint32_t taddr = sm.tmem;
  const uint32_t my_lanes = taddr + (uint32_t(warp * 32) << 16);  // this warp's TMEM lanes
  constexpr uint32_t idesc = tc::idesc_bf16_f32<kMlpTcRows, kMlpHidden>();
  constexpr uint32_t kSbo1 = kMlpIn / 8 * 128, kSbo2 = kMlpHidden / 8 * 128;
  // layer 1: one MMA of K = 16
  if (tid == 0) {
    tc::mma_bf16(taddr, tc::smem_desc(smem_addr(sm.a1), 128, kSbo1),
                 tc::smem_desc(smem_addr(sm.b1), 128, kSbo1), idesc, false);
    tc::mma_commit(&sm.bar[0]);
  }
  bool ok = !__syncthreads_or(!bulk_wait(&sm.bar[0], kSpinLimit));
  tc::fence_after_sync();
  if (ok) {  // block-uniform
#pragma unroll
    for (int q = 0; q < kMlpHidden / 16; ++q) {
      float h[16];
      tc::tmem_load16(my_lanes + uint32_t(16 * q), h);
#pragma unroll
      for (int i = 0; i < 16; ++i) h[i] = fmaxf(h[i] + sm.bias1[16 * q + i], 0.0f);
#pragma unroll
      for (int c = 0; c < 2; ++c)
        *reinterpret_cast<uint4*>(sm.a2 + tc::kmajor_offset<kMlpHidden>(tid, 16 * q + 8 * c)) =
            pack_bf16x8(h + 8 * c);
    }
  }
  tc::fence_smem_for_mma();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  // layer 2: four MMAs of K = 16 into columns [64, 128)
  bool issued2 = false;
  if (ok) {
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < kMlpHidden / 16; ++s)
        tc::mma_bf16(taddr + kMlpHidden,
                     tc::smem_desc(smem_addr(sm.a2) + 256u * s, 128, kSbo2),
                     tc::smem_desc(smem_addr(sm.b2) + 256u * s, 128, kSbo2), idesc, s > 0);
      tc::mma_commit(&sm.bar[1]);
    }
    issued2 = true;
    ok = !__syncthreads_or(!bulk_wait(&sm.bar[1], kSpinLimit));
    tc::fence_after_sync();
  }
  float y = b3;
  if (ok) {
#pragma unroll
    for (int q = 0; q < kMlpHidden / 16; ++q) {
      float h[16];
      tc::tmem_load16(my_lanes + uint32_t(kMlpHidden + 16 * q), h);
#pragma unroll
      for (int i = 0; i < 16; ++i)
        y = fmaf(sm.w3[16 * q + i], fmaxf(h[i] + sm.bias2[16 * q + i], 0.0f), y);
    }
  } else {
    // report, then give the MMAs in flight one more bounded wait before the
    // tensor memory they write is freed
    if (tid == 0 && err) atomicOr(err, 1u);
    bulk_wait(issued2 ? &sm.bar[1] : &sm.bar[0], kSpinLimit);
  }
  out(tid, y, ok);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(taddr, kMlpTcCols);
}

}  // namespace rwt
