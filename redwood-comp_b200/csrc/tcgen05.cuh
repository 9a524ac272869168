// Fifth-generation tensor core (tcgen05) helpers for sm_100a: tensor memory
// (TMEM) allocation, the shared-memory matrix and instruction descriptors of a
// BF16 x BF16 -> FP32 MMA, the MMA itself, its completion on an mbarrier and
// the accumulator read-back.  Inline PTX; used by the boundary network of the
// learned-CDF sort (k_learned.cu, k_mlp.cu).
//
// Operand layout (K-major, no swizzle): a matrix of R rows x K bf16 columns is
// stored as core matrices of 8 rows x 8 columns (8 rows of 16 bytes, 128
// contiguous bytes); element (r, k) sits at byte
//   (r / 8) * (K / 8) * 128 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// so the two 16-byte column chunks one MMA of K = 16 reads are 128 bytes apart
// (leading byte offset) and consecutive groups of 8 rows K / 8 * 128 bytes
// apart (stride byte offset); step s of K = 16 starts 256 s bytes further.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace rwt {
namespace tc {

// byte offset of element (r, k) in the layout above
template <int K>
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k) {
  return uint32_t((r >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all in 16-byte units, 14 bits each), descriptor version 1 (bits
// 46-47, sm_100), base offset 0, no swizzle (bits 61-63 zero).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((saddr >> 4) & 0x3fffu) | (uint64_t((lbo >> 4) & 0x3fffu) << 16) |
         (uint64_t((sbo >> 4) & 0x3fffu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B (both K-major) and an
// FP32 accumulator: D format bits 4-5 = 1, A and B format bits 7-9 and 10-12
// = 1 (BF16), N / 8 in bits 17-22, M / 16 in bits 24-28.
template <int M, int N>
__host__ __device__ constexpr uint32_t idesc_bf16_f32() {
  static_assert((M == 64 && N % 8 == 0 && N >= 8 && N <= 256) ||
                    (M == 128 && N % 16 == 0 && N >= 16 && N <= 256),
                "shape of a one-CTA kind::f16 MMA");
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// One warp: allocates `ncols` TMEM columns (a power of two >= 32) and writes
// their address to *slot; then gives up the right to allocate again, so that
// other CTAs on the SM are not kept waiting.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// The same warp that allocated: frees the columns.
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// Ordering of tcgen05 operations around a thread barrier.
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Makes this thread's ordinary shared-memory writes visible to the tensor
// core (the async proxy); each writer calls it before the barrier that
// precedes the MMA.
__device__ __forceinline__ void fence_smem_for_mma() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One thread: D[tmem] = A * B^T, or D += A * B^T when `accumulate`.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(uint32_t(accumulate))
      : "memory");
}

// The issuing thread: one arrival on `bar` once all its MMAs have completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

// Whole warp: 16 consecutive FP32 columns of the warp's 32 TMEM lanes (lane
// l of the warp gets its own TMEM lane's values).  The load and its wait are
// one asm statement, so no use of the registers can be scheduled between them.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace rwt
