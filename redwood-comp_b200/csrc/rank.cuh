// Stable warp-level ranking of keys by one radix digit, shared by the
// onesweep passes (k_keys.cu) and the per-bucket sort of the learned-CDF sort
// (k_learned.cu).  A warp holds 32*KPT keys, key i of lane l at position
// 32*i + l of the warp's run; ranks follow that order (stable).
#pragma once

#include <cstdint>

#include "common.cuh"

namespace rwt {

template <int D, int THREADS>
__device__ __forceinline__ void digit_exclusive_scan(const uint32_t* s_cnt,
                                                     uint32_t* s_start,
                                                     uint32_t* s_warp) {
  constexpr int RADIX = 1 << D;
  constexpr int R = (RADIX + THREADS - 1) / THREADS;  // digits per thread
  static_assert(R * THREADS >= RADIX, "every digit needs a start offset");
  const int first = threadIdx.x * R;
  uint32_t local = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) local += first + r < RADIX ? s_cnt[first + r] : 0u;
  uint32_t total;
  uint32_t run = block_exclusive_scan<THREADS>(local, s_warp, &total);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (first + r < RADIX) {
      s_start[first + r] = run;
      run += s_cnt[first + r];
    }
  }
}

// Warp ranking schemes: all return, for each lane, the mask of valid lanes in
// its warp holding the same digit (the lane's stable rank is the popcount of
// the mask below it).
enum RankMode : int {
  kRankBallot = 0,
  kRankMatchAny = 1,
  kRankAtomicOr = 2,
  kRankHalfPacked = 3,  // per half-warp: one word per digit, count << 16 | 16-lane mask
  // a sort's mode, not a warp_rank mode: atomic OR for the passes over full
  // digits, ballots over only the code's remaining bits for the top pass
  // (skewed top digits put many lanes of a warp on one shared word, which the
  // atomics serialise; ballots cost the same whatever the digits)
  kRankMixed = 4
};

// D ballots, one per digit bit (warp-level multi-split).
template <int D>
__device__ __forceinline__ uint32_t match_ballot(uint32_t digit, uint32_t valid_mask) {
  uint32_t peers = valid_mask;
#pragma unroll
  for (int b = 0; b < D; ++b) {
    const bool bit = (digit >> b) & 1u;
    const uint32_t v = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? v : ~v;
  }
  return peers;
}

// Warp ranks (< 32 * KPT) packed into registers: three 10-bit ranks per
// register while a warp holds at most 1,024 keys, else two 16-bit ranks.
template <int KPT>
struct RankPack {
  static_assert(32 * KPT <= 65536, "warp ranks fit 16 bits");
  static constexpr int kBits = 32 * KPT <= 1024 ? 10 : 16;
  static constexpr int kPer = 32 / kBits;
  static constexpr int kRegs = (KPT + kPer - 1) / kPer;
  __device__ __forceinline__ static void set(uint32_t (&r)[kRegs], int i, uint32_t v) {
    if (i % kPer == 0) r[i / kPer] = v;
    else r[i / kPer] |= v << ((i % kPer) * kBits);
  }
  __device__ __forceinline__ static uint32_t get(const uint32_t (&r)[kRegs], int i) {
    return (r[i / kPer] >> ((i % kPer) * kBits)) & ((1u << kBits) - 1u);
  }
};

// Stable ranks of one warp's 32*KPT keys among the warp's keys of the same
// digit (order: step, then lane); the warp's digit counters `wh` advance.
// FULL: every key is in range, so no per-key checks are made.
// BB: the digit bits the ballot scheme compares (the bits above them are zero
// in every key of this pass).
// RANK kRankMixed: `ballots` (block-uniform) picks the ballot scheme, else
// the atomic-OR one, per call.
template <int D, int KPT, int RANK, bool FULL, int BB = D, typename K>
__device__ __forceinline__ void warp_rank(const K (&keys)[KPT],
                                          uint32_t (&rank2)[RankPack<KPT>::kRegs],
                                          int shift, uint32_t wbase, uint32_t n, uint32_t* wh,
                                          uint32_t* wm, int steps = KPT, bool ballots = false) {
  const bool by_ballot = RANK == kRankBallot || (RANK == kRankMixed && ballots);
  constexpr uint32_t RADIX = 1u << D;
  const uint32_t lane = lane_id();
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    if (!FULL && i >= steps) break;  // warp-uniform: the warp's keys end here
    const bool valid = FULL || wbase + 32u * i < n;
    const uint32_t dig = uint32_t(keys[i] >> shift) & (RADIX - 1);
    uint32_t peers;
    static_assert(BB >= 1 && BB <= D, "ballot bits within the digit");
    if (by_ballot) {
      peers = match_ballot<BB>(dig, FULL ? 0xffffffffu : __ballot_sync(0xffffffffu, valid));
    } else if (RANK == kRankMatchAny) {
      peers = __match_any_sync(0xffffffffu, valid ? dig : 0xffffffffu);
      if (!valid) peers = 0;
    } else {
      if (valid) atomicOr(&wm[dig], 1u << lane);
      __syncwarp();
      peers = valid ? wm[dig] : 0u;
      __syncwarp();
    }
    const uint32_t below = __popc(peers & lanemask_lt());
    uint32_t prev = 0;
    if (valid && below == 0) {
      // one shared-memory access for the read-modify-write of the counter
      prev = atomicAdd(&wh[dig], uint32_t(__popc(peers)));
      if ((RANK == kRankAtomicOr || RANK == kRankMixed) && !by_ballot) wm[dig] = 0;
    }
    const int leader = valid ? __ffs(peers) - 1 : int(lane);
    prev = __shfl_sync(0xffffffffu, prev, leader);
    RankPack<KPT>::set(rank2, i, prev + below);
    __syncwarp();
  }
}

// Places the warp's keys at their tile positions (wh: the warp's offsets).
template <int D, int KPT, bool FULL, typename K>
__device__ __forceinline__ void warp_place(const K (&keys)[KPT],
                                           const uint32_t (&rank2)[RankPack<KPT>::kRegs], int shift,
                                           uint32_t wbase, uint32_t n, const uint32_t* wh,
                                           K* s_keys, int steps = KPT) {
  constexpr uint32_t RADIX = 1u << D;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    if (!FULL && i >= steps) break;
    if (FULL || wbase + 32u * i < n) {
      const uint32_t dig = uint32_t(keys[i] >> shift) & (RADIX - 1);
      s_keys[wh[dig] + RankPack<KPT>::get(rank2, i)] = keys[i];
    }
  }
}

// ---- half-warp packed ranking (kRankHalfPacked) -----------------------------
// Each half-warp (16 lanes) owns a contiguous run of 16 * KPT keys of its
// warp's 32 * KPT (key i of lane l at position 16 i + (l & 15) of the run), so
// ranks in the order (half-warp, step, lane) are stable.  Per digit a half-warp
// has one shared-memory word: the count of its earlier keys of that digit in
// the high 16 bits and, during a step, the mask of its lanes holding the digit
// in the low 16 bits.  A step costs an atomic OR, one read of the word (count
// and peers together, no shuffle) and the leader's store of the new count -
// three shared-memory accesses where the two-array scheme needs four.  The
// words of half-warp h of a warp sit at 2 d + h: the two halves use the even
// and the odd banks, so their accesses never conflict with each other.
__device__ __forceinline__ uint32_t half_slot(uint32_t dig) {
  return 2u * dig + (lane_id() >> 4);
}

template <int D, int KPT, bool FULL, typename K>
__device__ __forceinline__ void half_rank(const K (&keys)[KPT],
                                          uint32_t (&rank2)[RankPack<KPT>::kRegs], int shift,
                                          uint32_t hbase, uint32_t n, uint32_t* wp) {
  constexpr uint32_t RADIX = 1u << D;
  const uint32_t l16 = lane_id() & 15u;
  const uint32_t lt16 = (1u << l16) - 1u;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const bool valid = FULL || hbase + 16u * i < n;
    const uint32_t dig = uint32_t(keys[i] >> shift) & (RADIX - 1);
    uint32_t* w = wp + half_slot(dig);
    if (valid) atomicOr(w, 1u << l16);
    __syncwarp();
    const uint32_t word = valid ? *w : 0u;
    const uint32_t peers = word & 0xffffu, cnt = word >> 16;
    const uint32_t below = __popc(peers & lt16);
    __syncwarp();
    if (valid && below == 0) *w = (cnt + uint32_t(__popc(peers))) << 16;
    RankPack<KPT>::set(rank2, i, cnt + below);
    __syncwarp();
  }
}

// Places the half-warp's keys at their tile positions (wp: the warp's
// per-half-warp offsets, laid out as half_slot says).
template <int D, int KPT, bool FULL, typename K>
__device__ __forceinline__ void half_place(const K (&keys)[KPT],
                                           const uint32_t (&rank2)[RankPack<KPT>::kRegs],
                                           int shift, uint32_t hbase, uint32_t n,
                                           const uint32_t* wp, K* s_keys) {
  constexpr uint32_t RADIX = 1u << D;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    if (FULL || hbase + 16u * i < n) {
      const uint32_t dig = uint32_t(keys[i] >> shift) & (RADIX - 1);
      s_keys[wp[half_slot(dig)] + RankPack<KPT>::get(rank2, i)] = keys[i];
    }
  }
}

}  // namespace rwt
