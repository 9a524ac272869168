// Stage 1 (Morton encode) and stage 2 (onesweep LSD radix sort).
//
// Stage 1 follows apps/tree/cuda/01_morton.cu:8-19 (per-point
// xyz_to_morton32); in the fused pipeline it also builds the sort's digit
// histograms for every pass while the keys are in registers, which removes the
// reference's separate k_GlobalHistogram read of the keys
// (cu_dispatcher.cu:82-170).
//
// Stage 2 replaces k_GlobalHistogram / k_Scan / 4 x k_DigitBinningPass
// (cu_dispatcher.cu:82-468,528-591) with a onesweep sort designed for 148 SMs:
// one CTA per tile (grid = number of tiles, not 16), tiles handed out by an
// atomic ticket so that every look-back waits only on tiles already running,
// per-warp stable ranking (shared-memory atomic-OR peer masks by default;
// ballot multi-split and match.any in the variant menu), the tile reordered by
// digit in shared memory, and a per-digit decoupled look-back.  Digit width is
// 8, 10 or 11 bits; 32-bit keys take 4, 3 or 3 passes, 64-bit keys 8, 7 or 6.  The
// default 32-bit variant (384 threads x 24 keys) runs three blocks per SM.
#include <algorithm>

#include "internal.hpp"
#include "morton.cuh"
#include "rank.cuh"

namespace rwt {

// ---------------------------------------------------------------------------
// stage 1
// ---------------------------------------------------------------------------

// Points are walked in tiles of kPointTile that never straddle two segments;
// each CTA takes a contiguous run of tiles, so with HIST its shared-memory
// histograms are flushed to the segment's global ones only when the segment
// changes.  ghist: [segments][passes][RADIX].
template <typename K, int D, bool HIST, bool ENCODE, bool POW2>
__global__ void __launch_bounds__(256)
    k_keys_pass(const float4* __restrict__ pts, K* __restrict__ keys, SegTable seg,
                TileMap map, uint32_t tiles_per_cta, float min_coord, float range,
                float inv_range, uint32_t* __restrict__ ghist,
                const uint32_t* __restrict__ gate) {
  pdl_enter();
  if (gate && *gate == 0) return;  // a gated sort that is not needed this run
  constexpr int RADIX = 1 << D;
  // the sort's passes: ceil(code bits / D), as the storage computes them
  constexpr int P = (KeyTraits<K>::kCodeBits + D - 1) / D;
  extern __shared__ uint32_t s_hist[];  // [P][RADIX] when HIST
  const int nh = P * RADIX;
  if (HIST) {
    for (int i = threadIdx.x; i < nh; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
  }
  const uint32_t t0 = blockIdx.x * tiles_per_cta;
  const uint32_t t1 = min(t0 + tiles_per_cta, map.n_tiles);
  uint32_t cur = 0xffffffffu;
  auto flush = [&](uint32_t c) {
    __syncthreads();
    uint32_t* g = ghist + size_t(c) * nh;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
      const uint32_t v = s_hist[i];
      if (v) atomicAdd(&g[i], v);
      s_hist[i] = 0;
    }
    __syncthreads();
  };
  for (uint32_t t = t0; t < t1; ++t) {
    uint32_t first;
    const uint32_t c = tile_segment(seg, map, t, &first);
    if (HIST && c != cur && cur != 0xffffffffu) flush(cur);
    cur = c;
    const uint32_t sb = seg_begin(seg, c);
    const uint32_t lo = sb + (t - first) * kPointTile;
    const uint32_t hi = min(lo + kPointTile, sb + seg_size(seg, c));
    auto count = [&](K k) {
      if (HIST) {
#pragma unroll
        for (int ps = 0; ps < P; ++ps)
          atomicAdd(&s_hist[ps * RADIX + int((k >> (ps * D)) & K(RADIX - 1))], 1u);
      }
    };
    if (hi - lo == kPointTile) {
      // full tile: four loads in flight per thread before any is used
      static_assert(kPointTile % (4 * 256) == 0, "whole rounds of four points per thread");
      for (uint32_t i = lo + threadIdx.x; i < hi; i += 4 * 256) {
        K k[4];
        if (ENCODE) {
          float4 p[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) p[u] = __ldcs(pts + i + 256u * u);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            k[u] = encode<K, POW2>(p[u].x, p[u].y, p[u].z, min_coord, range, inv_range);
            keys[i + 256u * u] = k[u];
          }
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) k[u] = keys[i + 256u * u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) count(k[u]);
      }
    } else {
      for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        K k;
        if (ENCODE) {
          const float4 p = __ldcs(pts + i);
          k = encode<K, POW2>(p.x, p.y, p.z, min_coord, range, inv_range);
          keys[i] = k;
        } else {
          k = keys[i];
        }
        count(k);
      }
    }
  }
  if (HIST && cur != 0xffffffffu) flush(cur);
}

// One block per (segment, pass): exclusive scan of the segment's digit
// histogram, stored as the inclusive descriptor of the virtual tile before the
// segment's first tile.  Values are absolute positions (segment start added).
// Descriptor rows of a pass: segment c's init row is toff[c] + c, its tile j
// uses row toff[c] + c + 1 + j.
// For the top pass it also sets skew[c] when the digits are skewed: the
// chance that two keys share a digit, sum over digits of (count / n)^2, above
// 2^-skew_log2 (many lanes of a warp on one digit then serialise the
// atomic-OR ranking, which the ballot ranking does not).
template <int D>
__global__ void __launch_bounds__(256)
    k_sort_init(const uint32_t* __restrict__ ghist, uint32_t* __restrict__ desc,
                SegTable seg, TileMap map, int passes, uint32_t rows_per_pass,
                const uint32_t* __restrict__ gate, uint32_t* __restrict__ skew, int skew_log2) {
  pdl_enter();
  if (gate && *gate == 0) return;
  constexpr int RADIX = 1 << D;
  constexpr int R = (RADIX + 255) / 256;
  static_assert(R * 256 >= RADIX, "every digit needs an offset");
  __shared__ uint32_t s_warp[9];
  const uint32_t c = blockIdx.x / passes;
  const int pass = int(blockIdx.x % passes);
  if (map.toff && map.toff[c + 1] == map.toff[c]) return;  // no tile in this map
  const uint32_t* h = ghist + (size_t(c) * passes + pass) * RADIX;
  const uint32_t init_row = (map.toff ? map.toff[c] : 0u) + c;
  uint32_t* row0 = desc + (size_t(pass) * rows_per_pass + init_row) * RADIX;
  uint32_t v[R];
  uint32_t local = 0;
  const int first = threadIdx.x * R;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    v[r] = first + r < RADIX ? h[first + r] : 0u;
    local += v[r];
  }
  uint32_t total;
  uint32_t run = seg_begin(seg, c) + block_exclusive_scan<256>(local, s_warp, &total);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (first + r < RADIX) row0[first + r] = kFlagInc | (run << 2);
    run += v[r];
  }
  if (skew && pass == passes - 1) {  // block-uniform
    __shared__ unsigned long long s_sq[8];
    unsigned long long sq = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) sq += (unsigned long long)v[r] * v[r];
    sq = warp_sum(sq);
    if (lane_id() == 0) s_sq[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long all = 0;
      for (int w = 0; w < 8; ++w) all += s_sq[w];
      skew[c] = (all << skew_log2) > (unsigned long long)total * total ? 1u : 0u;
    }
  }
}

// ---------------------------------------------------------------------------
// stage 2: one onesweep pass
// ---------------------------------------------------------------------------


// Descriptors a look-back reads per round trip.
constexpr int kLookback = 8;

template <typename K, int D, int THREADS, int KPT, int RANK>
struct BinCfg {
  static constexpr int RADIX = 1 << D;
  static constexpr int NW = THREADS / 32;
  static constexpr int TILE = THREADS * KPT;
  static constexpr size_t kKeysBytes = size_t(TILE) * sizeof(K);
  static constexpr size_t kHistBytes = size_t(NW) * RADIX * 4;
  // the two-array scheme keeps a match-mask array beside the counters; the
  // half-warp scheme has two words per digit and warp (one per half-warp)
  static constexpr size_t kMatchBytes =
      (RANK == kRankAtomicOr || RANK == kRankHalfPacked || RANK == kRankMixed) ? kHistBytes : 0;
  static constexpr size_t kSmem =
      kKeysBytes + kHistBytes + kMatchBytes + 3 * size_t(RADIX) * 4 + 64 * 4;
  static_assert(kSmem <= 227 * 1024, "onesweep variant exceeds shared memory per CTA");
};

// One onesweep pass over `n` keys: digit `shift`..`shift+D-1`, stable.
// desc: [(tiles + 1) x RADIX] descriptors, row 0 prefilled with the global
// exclusive digit offsets (k_sort_init), rows 1.. zero.
// PERSIST: a CTA takes tiles by ticket until they run out (a grid of at most
// one wave), instead of one tile per CTA.  Used when the pass is gated, so
// that a pass that is not needed costs one short wave of CTAs.  A CTA holds a
// ticket only while it runs, so every look-back still waits only on running
// tiles, whatever the grid.
template <typename K, int D, int THREADS, int KPT, int RANK, int MINB, bool PERSIST, int BB = D>
__global__ void __launch_bounds__(THREADS, MINB)
    k_binning(const K* __restrict__ in, K* __restrict__ out, SegTable seg, TileMap map,
              int shift, uint32_t* __restrict__ desc,
              uint32_t* __restrict__ tile_ctr, DevStatus* __restrict__ st,
              uint32_t spin_limit, const uint32_t* __restrict__ gate,
              const uint32_t* __restrict__ skew) {
  pdl_enter();
  if (gate && *gate == 0) return;  // every tile of the pass returns: no look-back waits
  using C = BinCfg<K, D, THREADS, KPT, RANK>;
  constexpr int RADIX = C::RADIX, NW = C::NW, TILE = C::TILE;
  extern __shared__ __align__(16) unsigned char smem[];
  K* s_keys = reinterpret_cast<K*>(smem);
  uint32_t* s_hist = reinterpret_cast<uint32_t*>(smem + C::kKeysBytes);
  uint32_t* s_match = s_hist + NW * RADIX;  // only with kRankAtomicOr / kRankMixed
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + C::kKeysBytes + C::kHistBytes +
                                                C::kMatchBytes);
  uint32_t* s_start = s_cnt + RADIX;
  uint32_t* s_gofs = s_start + RADIX;
  uint32_t* s_misc = s_gofs + RADIX;  // [0] tile, [1..] warp scan scratch

  const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  for (;;) {
    if (tid == 0) s_misc[0] = atomicAdd(tile_ctr, 1u);
    {
      static_assert((NW * RADIX) % 4 == 0 && C::kKeysBytes % 16 == 0, "16-byte zeroing");
      const uint4 z = make_uint4(0, 0, 0, 0);
      constexpr int kWords =
          (RANK == kRankAtomicOr || RANK == kRankHalfPacked || RANK == kRankMixed ? 2 : 1) *
          NW * RADIX;
      for (int i = tid; i < kWords / 4; i += THREADS) reinterpret_cast<uint4*>(s_hist)[i] = z;
    }
    __syncthreads();
    const uint32_t tile = s_misc[0];
    if (PERSIST && tile >= map.n_tiles) break;  // block-uniform
    uint32_t first_tile;
    const uint32_t segc = tile_segment(seg, map, tile, &first_tile);
    const uint32_t base = seg_begin(seg, segc) + (tile - first_tile) * TILE;
    const uint32_t n = seg_begin(seg, segc) + seg_size(seg, segc);  // end of the segment
    const int row = int(tile + segc + 1);       // this tile's descriptor row
    const int init_row = int(first_tile + segc);  // the segment's inclusive row
    const bool full = base + TILE <= n;

    // load: warp w owns [w*32*KPT, (w+1)*32*KPT) of the tile, 32 keys per step
    // (half-warp scheme: half h of warp w owns [w*32*KPT + h*16*KPT, +16*KPT),
    // 16 keys per step)
    K keys[KPT];
    uint32_t rank2[RankPack<KPT>::kRegs];  // packed warp ranks
    const uint32_t wbase = base + warp * 32u * KPT + lane;
    const uint32_t hbase = base + warp * 32u * KPT + (lane >> 4) * 16u * KPT + (lane & 15u);
    uint32_t* wh = s_hist + warp * RADIX;
    uint32_t* wm = s_match + warp * RADIX;
    uint32_t* wp = s_hist + warp * 2u * RADIX;  // half-warp scheme: [2 RADIX] per warp
    if (RANK == kRankHalfPacked) {
      if (full) {
  #pragma unroll
        for (int i = 0; i < KPT; ++i) keys[i] = in[hbase + 16u * i];
        half_rank<D, KPT, true>(keys, rank2, shift, hbase, n, wp);
      } else {
  #pragma unroll
        for (int i = 0; i < KPT; ++i) {
          const uint32_t idx = hbase + 16u * i;
          keys[i] = idx < n ? in[idx] : K(0);
        }
        half_rank<D, KPT, false>(keys, rank2, shift, hbase, n, wp);
      }
    } else if (RANK == kRankMixed) {
      // this segment's digits decide the scheme (block-uniform)
      const bool ballots = skew != nullptr && skew[segc] != 0u;
      if (full) {
  #pragma unroll
        for (int i = 0; i < KPT; ++i) keys[i] = in[wbase + 32u * i];
        warp_rank<D, KPT, kRankMixed, true, BB>(keys, rank2, shift, wbase, n, wh, wm, KPT, ballots);
      } else {
  #pragma unroll
        for (int i = 0; i < KPT; ++i) {
          const uint32_t idx = wbase + 32u * i;
          keys[i] = idx < n ? in[idx] : K(0);
        }
        warp_rank<D, KPT, kRankMixed, false, BB>(keys, rank2, shift, wbase, n, wh, wm, KPT,
                                                 ballots);
      }
    } else if (full) {
  #pragma unroll
      for (int i = 0; i < KPT; ++i) keys[i] = in[wbase + 32u * i];
      warp_rank<D, KPT, RANK, true, BB>(keys, rank2, shift, wbase, n, wh, wm);
    } else {
  #pragma unroll
      for (int i = 0; i < KPT; ++i) {
        const uint32_t idx = wbase + 32u * i;
        keys[i] = idx < n ? in[idx] : K(0);
      }
      warp_rank<D, KPT, RANK, false, BB>(keys, rank2, shift, wbase, n, wh, wm);
    }
    __syncthreads();

    // per digit: exclusive scan over warps (half-warps) and publish the tile
    // aggregate
    uint32_t* drow = desc + size_t(row) * RADIX;
    if (RANK == kRankHalfPacked) {
      // lane pairs own a digit: the even lane its half-warp-0 words, the odd
      // lane its half-warp-1 words (consecutive addresses, no bank conflicts);
      // units run in the order (warp, half), the partner's count by a shuffle
      static_assert((2 * RADIX) % 32 == 0 && THREADS % 32 == 0, "whole warps per pass");
      for (int x = tid; x < 2 * RADIX; x += THREADS) {
        const uint32_t h = uint32_t(x) & 1u;
        uint32_t run = 0;
  #pragma unroll
        for (int w = 0; w < NW; ++w) {
          uint32_t* p = s_hist + w * 2 * RADIX + x;
          const uint32_t mine = *p >> 16;
          const uint32_t other = __shfl_xor_sync(0xffffffffu, mine, 1);
          *p = run + (h ? other : 0u);
          run += mine + other;
        }
        if (!h) {
          s_cnt[x >> 1] = run;
          st_relaxed(drow + (x >> 1), kFlagAgg | (run << 2));
        }
      }
    } else {
      for (int d = tid; d < RADIX; d += THREADS) {
        uint32_t run = 0;
  #pragma unroll
        for (int w = 0; w < NW; ++w) {
          const uint32_t c = s_hist[w * RADIX + d];
          s_hist[w * RADIX + d] = run;
          run += c;
        }
        s_cnt[d] = run;
        st_relaxed(drow + d, kFlagAgg | (run << 2));
      }
    }
    __syncthreads();
    digit_exclusive_scan<D, THREADS>(s_cnt, s_start, s_misc + 1);
    __syncthreads();
    // fold the digit starts into the per-warp offsets once per tile, so that
    // placing a key below reads one shared-memory word instead of two
    if (RANK == kRankHalfPacked) {
      for (int i = tid; i < 2 * NW * RADIX; i += THREADS)
        s_hist[i] += s_start[(i >> 1) & (RADIX - 1)];
    } else {
      for (int i = tid; i < NW * RADIX; i += THREADS) s_hist[i] += s_start[i & (RADIX - 1)];
    }
    __syncthreads();

    // reorder the tile by digit in shared memory first: it needs only the
    // tile's own counts, and gives the predecessors time to publish their
    // inclusive prefixes before the look-back below reads them
    if (RANK == kRankHalfPacked) {
      if (full) half_place<D, KPT, true>(keys, rank2, shift, hbase, n, wp, s_keys);
      else half_place<D, KPT, false>(keys, rank2, shift, hbase, n, wp, s_keys);
    } else if (full) {
      warp_place<D, KPT, true>(keys, rank2, shift, wbase, n, wh, s_keys);
    } else {
      warp_place<D, KPT, false>(keys, rank2, shift, wbase, n, wh, s_keys);
    }

    // decoupled look-back, kLookback descriptors per round trip.  The segment's
    // first row is always inclusive, so rows are read clamped to it and the
    // walk stops there at the latest.
    for (int d = tid; d < RADIX; d += THREADS) {
      uint32_t excl = 0;
      int k = row - 1;
      uint32_t spin = 0;
      while (true) {
        uint32_t v[kLookback];
  #pragma unroll
        for (int q = 0; q < kLookback; ++q)
          v[q] = ld_relaxed(desc + size_t(max(k - q, init_row)) * RADIX + d);
        int used = 0;
        bool done = false;
  #pragma unroll
        for (int q = 0; q < kLookback; ++q) {
          const uint32_t f = v[q] & kFlagMask;
          if (done || f == 0 || used != q) break;
          excl += v[q] >> 2;
          ++used;
          done = f == kFlagInc;
        }
        if (done) break;
        if (used) {
          k -= used;
          spin = 0;
          continue;
        }
        if (++spin > spin_limit || device_failed(st)) {
          report_error(st, RW_ERR_TIMEOUT, kSiteSort);
          break;
        }
        backoff(spin);
      }
      st_relaxed(drow + d, kFlagInc | ((excl + s_cnt[d]) << 2));
      s_gofs[d] = excl - s_start[d];
    }
    __syncthreads();

    // write runs of equal digits to their global positions (a destination is
    // out of range only if a look-back gave up)
    const uint32_t total = seg.total;
    if (full) {
  #pragma unroll 4
      for (int i = 0; i < KPT; ++i) {
        const uint32_t p = tid + uint32_t(i) * THREADS;
        const K k = s_keys[p];
        const uint32_t dst = s_gofs[uint32_t(k >> shift) & (RADIX - 1)] + p;
        if (dst < total) out[dst] = k;
      }
    } else {
      const uint32_t tile_n = n - base;
      for (uint32_t p = tid; p < tile_n; p += THREADS) {
        const K k = s_keys[p];
        const uint32_t dst = s_gofs[uint32_t(k >> shift) & (RADIX - 1)] + p;
        if (dst < total) out[dst] = k;
      }
    }
    if (!PERSIST) break;
    __syncthreads();  // the next tile reuses every shared array
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

namespace {

template <typename K, int D>
cudaError_t keys_t(const Bufs& b, const Scratch& sc, const Plan& pl, bool encode,
                   bool hist, cudaStream_t s) {
  const uint32_t tiles = pl.point_map.n_tiles;
  if (tiles == 0) return cudaSuccess;
  const uint32_t ctas = std::max(1u, std::min<uint32_t>(tiles, uint32_t(sc.num_sms) * 8));
  const uint32_t per = div_up(tiles, ctas);
  const uint32_t grid = div_up(tiles, per);
  if (hist && sc.passes != (KeyTraits<K>::kCodeBits + D - 1) / D) return cudaErrorInvalidValue;
  const size_t smem = hist ? size_t(sc.passes) * (1u << D) * 4 : 0;
  K* keys = static_cast<K*>(b.keys);
  const float inv = pow2_reciprocal(b.range);
#define RWT_KEYS_LAUNCH(H, E)                                                        \
  do {                                                                               \
    auto kern = inv != 0.0f ? k_keys_pass<K, D, H, E, true> : k_keys_pass<K, D, H, E, false>; \
    if (smem > 48 * 1024)                                                            \
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)); \
    launch_pdl(kern, grid, 256, smem, s, b.points, keys, pl.seg, pl.point_map, per, b.min_coord, \
                                 b.range, inv, sc.ghist, sc.gate);                   \
  } while (0)
  if (encode && hist) RWT_KEYS_LAUNCH(true, true);
  else if (encode) RWT_KEYS_LAUNCH(false, true);
  else RWT_KEYS_LAUNCH(true, false);
#undef RWT_KEYS_LAUNCH
  return cudaGetLastError();
}

// probe_spins != 0: the bounded-wait test hook (launch_sort_lookback_probe).
// RANK kRankMixed: atomic-OR ranking for the passes over full digits; the
// top pass ranks a segment by ballots over the code's remaining bits when
// k_sort_init found its top digits skewed (sum of squared digit frequencies
// above 1/32 for 32-bit keys, 1/64 for 64-bit keys, where the two schemes
// measured even), else by atomic OR.
template <typename K, int D, int THREADS, int KPT, int RANK, int MINB>
cudaError_t passes_t(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s,
                     cudaEvent_t* marks, uint32_t probe_spins) {
  constexpr int P = (KeyTraits<K>::kCodeBits + D - 1) / D;
  constexpr int RB = RANK == kRankMixed ? kRankAtomicOr : RANK;  // passes 0 .. P-2
  constexpr int RT = RANK;                                       // pass P-1
  constexpr int TB = RANK == kRankMixed ? KeyTraits<K>::kCodeBits - (P - 1) * D : D;
  constexpr int kSkewLog2 = sizeof(K) == 4 ? 5 : 6;
  uint32_t* skew = RANK == kRankMixed ? sc.skew : nullptr;
  using C = BinCfg<K, D, THREADS, KPT, RB>;
  using CT = BinCfg<K, D, THREADS, KPT, RT>;
  // a gated sort (a fallback that may not be needed) runs persistent passes
  const bool persist = sc.gate != nullptr && !probe_spins;
  auto kern = persist ? k_binning<K, D, THREADS, KPT, RB, MINB, true>
                      : k_binning<K, D, THREADS, KPT, RB, MINB, false>;
  auto kern_top = persist ? k_binning<K, D, THREADS, KPT, RT, MINB, true, TB>
                          : k_binning<K, D, THREADS, KPT, RT, MINB, false, TB>;
  const uint32_t tiles = pl.sort_map.n_tiles;
  if (tiles + pl.seg.count > sc.sort_rows || sc.passes != P) return cudaErrorInvalidValue;
  launch_pdl(k_sort_init<D>, pl.seg.count * sc.passes, 256, 0, s, sc.ghist, sc.sort_desc, pl.seg,
             pl.sort_map, sc.passes, sc.sort_rows, sc.gate, skew, kSkewLog2);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (marks) cudaEventRecord(marks[0], s);
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(C::kSmem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kern_top, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(CT::kSmem));
  if (e != cudaSuccess) return e;
  K* keys = static_cast<K*>(b.keys);
  K* alt = static_cast<K*>(b.alt);
  K* tmp = static_cast<K*>(b.tmp);
  if (probe_spins) {
    // pass 0 with the tile ticket starting at 1: tile 0 never runs, so its
    // descriptor row stays unpublished and every other tile's look-back runs
    // into its spin limit; tiles 1 .. tiles-1 are launched (all in range)
    if (tiles < 2 || pl.seg.count != 1) return cudaErrorInvalidValue;
    e = cudaMemsetAsync(sc.tile_ctr + kCtrSortBase, 0x01, 1, s);
    if (e != cudaSuccess) return e;
    launch_pdl(kern, tiles - 1, THREADS, C::kSmem, s, static_cast<const K*>(keys), alt, pl.seg,
               pl.sort_map, 0, sc.sort_desc, sc.tile_ctr + kCtrSortBase, sc.status,
               probe_spins, static_cast<const uint32_t*>(nullptr),
               static_cast<const uint32_t*>(nullptr));
    return cudaGetLastError();
  }
  const K* src = keys;
  const uint32_t grid =
      persist ? std::min<uint32_t>(tiles, uint32_t(sc.num_sms) * uint32_t(MINB)) : tiles;
  for (int p = 0; p < P; ++p) {
    K* dst = ((P - 1 - p) % 2 == 0) ? alt : tmp;
    if (tiles)
      launch_pdl(p == P - 1 ? kern_top : kern, grid, THREADS, p == P - 1 ? CT::kSmem : C::kSmem,
                 s, src, dst, pl.seg, pl.sort_map, p * D,
                 sc.sort_desc + size_t(p) * sc.sort_rows * C::RADIX,
                 sc.tile_ctr + kCtrSortBase + p, sc.status, sc.spin_limit, sc.gate,
                 static_cast<const uint32_t*>(p == P - 1 ? skew : nullptr));
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (marks) cudaEventRecord(marks[1 + p], s);
    src = dst;
  }
  return cudaSuccess;
}

using PassFn = cudaError_t (*)(const Bufs&, const Scratch&, const Plan&, cudaStream_t,
                               cudaEvent_t*, uint32_t);

struct SortVariant {
  int key_bits, radix_bits, threads, kpt, rank;
  PassFn fn;
};

// The menu the autotuner chooses from (entry 0 of each key/digit width is
// the default).
const SortVariant kVariants[] = {
    {32, 8, 384, 24, kRankAtomicOr, passes_t<uint32_t, 8, 384, 24, kRankAtomicOr, 3>},
    {32, 8, 384, 24, kRankMixed, passes_t<uint32_t, 8, 384, 24, kRankMixed, 3>},
    {32, 8, 384, 24, kRankHalfPacked, passes_t<uint32_t, 8, 384, 24, kRankHalfPacked, 3>},
    {32, 8, 512, 16, kRankHalfPacked, passes_t<uint32_t, 8, 512, 16, kRankHalfPacked, 2>},
    {32, 8, 256, 24, kRankHalfPacked, passes_t<uint32_t, 8, 256, 24, kRankHalfPacked, 4>},
    {32, 8, 512, 24, kRankHalfPacked, passes_t<uint32_t, 8, 512, 24, kRankHalfPacked, 2>},
    {32, 8, 512, 16, kRankAtomicOr, passes_t<uint32_t, 8, 512, 16, kRankAtomicOr, 2>},
    {32, 8, 384, 16, kRankAtomicOr, passes_t<uint32_t, 8, 384, 16, kRankAtomicOr, 2>},
    {32, 8, 256, 16, kRankAtomicOr, passes_t<uint32_t, 8, 256, 16, kRankAtomicOr, 3>},
    {32, 8, 256, 24, kRankAtomicOr, passes_t<uint32_t, 8, 256, 24, kRankAtomicOr, 2>},
    {32, 8, 512, 24, kRankAtomicOr, passes_t<uint32_t, 8, 512, 24, kRankAtomicOr, 1>},
    {32, 8, 256, 16, kRankBallot, passes_t<uint32_t, 8, 256, 16, kRankBallot, 3>},
    {32, 8, 512, 16, kRankBallot, passes_t<uint32_t, 8, 512, 16, kRankBallot, 1>},
    {32, 8, 384, 16, kRankMatchAny, passes_t<uint32_t, 8, 384, 16, kRankMatchAny, 2>},
    {32, 8, 512, 16, kRankBallot, passes_t<uint32_t, 8, 512, 16, kRankBallot, 2>},
    {32, 8, 384, 16, kRankBallot, passes_t<uint32_t, 8, 384, 16, kRankBallot, 2>},
    {32, 8, 256, 32, kRankBallot, passes_t<uint32_t, 8, 256, 32, kRankBallot, 2>},
    {32, 8, 512, 16, kRankMatchAny, passes_t<uint32_t, 8, 512, 16, kRankMatchAny, 2>},
    {32, 8, 1024, 16, kRankAtomicOr, passes_t<uint32_t, 8, 1024, 16, kRankAtomicOr, 1>},
    {32, 8, 1024, 8, kRankAtomicOr, passes_t<uint32_t, 8, 1024, 8, kRankAtomicOr, 1>},
    {32, 10, 256, 24, kRankAtomicOr, passes_t<uint32_t, 10, 256, 24, kRankAtomicOr, 2>},
    {32, 10, 256, 16, kRankAtomicOr, passes_t<uint32_t, 10, 256, 16, kRankAtomicOr, 2>},
    {32, 10, 256, 24, kRankBallot, passes_t<uint32_t, 10, 256, 24, kRankBallot, 3>},
    {32, 10, 384, 16, kRankBallot, passes_t<uint32_t, 10, 384, 16, kRankBallot, 2>},
    {32, 10, 512, 16, kRankBallot, passes_t<uint32_t, 10, 512, 16, kRankBallot, 2>},
    {32, 10, 256, 24, kRankMatchAny, passes_t<uint32_t, 10, 256, 24, kRankMatchAny, 3>},
    {32, 10, 256, 24, kRankHalfPacked, passes_t<uint32_t, 10, 256, 24, kRankHalfPacked, 2>},
    {32, 11, 512, 16, kRankBallot, passes_t<uint32_t, 11, 512, 16, kRankBallot, 1>},
    {32, 11, 256, 16, kRankAtomicOr, passes_t<uint32_t, 11, 256, 16, kRankAtomicOr, 1>},
    {32, 11, 256, 24, kRankAtomicOr, passes_t<uint32_t, 11, 256, 24, kRankAtomicOr, 1>},
    {32, 11, 256, 24, kRankBallot, passes_t<uint32_t, 11, 256, 24, kRankBallot, 1>},
    {32, 11, 256, 16, kRankBallot, passes_t<uint32_t, 11, 256, 16, kRankBallot, 2>},
    {32, 11, 384, 16, kRankBallot, passes_t<uint32_t, 11, 384, 16, kRankBallot, 1>},
    {64, 8, 384, 16, kRankAtomicOr, passes_t<uint64_t, 8, 384, 16, kRankAtomicOr, 2>},
    {64, 8, 384, 16, kRankMixed, passes_t<uint64_t, 8, 384, 16, kRankMixed, 2>},
    {64, 8, 384, 16, kRankHalfPacked, passes_t<uint64_t, 8, 384, 16, kRankHalfPacked, 2>},
    {64, 8, 256, 16, kRankHalfPacked, passes_t<uint64_t, 8, 256, 16, kRankHalfPacked, 3>},
    {64, 8, 256, 16, kRankAtomicOr, passes_t<uint64_t, 8, 256, 16, kRankAtomicOr, 2>},
    {64, 8, 256, 12, kRankAtomicOr, passes_t<uint64_t, 8, 256, 12, kRankAtomicOr, 3>},
    {64, 8, 256, 16, kRankBallot, passes_t<uint64_t, 8, 256, 16, kRankBallot, 2>},
    {64, 10, 256, 16, kRankAtomicOr, passes_t<uint64_t, 10, 256, 16, kRankAtomicOr, 2>},
    {64, 10, 256, 16, kRankBallot, passes_t<uint64_t, 10, 256, 16, kRankBallot, 2>},
    {64, 11, 384, 16, kRankBallot, passes_t<uint64_t, 11, 384, 16, kRankBallot, 1>},
    {64, 11, 256, 16, kRankAtomicOr, passes_t<uint64_t, 11, 256, 16, kRankAtomicOr, 1>},
    {64, 11, 256, 12, kRankAtomicOr, passes_t<uint64_t, 11, 256, 12, kRankAtomicOr, 1>},
    {64, 11, 256, 16, kRankBallot, passes_t<uint64_t, 11, 256, 16, kRankBallot, 1>},
};
constexpr int kNumVariants = int(sizeof(kVariants) / sizeof(kVariants[0]));

}  // namespace

// Smallest tile of any variant for this key/digit width: sizes the descriptors.
uint32_t sort_tile_for(int key_bits, int radix_bits) {
  uint32_t t = 0xffffffffu;
  for (const auto& v : kVariants)
    if (v.key_bits == key_bits && v.radix_bits == radix_bits)
      t = std::min<uint32_t>(t, uint32_t(v.threads * v.kpt));
  return t;
}

uint32_t sort_variant_tile(int idx) {
  if (idx < 0 || idx >= kNumVariants) return 0;
  return uint32_t(kVariants[idx].threads * kVariants[idx].kpt);
}

int sort_variant_count() { return kNumVariants; }

int sort_variant_info(int idx, int* key_bits, int* radix_bits, int* threads, int* kpt,
                      int* rank) {
  if (idx < 0 || idx >= kNumVariants) return -1;
  const auto& v = kVariants[idx];
  *key_bits = v.key_bits;
  *radix_bits = v.radix_bits;
  *threads = v.threads;
  *kpt = v.kpt;
  *rank = v.rank;
  return 0;
}

int default_sort_variant(int key_bits, int radix_bits) {
  for (int i = 0; i < kNumVariants; ++i)
    if (kVariants[i].key_bits == key_bits && kVariants[i].radix_bits == radix_bits) return i;
  return -1;
}

cudaError_t launch_keys(const Bufs& b, const Scratch& sc, const Plan& pl, bool encode,
                        bool hist, cudaStream_t s) {
  if (b.key_bits == 32) {
    if (sc.radix_bits == 8) return keys_t<uint32_t, 8>(b, sc, pl, encode, hist, s);
    if (sc.radix_bits == 10) return keys_t<uint32_t, 10>(b, sc, pl, encode, hist, s);
    return keys_t<uint32_t, 11>(b, sc, pl, encode, hist, s);
  }
  if (sc.radix_bits == 8) return keys_t<uint64_t, 8>(b, sc, pl, encode, hist, s);
  if (sc.radix_bits == 10) return keys_t<uint64_t, 10>(b, sc, pl, encode, hist, s);
  return keys_t<uint64_t, 11>(b, sc, pl, encode, hist, s);
}

cudaError_t launch_sort_passes(const Bufs& b, const Scratch& sc, const Plan& pl,
                               cudaStream_t s, cudaEvent_t* marks) {
  const int v = sc.sort_variant;
  if (v < 0 || v >= kNumVariants || kVariants[v].key_bits != b.key_bits ||
      kVariants[v].radix_bits != sc.radix_bits)
    return cudaErrorInvalidValue;
  return kVariants[v].fn(b, sc, pl, s, marks, 0u);
}

cudaError_t launch_sort_lookback_probe(const Bufs& b, const Scratch& sc, const Plan& pl,
                                       uint32_t spin_limit, cudaStream_t s) {
  const int v = sc.sort_variant;
  if (v < 0 || v >= kNumVariants || kVariants[v].key_bits != b.key_bits ||
      kVariants[v].radix_bits != sc.radix_bits || spin_limit == 0)
    return cudaErrorInvalidValue;
  cudaError_t e = launch_keys(b, sc, pl, false, true, s);
  if (e != cudaSuccess) return e;
  return kVariants[v].fn(b, sc, pl, s, nullptr, spin_limit);
}

}  // namespace rwt
