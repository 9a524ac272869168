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
// per-warp stable ranking (ballot multi-split), the tile reordered by digit in
// shared memory, and a per-digit decoupled look-back.  Digit width is 8 or 11
// bits; 32-bit keys take 4 or 3 passes, 64-bit keys 8 or 6.
#include <algorithm>

#include "internal.hpp"
#include "morton.cuh"

namespace rwt {

// ---------------------------------------------------------------------------
// stage 1
// ---------------------------------------------------------------------------

template <typename K, int D, bool HIST>
__global__ void __launch_bounds__(256)
    k_morton(const float4* __restrict__ pts, K* __restrict__ keys, uint32_t n,
             float min_coord, float range, uint32_t* __restrict__ ghist,
             int passes) {
  constexpr int RADIX = 1 << D;
  extern __shared__ uint32_t s_hist[];  // [passes][RADIX] when HIST
  if (HIST) {
    for (int i = threadIdx.x; i < passes * RADIX; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
  }
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float4 p = __ldcs(pts + i);
    const K k = encode<K>(p.x, p.y, p.z, min_coord, range);
    keys[i] = k;
    if (HIST) {
      for (int ps = 0; ps < passes; ++ps)
        atomicAdd(&s_hist[ps * RADIX + int((k >> (ps * D)) & K(RADIX - 1))], 1u);
    }
  }
  if (HIST) {
    __syncthreads();
    for (int i = threadIdx.x; i < passes * RADIX; i += blockDim.x) {
      const uint32_t c = s_hist[i];
      if (c) atomicAdd(&ghist[i], c);
    }
  }
}

// Digit histograms of all passes from keys already in memory (stage 2 called
// on its own).
template <typename K, int D>
__global__ void __launch_bounds__(256)
    k_histogram(const K* __restrict__ keys, uint32_t n,
                uint32_t* __restrict__ ghist, int passes) {
  constexpr int RADIX = 1 << D;
  extern __shared__ uint32_t s_hist[];
  for (int i = threadIdx.x; i < passes * RADIX; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const K k = keys[i];
    for (int ps = 0; ps < passes; ++ps)
      atomicAdd(&s_hist[ps * RADIX + int((k >> (ps * D)) & K(RADIX - 1))], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * RADIX; i += blockDim.x) {
    const uint32_t c = s_hist[i];
    if (c) atomicAdd(&ghist[i], c);
  }
}

// One block per pass: exclusive scan of the pass's digit histogram, stored as
// the inclusive descriptor of the virtual tile before tile 0.
template <int D>
__global__ void __launch_bounds__(256)
    k_sort_init(const uint32_t* __restrict__ ghist, uint32_t* __restrict__ desc,
                uint32_t tiles_plus_one) {
  constexpr int RADIX = 1 << D;
  constexpr int R = (RADIX + 255) / 256;
  static_assert(R * 256 >= RADIX, "every digit needs an offset");
  __shared__ uint32_t s_warp[9];
  const int pass = blockIdx.x;
  const uint32_t* h = ghist + pass * RADIX;
  uint32_t* row0 = desc + size_t(pass) * tiles_plus_one * RADIX;
  uint32_t v[R];
  uint32_t local = 0;
  const int first = threadIdx.x * R;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    v[r] = first + r < RADIX ? h[first + r] : 0u;
    local += v[r];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan<256>(local, s_warp, &total);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (first + r < RADIX) row0[first + r] = kFlagInc | (run << 2);
    run += v[r];
  }
}

// ---------------------------------------------------------------------------
// stage 2: one onesweep pass
// ---------------------------------------------------------------------------

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
enum RankMode : int { kRankBallot = 0, kRankMatchAny = 1, kRankAtomicOr = 2 };

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

template <typename K, int D, int THREADS, int KPT, int RANK>
struct BinCfg {
  static constexpr int RADIX = 1 << D;
  static constexpr int NW = THREADS / 32;
  static constexpr int TILE = THREADS * KPT;
  static constexpr size_t kKeysBytes = size_t(TILE) * sizeof(K);
  static constexpr size_t kHistBytes = size_t(NW) * RADIX * 4;
  static constexpr size_t kMatchBytes = RANK == kRankAtomicOr ? kHistBytes : 0;
  static constexpr size_t kSmem =
      kKeysBytes + kHistBytes + kMatchBytes + 3 * size_t(RADIX) * 4 + 64 * 4;
  static_assert(kSmem <= 227 * 1024, "onesweep variant exceeds shared memory per CTA");
};

// One onesweep pass over `n` keys: digit `shift`..`shift+D-1`, stable.
// desc: [(tiles + 1) x RADIX] descriptors, row 0 prefilled with the global
// exclusive digit offsets (k_sort_init), rows 1.. zero.
template <typename K, int D, int THREADS, int KPT, int RANK, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_binning(const K* __restrict__ in, K* __restrict__ out, uint32_t n,
              int shift, uint32_t* __restrict__ desc,
              uint32_t* __restrict__ tile_ctr, DevStatus* __restrict__ st) {
  using C = BinCfg<K, D, THREADS, KPT, RANK>;
  constexpr int RADIX = C::RADIX, NW = C::NW, TILE = C::TILE;
  extern __shared__ __align__(16) unsigned char smem[];
  K* s_keys = reinterpret_cast<K*>(smem);
  uint32_t* s_hist = reinterpret_cast<uint32_t*>(smem + C::kKeysBytes);
  uint32_t* s_match = s_hist + NW * RADIX;  // only with kRankAtomicOr
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + C::kKeysBytes + C::kHistBytes +
                                                C::kMatchBytes);
  uint32_t* s_start = s_cnt + RADIX;
  uint32_t* s_gofs = s_start + RADIX;
  uint32_t* s_misc = s_gofs + RADIX;  // [0] tile, [1..] warp scan scratch

  const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  if (tid == 0) s_misc[0] = atomicAdd(tile_ctr, 1u);
  for (int i = tid; i < NW * RADIX; i += THREADS) {
    s_hist[i] = 0;
    if (RANK == kRankAtomicOr) s_match[i] = 0;
  }
  __syncthreads();
  const uint32_t tile = s_misc[0];
  const uint32_t base = tile * TILE;

  // load: warp w owns [w*32*KPT, (w+1)*32*KPT) of the tile, 32 keys per step
  K keys[KPT];
  uint32_t rank[KPT];
  const uint32_t wbase = base + warp * 32u * KPT + lane;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t idx = wbase + 32u * i;
    keys[i] = idx < n ? in[idx] : K(0);
  }

  // per-warp stable ranks (key order inside the warp = step, then lane)
  uint32_t* wh = s_hist + warp * RADIX;
  uint32_t* wm = s_match + warp * RADIX;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t idx = wbase + 32u * i;
    const bool valid = idx < n;
    const uint32_t dig = uint32_t(keys[i] >> shift) & (RADIX - 1);
    uint32_t peers;
    if (RANK == kRankBallot) {
      peers = match_ballot<D>(dig, __ballot_sync(0xffffffffu, valid));
    } else if (RANK == kRankMatchAny) {
      peers = __match_any_sync(0xffffffffu, valid ? dig : 0xffffffffu);
      if (!valid) peers = 0;
    } else {
      if (valid) atomicOr(&wm[dig], 1u << lane);
      __syncwarp();
      peers = valid ? wm[dig] : 0u;
    }
    const uint32_t below = __popc(peers & lanemask_lt());
    uint32_t prev = 0;
    if (RANK == kRankAtomicOr) __syncwarp();
    if (valid && below == 0) {
      prev = wh[dig];
      wh[dig] = prev + __popc(peers);
      if (RANK == kRankAtomicOr) wm[dig] = 0;
    }
    const int leader = valid ? __ffs(peers) - 1 : int(lane);
    prev = __shfl_sync(0xffffffffu, prev, leader);
    rank[i] = prev + below;
    __syncwarp();
  }
  __syncthreads();

  // per digit: exclusive scan over warps, publish the tile aggregate, then
  // look back at once so the inclusive prefix is out as early as possible
  uint32_t* drow = desc + size_t(tile + 1) * RADIX;
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
  for (int d = tid; d < RADIX; d += THREADS) {
    // walk back 4 descriptors per round trip; row 0 is always inclusive
    uint32_t excl = 0;
    int64_t k = tile;  // row k holds tile k-1's descriptor (row 0: global)
    uint32_t spin = 0;
    while (true) {
      uint32_t v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        v[q] = k - q >= 0 ? ld_relaxed(desc + size_t(k - q) * RADIX + d) : kFlagInc;
      bool done = false;
      int used = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (done || used != q) break;
        const uint32_t f = v[q] & kFlagMask;
        if (f == kFlagInc) {
          excl += v[q] >> 2;
          done = true;
        } else if (f == kFlagAgg) {
          excl += v[q] >> 2;
          ++used;
        }
      }
      if (done) break;
      k -= used;
      if (used) {
        spin = 0;
        continue;
      }
      if (++spin > kSpinLimit || device_failed(st)) {
        report_error(st, RW_ERR_TIMEOUT, kSiteSort);
        break;
      }
      backoff(spin);
    }
    st_relaxed(drow + d, kFlagInc | ((excl + s_cnt[d]) << 2));
    s_gofs[d] = excl;
  }
  __syncthreads();
  digit_exclusive_scan<D, THREADS>(s_cnt, s_start, s_misc + 1);
  __syncthreads();

  // reorder the tile by digit in shared memory
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t idx = wbase + 32u * i;
    if (idx < n) {
      const uint32_t dig = uint32_t(keys[i] >> shift) & (RADIX - 1);
      s_keys[s_start[dig] + wh[dig] + rank[i]] = keys[i];
    }
  }
  for (int d = tid; d < RADIX; d += THREADS) s_gofs[d] -= s_start[d];
  __syncthreads();

  // write runs of equal digits to their global positions
  const uint32_t tile_n = min(uint32_t(TILE), n - base);
  for (uint32_t p = tid; p < tile_n; p += THREADS) {
    const K k = s_keys[p];
    const uint32_t dig = uint32_t(k >> shift) & (RADIX - 1);
    const uint32_t dst = s_gofs[dig] + p;
    if (dst < n) out[dst] = k;  // always true unless a look-back gave up
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

namespace {

template <typename K, int D>
cudaError_t morton_t(const rw_tree_app_data& app, rw_tree_im_storage* im,
                     bool hist, cudaStream_t s) {
  const uint32_t n = app.n_input;
  const int blocks = std::max(1, std::min<int>(div_up(n, 256), im->num_sms * 8));
  const float4* pts = reinterpret_cast<const float4*>(app.u_input_points);
  K* keys = static_cast<K*>(app.u_morton_keys);
  if (hist) {
    const size_t smem = size_t(im->passes) * (1u << D) * 4;
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_morton<K, D, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    k_morton<K, D, true><<<blocks, 256, smem, s>>>(
        pts, keys, n, app.min_coord, app.range, im->d_ghist, im->passes);
  } else {
    k_morton<K, D, false><<<blocks, 256, 0, s>>>(pts, keys, n, app.min_coord,
                                                 app.range, nullptr, 0);
  }
  return cudaGetLastError();
}

template <typename K, int D>
cudaError_t histogram_t(const rw_tree_app_data& app, rw_tree_im_storage* im,
                        cudaStream_t s) {
  const uint32_t n = app.n_input;
  const int blocks = std::max(1, std::min<int>(div_up(n, 256), im->num_sms * 8));
  const size_t smem = size_t(im->passes) * (1u << D) * 4;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_histogram<K, D>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  k_histogram<K, D><<<blocks, 256, smem, s>>>(
      static_cast<const K*>(app.u_morton_keys), n, im->d_ghist, im->passes);
  return cudaGetLastError();
}

template <typename K, int D, int THREADS, int KPT, int RANK, int MINB>
cudaError_t passes_t(const rw_tree_app_data& app, rw_tree_im_storage* im,
                     cudaStream_t s, cudaEvent_t* marks) {
  using C = BinCfg<K, D, THREADS, KPT, RANK>;
  auto kern = k_binning<K, D, THREADS, KPT, RANK, MINB>;
  const uint32_t n = app.n_input;
  const uint32_t tiles = div_up(n, C::TILE);
  const uint32_t rows = im->sort_tiles + 1;
  if (tiles > im->sort_tiles) return cudaErrorInvalidValue;
  k_sort_init<D><<<im->passes, 256, 0, s>>>(im->d_ghist, im->d_sort_desc, rows);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (marks) cudaEventRecord(marks[0], s);
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(C::kSmem));
  if (e != cudaSuccess) return e;
  K* keys = static_cast<K*>(app.u_morton_keys);
  K* alt = static_cast<K*>(app.u_morton_keys_alt);
  K* tmp = static_cast<K*>(im->d_tmp_keys);
  const K* src = keys;
  for (int p = 0; p < im->passes; ++p) {
    K* dst = ((im->passes - 1 - p) % 2 == 0) ? alt : tmp;
    kern<<<tiles, THREADS, C::kSmem, s>>>(
        src, dst, n, p * D, im->d_sort_desc + size_t(p) * rows * C::RADIX,
        im->d_tile_ctr + kCtrSortBase + p, im->d_status);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (marks) cudaEventRecord(marks[1 + p], s);
    src = dst;
  }
  return cudaSuccess;
}

using PassFn = cudaError_t (*)(const rw_tree_app_data&, rw_tree_im_storage*, cudaStream_t,
                               cudaEvent_t*);

struct SortVariant {
  int key_bits, radix_bits, threads, kpt, rank;
  PassFn fn;
};

// The menu the autotuner chooses from (entry 0 of each key/digit width is
// the default).
const SortVariant kVariants[] = {
    {32, 8, 512, 16, kRankAtomicOr, passes_t<uint32_t, 8, 512, 16, kRankAtomicOr, 2>},
    {32, 8, 384, 16, kRankAtomicOr, passes_t<uint32_t, 8, 384, 16, kRankAtomicOr, 2>},
    {32, 8, 256, 16, kRankAtomicOr, passes_t<uint32_t, 8, 256, 16, kRankAtomicOr, 3>},
    {32, 8, 256, 24, kRankAtomicOr, passes_t<uint32_t, 8, 256, 24, kRankAtomicOr, 2>},
    {32, 8, 384, 24, kRankAtomicOr, passes_t<uint32_t, 8, 384, 24, kRankAtomicOr, 2>},
    {32, 8, 512, 24, kRankAtomicOr, passes_t<uint32_t, 8, 512, 24, kRankAtomicOr, 1>},
    {32, 8, 256, 16, kRankBallot, passes_t<uint32_t, 8, 256, 16, kRankBallot, 3>},
    {32, 8, 512, 16, kRankBallot, passes_t<uint32_t, 8, 512, 16, kRankBallot, 1>},
    {32, 8, 384, 16, kRankMatchAny, passes_t<uint32_t, 8, 384, 16, kRankMatchAny, 2>},
    {32, 11, 512, 16, kRankBallot, passes_t<uint32_t, 11, 512, 16, kRankBallot, 1>},
    {32, 11, 256, 16, kRankAtomicOr, passes_t<uint32_t, 11, 256, 16, kRankAtomicOr, 1>},
    {32, 11, 256, 24, kRankAtomicOr, passes_t<uint32_t, 11, 256, 24, kRankAtomicOr, 1>},
    {32, 11, 256, 24, kRankBallot, passes_t<uint32_t, 11, 256, 24, kRankBallot, 1>},
    {64, 8, 384, 16, kRankAtomicOr, passes_t<uint64_t, 8, 384, 16, kRankAtomicOr, 2>},
    {64, 8, 256, 16, kRankAtomicOr, passes_t<uint64_t, 8, 256, 16, kRankAtomicOr, 2>},
    {64, 8, 256, 12, kRankAtomicOr, passes_t<uint64_t, 8, 256, 12, kRankAtomicOr, 3>},
    {64, 8, 256, 16, kRankBallot, passes_t<uint64_t, 8, 256, 16, kRankBallot, 2>},
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

cudaError_t launch_morton(const rw_tree_app_data& app, rw_tree_im_storage* im,
                          bool with_histogram, cudaStream_t s) {
  if (app.key_bits == 32)
    return im->radix_bits == 8 ? morton_t<uint32_t, 8>(app, im, with_histogram, s)
                               : morton_t<uint32_t, 11>(app, im, with_histogram, s);
  return im->radix_bits == 8 ? morton_t<uint64_t, 8>(app, im, with_histogram, s)
                             : morton_t<uint64_t, 11>(app, im, with_histogram, s);
}

cudaError_t launch_histogram(const rw_tree_app_data& app, rw_tree_im_storage* im,
                             cudaStream_t s) {
  if (app.key_bits == 32)
    return im->radix_bits == 8 ? histogram_t<uint32_t, 8>(app, im, s)
                               : histogram_t<uint32_t, 11>(app, im, s);
  return im->radix_bits == 8 ? histogram_t<uint64_t, 8>(app, im, s)
                             : histogram_t<uint64_t, 11>(app, im, s);
}

cudaError_t launch_sort_passes(const rw_tree_app_data& app,
                               rw_tree_im_storage* im, cudaStream_t s,
                               cudaEvent_t* marks) {
  const int v = im->sort_variant;
  if (v < 0 || v >= kNumVariants || kVariants[v].key_bits != app.key_bits ||
      kVariants[v].radix_bits != im->radix_bits)
    return cudaErrorInvalidValue;
  return kVariants[v].fn(app, im, s, marks);
}

}  // namespace rwt
