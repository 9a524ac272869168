// Learned-CDF bucketed sort of 32-bit keys (no reference counterpart; the
// reference sorts with an LSD radix sort only).
//
//  1. a stratified 64K-key sample of the input, sorted with the onesweep sort;
//  2. 4,095 bucket boundaries.  Without the network boundary j is the sample
//     key of rank c = 16(j+1) (the plain sample quantile).  With it, the MLP
//     (mlp.cuh) reads a context of 16g sorted sample keys centred on c (eight
//     inputs: mean positions of eight groups of 2g keys; eight more: the exact
//     positions of the keys of ranks c-4 .. c+3; all normalised to the
//     context's key range) and returns the boundary's offset from c in sample
//     ranks; the key is interpolated between the two sample keys around that
//     fractional rank.  This is a smoothed inversion of the sample's CDF that
//     averages the sampling noise of the whole context instead of taking one
//     order statistic.  A prefix maximum then makes the boundaries
//     non-decreasing;//  3. bucket(k) = number of boundaries <= k, a non-decreasing function, so
//     sorting every bucket and concatenating them sorts the input;
//  4. one histogram pass, a plan (offsets, overflow), one scatter pass;
//  5. one CTA per bucket sorts it in shared memory (stable LSD over only the
//     bits its keys span); a bucket above the CTA's capacity is sorted by one
//     CTA in chunks through global memory; a bucket above kBigCap sends the
//     whole input back to the onesweep sort (decided on the host).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "internal.hpp"
#include "mlp.cuh"

namespace rwt {

constexpr uint32_t kSample = 65536, kBuckets = 4096, kBounds = kBuckets - 1;
constexpr uint32_t kSpacing = kSample / kBuckets;  // sample keys per bucket
static_assert(kSpacing == uint32_t(kMlpIn), "one window of MLP inputs per bucket");
constexpr int kBsThreads = 1024, kBsKpt = 32;
constexpr uint32_t kBucketCap = kBsThreads * kBsKpt;  // keys one CTA sorts in smem
constexpr uint32_t kBigCap = 1u << 21;              // beyond: onesweep for everything
constexpr int kScThreads = 512, kScKpt = 32;
constexpr uint32_t kScTile = kScThreads * kScKpt;

struct LearnedPlan {
  uint32_t max_count;
  uint32_t n_big;       // buckets above kBucketCap
  uint32_t fallback;    // some bucket above kBigCap
  uint32_t pad;
};

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// 1. stratified sample: one key from each of kSample equal strata
__global__ void k_sample(const uint32_t* __restrict__ keys, uint32_t n,
                         uint32_t* __restrict__ sample) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kSample) return;
  const uint64_t lo = (uint64_t(i) * n) / kSample, hi = (uint64_t(i + 1) * n) / kSample;
  const uint32_t w = uint32_t(hi - lo);
  const uint64_t pos = w ? lo + mix32(i * 2654435761u + 12345u) % w : (uint64_t(i) % n);
  sample[i] = keys[pos];
}

// Context group sizes the boundary MLP accepts (context = 16 * group keys).
constexpr uint32_t kMaxGroup = 16;

// MLP inputs of boundary j (sample rank c, context [c - half, c + half)).
__device__ __forceinline__ void boundary_features(const uint32_t* __restrict__ s, uint32_t c,
                                                  uint32_t half, uint32_t group,
                                                  float (&x)[kMlpIn]) {
  const uint32_t* ctx = s + (c - half);
  const uint32_t lo = ctx[0], span = max(ctx[2 * half - 1] - lo, 1u);
  const uint32_t g2 = 2 * group;  // keys per coarse group
  const float fspan = float(span);
  const float denom = __fmul_rn(float(g2), fspan);
#pragma unroll
  for (int i = 0; i < kMlpIn / 2; ++i) {
    uint64_t sum = 0;
    for (uint32_t q = 0; q < g2; ++q) sum += ctx[i * g2 + q] - lo;
    x[i] = __fdiv_rn(__ull2float_rn(sum), denom);
  }
#pragma unroll
  for (int i = 0; i < kMlpIn / 2; ++i)
    x[kMlpIn / 2 + i] = __fdiv_rn(float(s[c - kMlpIn / 4 + i] - lo), fspan);
}

// 2. boundaries (and, for training, the MLP inputs of every boundary; rows
// whose context does not fit inside the sample are written as zeros and keep
// the sample quantile).  MLP boundaries still need k_bounds_monotone.
template <bool USE_MLP>
__global__ void __launch_bounds__(256)
    k_boundaries(const uint32_t* __restrict__ sorted_sample, const float* __restrict__ params,
                 uint32_t group, uint32_t* __restrict__ bounds, float* __restrict__ features) {
  __shared__ float s_w1[kMlpHidden * kMlpIn], s_w2[kMlpHidden * kMlpHidden], s_w3[kMlpHidden],
      s_b1[kMlpHidden], s_b2[kMlpHidden];
  if (USE_MLP) {
    constexpr int oW1 = 0, oB1 = oW1 + kMlpHidden * kMlpIn, oW2 = oB1 + kMlpHidden,
                  oB2 = oW2 + kMlpHidden * kMlpHidden, oW3 = oB2 + kMlpHidden;
    for (int i = threadIdx.x; i < kMlpHidden * kMlpIn; i += blockDim.x)
      s_w1[i] = __bfloat162float(__float2bfloat16_rn(params[oW1 + i]));
    for (int i = threadIdx.x; i < kMlpHidden * kMlpHidden; i += blockDim.x)
      s_w2[i] = __bfloat162float(__float2bfloat16_rn(params[oW2 + i]));
    for (int i = threadIdx.x; i < kMlpHidden; i += blockDim.x) {
      s_w3[i] = __bfloat162float(__float2bfloat16_rn(params[oW3 + i]));
      s_b1[i] = params[oB1 + i];
      s_b2[i] = params[oB2 + i];
    }
    __syncthreads();
  }
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= kBounds) return;
  const uint32_t c = (j + 1) * kSpacing;  // sample rank of the ideal boundary
  const uint32_t half = (kMlpIn / 2) * group;
  const bool fits = c >= half && c + half <= kSample;
  uint32_t b = sorted_sample[c];
  if ((USE_MLP || features) && fits) {
    float x[kMlpIn];
    boundary_features(sorted_sample, c, half, group, x);
    if (features) {
#pragma unroll
      for (int i = 0; i < kMlpIn; ++i) features[size_t(j) * kMlpIn + i] = x[i];
    }
    if (USE_MLP) {
      // offset in sample ranks, d in [-half, half - 1]
      const float y = mlp_eval(x, s_w1, s_b1, s_w2, s_b2, s_w3, params[kMlpParams - 1]);
      const float fh = float(half);
      const float d = fminf(fmaxf(__fmul_rn(y, fh), -fh), fh - 1.0f);
      const float fl = floorf(d);
      const uint32_t i0 = uint32_t(int(c) + int(fl));
      const uint32_t i1 = min(i0 + 1, kSample - 1);
      const uint32_t a0 = sorted_sample[i0], gap = sorted_sample[i1] - a0;
      b = a0 + min(uint32_t(__fmul_rn(d - fl, float(gap)) + 0.5f), gap);
    }
  } else if (features) {
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) features[size_t(j) * kMlpIn + i] = 0.0f;
  }
  bounds[j] = b;
}

// prefix maximum over the boundaries (one block): non-decreasing boundaries
// are what makes "bucket = number of boundaries <= key" order-preserving
__global__ void __launch_bounds__(1024) k_bounds_monotone(uint32_t* __restrict__ bounds) {
  __shared__ uint32_t s_warp[32];
  constexpr int R = kBuckets / 1024;
  const int first = threadIdx.x * R;
  uint32_t v[R], mx = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    v[r] = first + r < int(kBounds) ? bounds[first + r] : 0u;
    mx = max(mx, v[r]);
  }
  // inclusive max-scan of the per-thread maxima
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t inc = mx;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, inc, d);
    if (int(lane) >= d) inc = max(inc, o);
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = s_warp[lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, w, d);
      if (int(lane) >= d) w = max(w, o);
    }
    s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t run = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) run = 0;
  if (warp > 0) run = max(run, s_warp[warp - 1]);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    run = max(run, v[r]);
    if (first + r < int(kBounds)) bounds[first + r] = run;
  }
}

// Splitter tree (Sanders & Winkel, "Super Scalar Sample Sort", ESA 2004): the
// 4,095 sorted boundaries in breadth-first order, t[1] the median, children of
// node i at 2i and 2i+1.  A descent reads one node per level; the five top
// levels are 31 consecutive words (no bank conflicts between lanes), where a
// binary search over the sorted array would put its top levels in one bank.
// t[0] is unused.
__device__ __forceinline__ void load_tree(const uint32_t* __restrict__ bounds, uint32_t* s_t) {
  constexpr int kLevels = 12;
  static_assert((1u << kLevels) == kBuckets, "complete tree");
  for (int i = threadIdx.x + 1; i < int(kBuckets); i += blockDim.x) {
    const int d = 31 - __clz(i);   // depth of node i
    const int p = i - (1 << d);    // position in its level
    s_t[i] = bounds[((2 * p + 1) << (kLevels - 1 - d)) - 1];
  }
}

// bucket of key k: number of boundaries <= k
__device__ __forceinline__ uint32_t bucket_of(const uint32_t* s_t, uint32_t k) {
  uint32_t i = 1;
#pragma unroll
  for (int it = 0; it < 12; ++it) i = 2 * i + (k >= s_t[i] ? 1u : 0u);
  return i - kBuckets;
}

// 4a. histogram of the buckets
__global__ void __launch_bounds__(512)
    k_bucket_hist(const uint32_t* __restrict__ keys, uint32_t n,
                  const uint32_t* __restrict__ bounds, uint32_t* __restrict__ counts) {
  __shared__ uint32_t s_b[kBuckets], s_cnt[kBuckets];
  load_tree(bounds, s_b);
  for (int i = threadIdx.x; i < int(kBuckets); i += blockDim.x) s_cnt[i] = 0;
  __syncthreads();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    atomicAdd(&s_cnt[bucket_of(s_b, __ldcs(keys + i))], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < int(kBuckets); i += blockDim.x)
    if (s_cnt[i]) atomicAdd(&counts[i], s_cnt[i]);
}

// 4b. plan: offsets, write cursors, overflow summary (one block)
__global__ void __launch_bounds__(1024)
    k_bucket_plan(const uint32_t* __restrict__ counts, uint32_t* __restrict__ offsets,
                  uint32_t* __restrict__ cursor, LearnedPlan* __restrict__ plan) {
  __shared__ uint32_t s_warp[33];
  constexpr int R = kBuckets / 1024;
  const int first = threadIdx.x * R;
  uint32_t v[R], local = 0, mx = 0, big = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    v[r] = counts[first + r];
    local += v[r];
    mx = max(mx, v[r]);
    big += v[r] > kBucketCap;
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan<1024>(local, s_warp, &total);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    offsets[first + r] = run;
    cursor[first + r] = run;
    run += v[r];
  }
  offsets[kBuckets] = total;
  atomicMax(&plan->max_count, mx);
  if (big) atomicAdd(&plan->n_big, big);
  if (mx > kBigCap) plan->fallback = 1;
}

// 4c. scatter into the buckets: within a tile keys are grouped by bucket in
// shared memory and each bucket's run is written at a position reserved with
// one atomic on the bucket's cursor (the order inside a bucket is free: the
// bucket is sorted next).  The bucket id of every placed key is kept in shared
// memory so that the write-out does not search the boundaries again.
__global__ void __launch_bounds__(kScThreads)
    k_bucket_scatter(const uint32_t* __restrict__ keys, uint32_t n,
                     const uint32_t* __restrict__ bounds, uint32_t* __restrict__ cursor,
                     uint32_t* __restrict__ out) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint32_t* s_keys = sm;                  // [kScTile]
  uint32_t* s_b = s_keys + kScTile;       // [kBuckets] splitter tree
  uint32_t* s_cnt = s_b + kBuckets;       // [kBuckets] counts, then global bases
  uint32_t* s_pos = s_cnt + kBuckets;     // [kBuckets] starts, then fill cursors
  uint32_t* s_start = s_pos + kBuckets;   // [kBuckets]
  uint16_t* s_bid = reinterpret_cast<uint16_t*>(s_start + kBuckets);  // [kScTile]
  uint32_t* s_warp = reinterpret_cast<uint32_t*>(s_bid + kScTile);    // [kScThreads/32+1]
  load_tree(bounds, s_b);
  for (int i = threadIdx.x; i < int(kBuckets); i += kScThreads) s_cnt[i] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * kScTile;
  uint32_t k[kScKpt];
  uint16_t bid[kScKpt];
#pragma unroll
  for (int i = 0; i < kScKpt; ++i) {
    const uint32_t idx = base + i * kScThreads + threadIdx.x;
    k[i] = idx < n ? __ldcs(keys + idx) : 0u;
    bid[i] = uint16_t(bucket_of(s_b, k[i]));
    if (idx < n) atomicAdd(&s_cnt[bid[i]], 1u);
  }
  __syncthreads();
  constexpr int R = kBuckets / kScThreads;
  const int first = threadIdx.x * R;
  uint32_t c[R], local = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    c[r] = s_cnt[first + r];
    local += c[r];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan<kScThreads>(local, s_warp, &total);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    s_start[first + r] = run;
    s_pos[first + r] = run;
    run += c[r];
    s_cnt[first + r] = c[r] ? atomicAdd(&cursor[first + r], c[r]) : 0u;  // global base
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScKpt; ++i) {
    const uint32_t idx = base + i * kScThreads + threadIdx.x;
    if (idx < n) {
      const uint32_t p = atomicAdd(&s_pos[bid[i]], 1u);
      s_keys[p] = k[i];
      s_bid[p] = bid[i];
    }
  }
  __syncthreads();
  const uint32_t tile_n = min(kScTile, n - base);
  for (uint32_t p = threadIdx.x; p < tile_n; p += kScThreads) {
    const uint32_t b = s_bid[p];
    out[s_cnt[b] + (p - s_start[b])] = s_keys[p];
  }
}

constexpr size_t kScSmem =
    (size_t(kScTile) + 4 * size_t(kBuckets) + 64) * 4 + size_t(kScTile) * 2;

// Stable block-wide LSD sort of `cnt` <= kBucketCap keys held in registers
// (warp w holds items [w*32*KPT, (w+1)*32*KPT), step i, lane l -> item
// w*32*KPT + i*32 + l), over bits [0, bits).  Each pass counts the digits per
// warp (shared-memory atomic-OR peer matching), scans them, then ranks again
// and scatters straight to shared memory: no ranks are kept in registers.
// The result is left in s_keys[0, cnt).
template <int THREADS, int KPT>
__device__ void block_lsd_sort(uint32_t (&k)[KPT], uint32_t cnt, int bits, uint32_t* s_keys,
                               uint32_t* s_hist, uint32_t* s_match, uint32_t* s_tot,
                               uint32_t* s_warp) {
  constexpr int NW = THREADS / 32, RADIX = 256;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t wbase = warp * 32u * KPT + lane;
  uint32_t* wh = s_hist + warp * RADIX;
  uint32_t* wm = s_match + warp * RADIX;
  for (int shift = 0; shift < bits; shift += 8) {
    for (int i = threadIdx.x; i < NW * RADIX; i += THREADS) {
      s_hist[i] = 0;
      s_match[i] = 0;
    }
    __syncthreads();
    // count per warp
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      const bool valid = wbase + 32u * i < cnt;
      const uint32_t dig = (k[i] >> shift) & 255u;
      if (valid) atomicOr(&wm[dig], 1u << lane);
      __syncwarp();
      const uint32_t peers = valid ? wm[dig] : 0u;
      __syncwarp();
      if (valid && __popc(peers & lanemask_lt()) == 0) {
        wh[dig] += __popc(peers);
        wm[dig] = 0;
      }
      __syncwarp();
    }
    __syncthreads();
    // digit totals, exclusive over digits, then per-warp starts
    if (threadIdx.x < RADIX) {
      uint32_t t = 0;
      for (int w = 0; w < NW; ++w) t += s_hist[w * RADIX + threadIdx.x];
      s_tot[threadIdx.x] = t;
    }
    __syncthreads();
    {
      const uint32_t t = threadIdx.x < RADIX ? s_tot[threadIdx.x] : 0u;
      uint32_t tot;
      const uint32_t ex = block_exclusive_scan<THREADS>(t, s_warp, &tot);
      if (threadIdx.x < RADIX) {
        uint32_t run = ex;
        for (int w = 0; w < NW; ++w) {
          const uint32_t c = s_hist[w * RADIX + threadIdx.x];
          s_hist[w * RADIX + threadIdx.x] = run;
          run += c;
        }
      }
    }
    __syncthreads();
    // rank again and scatter
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      const bool valid = wbase + 32u * i < cnt;
      const uint32_t dig = (k[i] >> shift) & 255u;
      if (valid) atomicOr(&wm[dig], 1u << lane);
      __syncwarp();
      const uint32_t peers = valid ? wm[dig] : 0u;
      __syncwarp();
      const uint32_t below = __popc(peers & lanemask_lt());
      uint32_t prev = 0;
      if (valid && below == 0) {
        prev = wh[dig];
        wh[dig] = prev + __popc(peers);
        wm[dig] = 0;
      }
      const int leader = valid ? __ffs(peers) - 1 : int(lane);
      prev = __shfl_sync(0xffffffffu, prev, leader);
      if (valid) s_keys[prev + below] = k[i];
      __syncwarp();
    }
    __syncthreads();
    if (shift + 8 < bits) {
#pragma unroll
      for (int i = 0; i < KPT; ++i) {
        const uint32_t idx = wbase + 32u * i;
        k[i] = idx < cnt ? s_keys[idx] : 0u;
      }
      __syncthreads();
    }
  }
  if (bits <= 0) {  // every key equal: keep them as they are
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      const uint32_t idx = wbase + 32u * i;
      if (idx < cnt) s_keys[idx] = k[i];
    }
    __syncthreads();
  }
}

// smem layout of the bucket sort kernel
constexpr size_t kBsSmem =
    (size_t(kBucketCap) + 2 * size_t(kBsThreads / 32) * 256 + 256 + 64) * 4;

// 5a. one CTA per bucket of at most kBucketCap keys
__global__ void __launch_bounds__(kBsThreads, 1)
    k_bucket_sort(const uint32_t* __restrict__ in, const uint32_t* __restrict__ offsets,
                  uint32_t* __restrict__ out) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint32_t* s_keys = sm;
  uint32_t* s_hist = s_keys + kBucketCap;
  uint32_t* s_match = s_hist + (kBsThreads / 32) * 256;
  uint32_t* s_tot = s_match + (kBsThreads / 32) * 256;
  uint32_t* s_warp = s_tot + 256;
  const uint32_t b = blockIdx.x;
  const uint32_t off = offsets[b], cnt = offsets[b + 1] - off;
  if (cnt == 0 || cnt > kBucketCap) return;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t wbase = warp * 32u * kBsKpt + lane;
  uint32_t k[kBsKpt];
  uint32_t mn = 0xffffffffu, mx = 0;
#pragma unroll
  for (int i = 0; i < kBsKpt; ++i) {
    const uint32_t idx = wbase + 32u * i;
    k[i] = idx < cnt ? in[off + idx] : 0u;
    if (idx < cnt) {
      mn = min(mn, k[i]);
      mx = max(mx, k[i]);
    }
  }
  // key span of the bucket: only the bits below the common prefix are sorted
  for (int d = 16; d > 0; d >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, d));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
  }
  if (threadIdx.x == 0) {
    s_warp[40] = 0xffffffffu;
    s_warp[41] = 0;
  }
  __syncthreads();
  if (lane == 0) {
    atomicMin(&s_warp[40], mn);
    atomicMax(&s_warp[41], mx);
  }
  __syncthreads();
  const uint32_t diff = s_warp[40] ^ s_warp[41];
  const int bits = diff ? 32 - __clz(diff) : 0;
  __syncthreads();
  block_lsd_sort<kBsThreads, kBsKpt>(k, cnt, bits, s_keys, s_hist, s_match, s_tot, s_warp);
  for (uint32_t p = threadIdx.x; p < cnt; p += kBsThreads) out[off + p] = s_keys[p];
}

// 5b. a bucket above kBucketCap, one CTA, LSD through global memory: every
// pass histograms the whole bucket, then places chunks of kBucketCap keys in
// order (stable), ping-ponging between the bucket's ranges in `a` and `b`.
// The sorted bucket ends in `out` (== a or b).
__global__ void __launch_bounds__(kBsThreads, 1)
    k_bucket_sort_big(uint32_t* __restrict__ a, uint32_t* __restrict__ bb,
                      const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ counts,
                      uint32_t* __restrict__ out) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint32_t* s_keys = sm;
  uint32_t* s_hist = s_keys + kBucketCap;
  uint32_t* s_match = s_hist + (kBsThreads / 32) * 256;
  uint32_t* s_tot = s_match + (kBsThreads / 32) * 256;
  uint32_t* s_warp = s_tot + 256;
  const uint32_t bkt = blockIdx.x;
  const uint32_t off = offsets[bkt], cnt = counts[bkt];
  if (cnt <= kBucketCap || cnt > kBigCap) return;
  constexpr int NW = kBsThreads / 32, RADIX = 256;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  // key span
  uint32_t mn = 0xffffffffu, mx = 0;
  for (uint32_t p = threadIdx.x; p < cnt; p += kBsThreads) {
    const uint32_t v = a[off + p];
    mn = min(mn, v);
    mx = max(mx, v);
  }
  if (threadIdx.x == 0) {
    s_warp[40] = 0xffffffffu;
    s_warp[41] = 0;
  }
  __syncthreads();
  atomicMin(&s_warp[40], mn);
  atomicMax(&s_warp[41], mx);
  __syncthreads();
  const uint32_t diff = s_warp[40] ^ s_warp[41];
  const int bits = diff ? 32 - __clz(diff) : 0;
  __syncthreads();
  uint32_t* src = a + off;
  uint32_t* dst = bb + off;
  uint32_t* s_run = s_tot;  // running digit starts across chunks
  for (int shift = 0; shift < bits; shift += 8) {
    // digit histogram of the whole bucket -> exclusive starts
    for (int i = threadIdx.x; i < RADIX; i += kBsThreads) s_hist[i] = 0;
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < cnt; p += kBsThreads)
      atomicAdd(&s_hist[(src[p] >> shift) & 255u], 1u);
    __syncthreads();
    {
      const uint32_t t = threadIdx.x < RADIX ? s_hist[threadIdx.x] : 0u;
      uint32_t tot;
      const uint32_t ex = block_exclusive_scan<kBsThreads>(t, s_warp, &tot);
      if (threadIdx.x < RADIX) s_run[threadIdx.x] = ex;
    }
    __syncthreads();
    for (uint32_t c0 = 0; c0 < cnt; c0 += kBucketCap) {
      const uint32_t ccount = min(kBucketCap, cnt - c0);
      const uint32_t wbase = warp * 32u * kBsKpt + lane;
      uint32_t k[kBsKpt];
#pragma unroll
      for (int i = 0; i < kBsKpt; ++i) {
        const uint32_t idx = wbase + 32u * i;
        k[i] = idx < ccount ? src[c0 + idx] : 0u;
      }
      // per-warp counts of this chunk
      uint32_t* wh = s_hist + warp * RADIX;
      uint32_t* wm = s_match + warp * RADIX;
      for (int i = threadIdx.x; i < NW * RADIX; i += kBsThreads) {
        s_hist[i] = 0;
        s_match[i] = 0;
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < kBsKpt; ++i) {
        const bool valid = wbase + 32u * i < ccount;
        const uint32_t dig = (k[i] >> shift) & 255u;
        if (valid) atomicOr(&wm[dig], 1u << lane);
        __syncwarp();
        const uint32_t peers = valid ? wm[dig] : 0u;
        __syncwarp();
        if (valid && __popc(peers & lanemask_lt()) == 0) {
          wh[dig] += __popc(peers);
          wm[dig] = 0;
        }
        __syncwarp();
      }
      __syncthreads();
      // per-warp starts = running start of the digit + earlier warps
      if (threadIdx.x < RADIX) {
        uint32_t run = s_run[threadIdx.x];
        for (int w = 0; w < NW; ++w) {
          const uint32_t c = s_hist[w * RADIX + threadIdx.x];
          s_hist[w * RADIX + threadIdx.x] = run;
          run += c;
        }
        s_run[threadIdx.x] = run;
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < kBsKpt; ++i) {
        const bool valid = wbase + 32u * i < ccount;
        const uint32_t dig = (k[i] >> shift) & 255u;
        if (valid) atomicOr(&wm[dig], 1u << lane);
        __syncwarp();
        const uint32_t peers = valid ? wm[dig] : 0u;
        __syncwarp();
        const uint32_t below = __popc(peers & lanemask_lt());
        uint32_t prev = 0;
        if (valid && below == 0) {
          prev = wh[dig];
          wh[dig] = prev + __popc(peers);
          wm[dig] = 0;
        }
        const int leader = valid ? __ffs(peers) - 1 : int(lane);
        prev = __shfl_sync(0xffffffffu, prev, leader);
        if (valid && prev + below < cnt) dst[prev + below] = k[i];
        __syncwarp();
      }
      __syncthreads();
    }
    uint32_t* t = src;
    src = dst;
    dst = t;
    __threadfence_block();
    __syncthreads();
  }
  if (src != out + off)
    for (uint32_t p = threadIdx.x; p < cnt; p += kBsThreads) out[off + p] = src[p];
}

}  // namespace rwt

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

struct rw_tree_learned {
  uint32_t n_max = 0;
  int num_sms = 148;
  rw_tree_im_storage* sample_im = nullptr;  // onesweep scratch for the sample
  void* d_mem = nullptr;
  uint32_t *d_sample = nullptr, *d_sample_sorted = nullptr, *d_bounds = nullptr,
           *d_counts = nullptr, *d_offsets = nullptr, *d_cursor = nullptr,
           *d_tmp = nullptr;
  float* d_params = nullptr;
  float* d_features = nullptr;
  rwt::LearnedPlan* d_plan = nullptr;
  rwt::LearnedPlan* h_plan = nullptr;
  uint32_t group = 4;  // sample keys per MLP input
  bool has_params = false;
};

namespace {

int lfail(cudaError_t e, const char* what) {
  rwt::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return RW_ERR_CUDA;
}

#define RWL_CUDA(call)                                  \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return lfail(e_, #call);     \
  } while (0)

// sorts the sample (kSample keys) into d_sample_sorted with the onesweep sort
int sort_sample(rw_tree_learned* L, cudaStream_t s) {
  rw_tree_app_data app;
  rw_tree_app_data_init(&app, rwt::kSample, 32);
  app.u_morton_keys = L->d_sample;
  app.u_morton_keys_alt = L->d_sample_sorted;
  return rw_tree_sort_enqueue(&app, L->sample_im, reinterpret_cast<rw_stream_t>(s));
}

int boundaries(rw_tree_learned* L, bool mlp, bool features, cudaStream_t s) {
  if (mlp && !L->has_params) return RW_ERR_NOT_READY;
  float* f = features ? L->d_features : nullptr;
  const uint32_t blocks = (rwt::kBounds + 255) / 256;
  if (mlp) {
    rwt::k_boundaries<true><<<blocks, 256, 0, s>>>(L->d_sample_sorted, L->d_params, L->group,
                                                   L->d_bounds, f);
    RWL_CUDA(cudaGetLastError());
    rwt::k_bounds_monotone<<<1, 1024, 0, s>>>(L->d_bounds);
  } else
    rwt::k_boundaries<false><<<blocks, 256, 0, s>>>(L->d_sample_sorted, L->d_params, L->group,
                                                    L->d_bounds, f);
  RWL_CUDA(cudaGetLastError());
  return RW_OK;
}

int front_half(rw_tree_learned* L, const uint32_t* keys, uint32_t n, bool mlp, bool features,
               cudaStream_t s) {
  rwt::k_sample<<<rwt::kSample / 256, 256, 0, s>>>(keys, n, L->d_sample);
  RWL_CUDA(cudaGetLastError());
  if (int rc = sort_sample(L, s)) return rc;
  return boundaries(L, mlp, features, s);
}

int counts_and_plan(rw_tree_learned* L, const uint32_t* keys, uint32_t n, cudaStream_t s) {
  RWL_CUDA(cudaMemsetAsync(L->d_counts, 0, 4 * rwt::kBuckets, s));
  RWL_CUDA(cudaMemsetAsync(L->d_plan, 0, sizeof(rwt::LearnedPlan), s));
  const int blocks = std::max(1, std::min<int>(rwt::div_up(n, 512 * 16), L->num_sms * 4));
  rwt::k_bucket_hist<<<blocks, 512, 0, s>>>(keys, n, L->d_bounds, L->d_counts);
  RWL_CUDA(cudaGetLastError());
  rwt::k_bucket_plan<<<1, 1024, 0, s>>>(L->d_counts, L->d_offsets, L->d_cursor, L->d_plan);
  RWL_CUDA(cudaGetLastError());
  RWL_CUDA(cudaMemcpyAsync(L->h_plan, L->d_plan, sizeof(rwt::LearnedPlan),
                           cudaMemcpyDeviceToHost, s));
  return RW_OK;
}

}  // namespace

extern "C" {

int rw_tree_learned_create(uint32_t n_max, rw_tree_learned** out) {
  if (!out || n_max < rwt::kSample || n_max >= RW_MAX_POINTS) return RW_ERR_ARG;
  *out = nullptr;
  auto* L = new rw_tree_learned();
  L->n_max = n_max;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&L->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (int rc = rw_tree_im_storage_create(rwt::kSample, 32, &L->sample_im)) {
    delete L;
    return rc;
  }
  const size_t words = 2 * size_t(rwt::kSample) + rwt::kBuckets + rwt::kBuckets +
                       (rwt::kBuckets + 1) + rwt::kBuckets + size_t(n_max) +
                       rwt::kMlpParams + size_t(rwt::kBounds) * rwt::kMlpIn +
                       64 /* alignment of the plan */ + 64 /* plan */;
  cudaError_t e = cudaMalloc(&L->d_mem, 4 * words);
  if (e == cudaSuccess) e = cudaMallocHost(&L->h_plan, sizeof(rwt::LearnedPlan));
  if (e != cudaSuccess) {
    rw_tree_learned_destroy(L);
    return lfail(e, "rw_tree_learned_create");
  }
  uint32_t* p = static_cast<uint32_t*>(L->d_mem);
  L->d_sample = p; p += rwt::kSample;
  L->d_sample_sorted = p; p += rwt::kSample;
  L->d_bounds = p; p += rwt::kBuckets;
  L->d_counts = p; p += rwt::kBuckets;
  L->d_offsets = p; p += rwt::kBuckets + 1;
  L->d_cursor = p; p += rwt::kBuckets;
  L->d_params = reinterpret_cast<float*>(p); p += rwt::kMlpParams;
  L->d_features = reinterpret_cast<float*>(p); p += size_t(rwt::kBounds) * rwt::kMlpIn;
  p = reinterpret_cast<uint32_t*>((reinterpret_cast<uintptr_t>(p) + 255) & ~uintptr_t(255));
  L->d_plan = reinterpret_cast<rwt::LearnedPlan*>(p); p += 64;
  L->d_tmp = p;
  if ((reinterpret_cast<uintptr_t>(L->d_tmp) & 15u) != 0) {
    rw_tree_learned_destroy(L);
    return RW_ERR_ARG;
  }
  cudaFuncSetAttribute(rwt::k_bucket_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       int(rwt::kBsSmem));
  cudaFuncSetAttribute(rwt::k_bucket_sort_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       int(rwt::kBsSmem));
  cudaFuncSetAttribute(rwt::k_bucket_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       int(rwt::kScSmem));
  *out = L;
  return RW_OK;
}

int rw_tree_learned_destroy(rw_tree_learned* L) {
  if (!L) return RW_OK;
  if (L->sample_im) rw_tree_im_storage_destroy(L->sample_im);
  if (L->d_mem) cudaFree(L->d_mem);
  if (L->h_plan) cudaFreeHost(L->h_plan);
  delete L;
  return RW_OK;
}

int rw_tree_learned_set_params(rw_tree_learned* L, const float* params, int32_t count,
                               int32_t group) {
  if (!L || !params || count != rwt::kMlpParams) return RW_ERR_ARG;
  if (int rc = rw_tree_learned_set_group(L, group)) return rc;
  RWL_CUDA(cudaMemcpy(L->d_params, params, 4 * size_t(count), cudaMemcpyHostToDevice));
  L->has_params = true;
  return RW_OK;
}

int rw_tree_learned_set_group(rw_tree_learned* L, int32_t group) {
  if (!L || group < 1 || uint32_t(group) > rwt::kMaxGroup || (group & (group - 1))) return RW_ERR_ARG;
  L->group = uint32_t(group);
  return RW_OK;
}

int rw_tree_learned_features(rw_tree_learned* L, const uint32_t* d_keys, uint32_t n,
                             float* h_features, uint32_t* h_sorted_sample, rw_stream_t stream) {
  if (!L || !d_keys || n < rwt::kSample || n > L->n_max) return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = front_half(L, d_keys, n, false, true, s)) return rc;
  if (h_features)
    RWL_CUDA(cudaMemcpyAsync(h_features, L->d_features,
                             4 * size_t(rwt::kBounds) * rwt::kMlpIn, cudaMemcpyDeviceToHost, s));
  if (h_sorted_sample)
    RWL_CUDA(cudaMemcpyAsync(h_sorted_sample, L->d_sample_sorted, 4 * size_t(rwt::kSample),
                             cudaMemcpyDeviceToHost, s));
  RWL_CUDA(cudaStreamSynchronize(s));
  return RW_OK;
}

int rw_tree_learned_bucket_counts(rw_tree_learned* L, const uint32_t* d_keys, uint32_t n,
                                  int32_t mode, uint32_t* h_counts, rw_stream_t stream) {
  if (!L || !d_keys || !h_counts || n < rwt::kSample || n > L->n_max) return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = front_half(L, d_keys, n, mode == RW_LEARNED_MLP, false, s)) return rc;
  if (int rc = counts_and_plan(L, d_keys, n, s)) return rc;
  RWL_CUDA(cudaMemcpyAsync(h_counts, L->d_counts, 4 * rwt::kBuckets, cudaMemcpyDeviceToHost, s));
  RWL_CUDA(cudaStreamSynchronize(s));
  return RW_OK;
}

int rw_tree_learned_sort(rw_tree_learned* L, const uint32_t* d_keys, uint32_t* d_sorted,
                         uint32_t n, int32_t mode, rw_tree_im_storage* fallback_im,
                         rw_stream_t stream, rw_tree_learned_stats* stats) {
  if (!L || !d_keys || !d_sorted || n > L->n_max || n < 1 ||
      (mode != RW_LEARNED_MLP && mode != RW_LEARNED_SAMPLE_QUANTILES))
    return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (stats) std::memset(stats, 0, sizeof *stats);
  bool fallback = n < rwt::kSample;
  if (!fallback) {
    if (int rc = front_half(L, d_keys, n, mode == RW_LEARNED_MLP, false, s)) return rc;
    if (int rc = counts_and_plan(L, d_keys, n, s)) return rc;
    RWL_CUDA(cudaStreamSynchronize(s));  // the plan decides the path
    fallback = L->h_plan->fallback != 0;
    if (stats) {
      stats->max_bucket = L->h_plan->max_count;
      stats->big_buckets = L->h_plan->n_big;
    }
  }
  if (fallback) {
    if (!fallback_im) return RW_ERR_CAPACITY;
    rw_tree_app_data app;
    rw_tree_app_data_init(&app, n, 32);
    app.u_morton_keys = const_cast<uint32_t*>(d_keys);
    app.u_morton_keys_alt = d_sorted;
    if (stats) stats->fell_back = 1;
    return rw_tree_sort_enqueue(&app, fallback_im, stream);
  }
  const uint32_t tiles = rwt::div_up(n, rwt::kScTile);
  rwt::k_bucket_scatter<<<tiles, rwt::kScThreads, rwt::kScSmem, s>>>(d_keys, n, L->d_bounds,
                                                                     L->d_cursor, L->d_tmp);
  RWL_CUDA(cudaGetLastError());
  rwt::k_bucket_sort<<<rwt::kBuckets, rwt::kBsThreads, rwt::kBsSmem, s>>>(L->d_tmp, L->d_offsets,
                                                                         d_sorted);
  RWL_CUDA(cudaGetLastError());
  if (L->h_plan->n_big) {
    rwt::k_bucket_sort_big<<<rwt::kBuckets, rwt::kBsThreads, rwt::kBsSmem, s>>>(
        L->d_tmp, d_sorted, L->d_offsets, L->d_counts, d_sorted);
    RWL_CUDA(cudaGetLastError());
  }
  return RW_OK;
}

}  // extern "C"
