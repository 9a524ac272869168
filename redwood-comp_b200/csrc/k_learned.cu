// Learned-CDF bucketed sort of 32-bit keys (no reference counterpart; the
// reference sorts with an LSD radix sort only).
//
//  1. a stratified 64K-key sample of the input, sorted with the onesweep sort;
//  2. 4,095 bucket boundaries.  Without the network boundary j is the sample
//     key of rank c = 16(j+1) (the plain sample quantile).  With it, the MLP
//     (16 -> 64 -> 64 -> 1, BF16 weights, FP32 accumulation) reads a context of 16g sorted sample keys centred on c (eight
//     inputs: mean positions of eight groups of 2g keys; eight more: the exact
//     positions of the keys of ranks c-4 .. c+3; all normalised to the
//     context's key range) and returns the boundary's offset from c in sample
//     ranks; the key is interpolated between the two sample keys around that
//     fractional rank.  This is a smoothed inversion of the sample's CDF that
//     averages the sampling noise of the whole context instead of taking one
//     order statistic.  A prefix maximum then makes the boundaries
//     non-decreasing;//  3. bucket(k) = number of boundaries <= k, found by descending a splitter
//     tree; a non-decreasing function, so sorting every bucket and
//     concatenating them sorts the input;
//  4. two split passes, each writing runs long enough to coalesce: the
//     first descends the top 8 levels of the splitter tree and scatters into
//     256 super-bucket regions, the second descends each super-bucket's own
//     4 levels into its 16 buckets.  Regions have fixed capacities (1.5x the
//     mean super-bucket, 4x the mean bucket), so no histogram pass comes
//     first; a tile counts its keys per bin, reserves each bin's run with one
//     atomic and writes the run from shared memory.  The order inside a
//     bucket is free (the bucket is sorted next);
//  5. a plan (bucket offsets, overflow, big buckets first) and one CTA per
//     bucket.  The output is keys only, so a bucket whose keys span at most
//     2^15 values is a counting sort: a histogram over its value range,
//     a scan, and an expansion of every value into its copies.  Wider buckets
//     run a stable LSD in shared memory over the bits they span, with the
//     onesweep passes' warp ranking; a bucket above one CTA's capacity is
//     sorted by its CTA in chunks through global memory.  A region that
//     overflowed sends the whole input to the onesweep sort, decided on the
//     device: the onesweep kernels are enqueued behind the bucket sort with a
//     gate on the plan's overflow word (they return at once when it is 0, the
//     bucket sort returns at once when it is 1), so no host wait is needed
//     and the whole sort can be captured in a CUDA graph.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "internal.hpp"
#include "mlp.cuh"
#include "rank.cuh"

namespace rwt {

constexpr uint32_t kSample = 65536, kBuckets = 4096, kBounds = kBuckets - 1;
constexpr uint32_t kSpacing = kSample / kBuckets;  // sample keys per bucket
static_assert(kSpacing == uint32_t(kMlpIn), "one window of MLP inputs per bucket");
constexpr int kBsThreads = 1024, kBsKpt = 32;
constexpr uint32_t kBucketCap = kBsThreads * kBsKpt;  // keys one CTA sorts in smem

// Region of one bucket for n keys: 4x the mean bucket size (at least the
// mean + 64), a multiple of 32 keys.
__host__ __device__ inline uint32_t region_cap(uint32_t n) {
  const uint32_t mean = (n + kBuckets - 1) / kBuckets;
  const uint32_t c = mean * 4 > mean + 64 ? mean * 4 : mean + 64;
  return (c + 31) & ~31u;
}

constexpr uint32_t kSupers = 256;  // first split: top 8 tree levels
constexpr uint32_t kCountSpan = 1u << 15;  // value range of the counting path

// Region of one super-bucket for n keys: 1.5x the mean plus 1,024 keys.
__host__ __device__ inline uint32_t super_cap(uint32_t n) {
  const uint32_t mean = (n + kSupers - 1) / kSupers;
  return (mean + mean / 2 + 1024 + 31) & ~31u;
}

struct LearnedPlan {
  uint32_t max_count;
  uint32_t n_big;       // buckets above kBucketCap
  uint32_t fallback;    // some bucket overflowed its region
  uint32_t mlp_timeout; // copy of the boundary network's error word
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
  pdl_enter();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kSample) return;
  const uint64_t lo = (uint64_t(i) * n) / kSample, hi = (uint64_t(i + 1) * n) / kSample;
  const uint32_t w = uint32_t(hi - lo);
  const uint64_t pos = w ? lo + mix32(i * 2654435761u + 12345u) % w : (uint64_t(i) % n);
  sample[i] = keys[pos];
}

// Context group sizes the boundary MLP accepts (context = 16 * group keys).
constexpr uint32_t kMaxGroup = 16;

// MLP input i of boundary j (sample rank c, context [c - half, c + half)):
// i < 8 the mean position of the i-th group of 2g context keys, i >= 8 the
// position of the key of rank c - 12 + i; normalised to the context's range.
__device__ __forceinline__ float boundary_feature(const uint32_t* __restrict__ s, uint32_t c,
                                                  uint32_t half, uint32_t group, int i) {
  const uint32_t* ctx = s + (c - half);
  const uint32_t lo = ctx[0], span = max(ctx[2 * half - 1] - lo, 1u);
  const float fspan = float(span);
  if (i < kMlpIn / 2) {
    const uint32_t g2 = 2 * group;  // keys per coarse group
    uint64_t sum = 0;
    for (uint32_t q = 0; q < g2; ++q) sum += ctx[i * g2 + q] - lo;
    return __fdiv_rn(__ull2float_rn(sum), __fmul_rn(float(g2), fspan));
  }
  return __fdiv_rn(float(s[c - kMlpIn / 4 + (i - kMlpIn / 2)] - lo), fspan);
}

__device__ __forceinline__ void boundary_features(const uint32_t* __restrict__ s, uint32_t c,
                                                  uint32_t half, uint32_t group,
                                                  float (&x)[kMlpIn]) {
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) x[i] = boundary_feature(s, c, half, group, i);
}

// Boundary key from the network's output y: offset d = y * half sample ranks
// from c (clamped to the context), interpolated between the two sample keys
// around the fractional rank c + d.
__device__ __forceinline__ uint32_t boundary_from_output(const uint32_t* __restrict__ s,
                                                         uint32_t c, uint32_t half, float y) {
  const float fh = float(half);
  const float d = fminf(fmaxf(__fmul_rn(y, fh), -fh), fh - 1.0f);
  const float fl = floorf(d);
  const uint32_t i0 = uint32_t(int(c) + int(fl));
  const uint32_t i1 = min(i0 + 1, kSample - 1);
  const uint32_t a0 = s[i0], gap = s[i1] - a0;
  return a0 + min(uint32_t(__fmul_rn(d - fl, float(gap)) + 0.5f), gap);
}

// 2. sample-quantile boundaries (and, for training, the MLP inputs of every
// boundary; rows whose context does not fit inside the sample are zero)
__global__ void __launch_bounds__(256)
    k_boundaries(const uint32_t* __restrict__ sorted_sample, uint32_t group,
                 uint32_t* __restrict__ bounds, float* __restrict__ features) {
  pdl_enter();
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= kBounds) return;
  const uint32_t c = (j + 1) * kSpacing;  // sample rank of the ideal boundary
  bounds[j] = sorted_sample[c];
  if (!features) return;
  const uint32_t half = (kMlpIn / 2) * group;
  const bool fits = c >= half && c + half <= kSample;
  float x[kMlpIn];
  if (fits) boundary_features(sorted_sample, c, half, group, x);
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) features[size_t(j) * kMlpIn + i] = fits ? x[i] : 0.0f;
}

// prefix maximum over the boundaries (one block): non-decreasing boundaries
// are what makes "bucket = number of boundaries <= key" order-preserving
__global__ void __launch_bounds__(1024) k_bounds_monotone(uint32_t* __restrict__ bounds) {
  pdl_enter();
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

// 2'. MLP boundaries on the tensor cores: one CTA per 128 boundaries, thread
// t computes boundary (CTA * 128 + t)'s inputs (those k_boundaries writes for
// training), the two hidden layers are tcgen05 MMAs (mlp.cuh), and the thread
// turns its row's output into the boundary key.  A boundary whose context does
// not fit inside the sample, or whose CTA's tensor-core wait ran out (*err set),
// stays the sample quantile.
__global__ void __launch_bounds__(kMlpTcThreads)
    k_boundaries_mlp(const uint32_t* __restrict__ sorted_sample, const float* __restrict__ params,
                     uint32_t group, uint32_t* __restrict__ bounds, uint32_t* __restrict__ err) {
  pdl_enter();
  const uint32_t half = (kMlpIn / 2) * group;
  const uint32_t j = blockIdx.x * uint32_t(kMlpTcRows) + threadIdx.x;
  const uint32_t c = (j + 1) * kSpacing;  // sample rank of the ideal boundary
  const bool fits = j < kBounds && c >= half && c + half <= kSample;
  mlp_tile_tc(
      params,
      [&](int, float (&x)[kMlpIn]) {
        if (fits) boundary_features(sorted_sample, c, half, group, x);
        return fits;
      },
      [&](int, float y, bool ok) {
        if (j < kBounds)
          bounds[j] = fits && ok ? boundary_from_output(sorted_sample, c, half, y)
                                 : sorted_sample[c];
      },
      err);
}

// 4. one split pass.  Segment `seg` of the source (its keys: n, or
// seg_counts[seg] at src + seg * src_cap) is split by the LEVELS tree levels
// below node root0 + seg into 2^LEVELS bins; bin i goes to output region
// out0 + i, out0 = (root0 + seg) * 2^LEVELS - 2^(depth of the bins' level).
// Tiles of TILE keys: grid = segments * tiles_per_seg.
constexpr int kSpThreads = 512, kSpKpt = 16;
constexpr uint32_t kSpTile = kSpThreads * kSpKpt;

template <int LEVELS>
struct SplitCfg {
  static constexpr uint32_t BINS = 1u << LEVELS;
  static constexpr size_t kSmem = size_t(kSpTile) * 4 + size_t(kSpTile) + 4 * size_t(BINS) * 4;
};

template <int LEVELS>
__global__ void __launch_bounds__(kSpThreads, 2)
    k_split(const uint32_t* __restrict__ src, uint32_t n, const uint32_t* __restrict__ seg_counts,
            uint32_t src_cap, uint32_t tiles_per_seg, uint32_t root0,
            const uint32_t* __restrict__ bounds, uint32_t* __restrict__ cursor,
            uint32_t* __restrict__ region, uint32_t cap) {
  pdl_enter();
  using C = SplitCfg<LEVELS>;
  constexpr uint32_t BINS = C::BINS;
  static_assert(BINS <= 256, "bins are kept in bytes");
  extern __shared__ __align__(16) uint32_t sm[];
  uint32_t* s_keys = sm;                                   // [kSpTile]
  uint8_t* s_bin = reinterpret_cast<uint8_t*>(s_keys + kSpTile);  // [kSpTile]
  uint32_t* s_t = reinterpret_cast<uint32_t*>(s_bin + kSpTile);   // local tree [BINS]
  uint32_t* s_cnt = s_t + BINS;
  uint32_t* s_start = s_cnt + BINS;
  uint32_t* s_base = s_start + BINS;
  const uint32_t seg = blockIdx.x / tiles_per_seg, chunk = blockIdx.x % tiles_per_seg;
  const uint32_t seg_n = seg_counts ? min(seg_counts[seg], src_cap) : n;
  const uint32_t base = chunk * kSpTile;
  if (base >= seg_n) return;  // the whole CTA: the segment is shorter
  const uint32_t* in = src + size_t(seg) * src_cap + base;
  const uint32_t tile_n = min(kSpTile, seg_n - base);
  const uint32_t root = root0 + seg;
  const int root_depth = 31 - __clz(root);
  // the subtree below root, LEVELS deep, as a local heap (local node m at
  // depth d = global node root * 2^d + m - 2^d)
  for (uint32_t m = threadIdx.x + 1; m < BINS; m += kSpThreads) {
    const int d = 31 - __clz(m);
    const uint32_t g = (root << d) + (m - (1u << d));
    const int D = root_depth + d;
    const uint32_t pg = g - (1u << D);
    s_t[m] = bounds[((2 * pg + 1) << (11 - D)) - 1];
  }
  for (uint32_t i = threadIdx.x; i < BINS; i += kSpThreads) s_cnt[i] = 0;
  __syncthreads();
  uint32_t k[kSpKpt];
  // vector loads need a whole tile on a 16-byte boundary (a cloud of a batch
  // may start anywhere)
  const bool full = tile_n == kSpTile && (reinterpret_cast<uintptr_t>(in) & 15u) == 0;
  if (full) {
    const uint4* v = reinterpret_cast<const uint4*>(in);
#pragma unroll
    for (int i = 0; i < kSpKpt / 4; ++i) {
      const uint4 q = __ldcs(v + threadIdx.x + i * kSpThreads);
      k[4 * i] = q.x;
      k[4 * i + 1] = q.y;
      k[4 * i + 2] = q.z;
      k[4 * i + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < kSpKpt / 4; ++i)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t p = 4 * (threadIdx.x + i * kSpThreads) + e;
        k[4 * i + e] = p < tile_n ? in[p] : 0u;
      }
  }
  // bins, 8 keys at a time level by level; the count atomic's old value is
  // the key's slot in its bin's run (any order inside a bucket will do)
  uint32_t meta[kSpKpt];  // bin | slot << 8
#pragma unroll
  for (int i0 = 0; i0 < kSpKpt; i0 += 8) {
    uint32_t m[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) m[j] = 1;
#pragma unroll
    for (int lvl = 0; lvl < LEVELS; ++lvl)
#pragma unroll
      for (int j = 0; j < 8; ++j) m[j] = 2 * m[j] + (k[i0 + j] >= s_t[m[j]] ? 1u : 0u);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int i = i0 + j;
      const uint32_t p = 4 * (threadIdx.x + (i / 4) * kSpThreads) + (i % 4);
      const uint32_t bin = m[j] - BINS;
      meta[i] = p < tile_n ? bin | (atomicAdd(&s_cnt[bin], 1u) << 8) : 0xffffffffu;
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {  // exclusive scan of the bin counts (BINS <= 256)
    uint32_t run = 0;
    for (uint32_t b0 = 0; b0 < BINS; b0 += 32) {
      const uint32_t c = b0 + threadIdx.x < BINS ? s_cnt[b0 + threadIdx.x] : 0u;
      const uint32_t inc = warp_inclusive_scan(c);
      if (b0 + threadIdx.x < BINS) s_start[b0 + threadIdx.x] = run + inc - c;
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
  }
  const uint32_t out0 = (root << LEVELS) - (1u << (root_depth + LEVELS));
  for (uint32_t b = threadIdx.x; b < BINS; b += kSpThreads) {
    const uint32_t c = s_cnt[b];
    s_base[b] = c ? atomicAdd(&cursor[out0 + b], c) : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kSpKpt; ++i) {
    if (meta[i] != 0xffffffffu) {
      const uint32_t bin = meta[i] & 0xffu, q = s_start[bin] + (meta[i] >> 8);
      s_keys[q] = k[i];
      s_bin[q] = uint8_t(bin);
    }
  }
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < tile_n; q += kSpThreads) {
    const uint32_t bin = s_bin[q];
    const uint32_t pos = s_base[bin] + (q - s_start[bin]);
    if (pos < cap) region[size_t(out0 + bin) * cap + pos] = s_keys[q];
  }
}

// 5a. plan (one block): bucket offsets, overflow, and the order the bucket
// sort takes the buckets in: those above one CTA's capacity first (they take
// longest), the rest after them.
__global__ void __launch_bounds__(1024)
    k_bucket_plan(const uint32_t* __restrict__ counts, uint32_t cap,
                  const uint32_t* __restrict__ super_counts, uint32_t scap,
                  uint32_t* __restrict__ offsets, uint32_t* __restrict__ order,
                  LearnedPlan* __restrict__ plan, const uint32_t* __restrict__ mlp_err) {
  pdl_enter();
  if (threadIdx.x == 0) plan->mlp_timeout = *mlp_err;
  __shared__ uint32_t s_warp[33];
  __shared__ uint32_t s_front, s_back;
  constexpr int R = kBuckets / 1024;
  if (threadIdx.x == 0) s_front = s_back = 0;
  const int first = threadIdx.x * R;
  uint32_t v[R], local = 0, mx = 0, big = 0, over = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    v[r] = counts[first + r];
    local += v[r];
    mx = max(mx, v[r]);
    big += v[r] > kBucketCap && v[r] <= cap;
    over |= v[r] > cap;
  }
  if (threadIdx.x < kSupers) over |= super_counts[threadIdx.x] > scap;
  uint32_t total;
  uint32_t run = block_exclusive_scan<1024>(local, s_warp, &total);  // synchronises
#pragma unroll
  for (int r = 0; r < R; ++r) {
    offsets[first + r] = run;
    run += v[r];
    if (v[r] > kBucketCap) order[atomicAdd(&s_front, 1u)] = first + r;
    else order[kBuckets - 1 - atomicAdd(&s_back, 1u)] = first + r;
  }
  if (threadIdx.x == 0) offsets[kBuckets] = total;
  atomicMax(&plan->max_count, mx);
  if (big) atomicAdd(&plan->n_big, big);
  if (over) plan->fallback = 1;
}

// smem of the bucket sort: keys, per-warp counters and match masks, digit
// totals and starts, scan scratch
constexpr int kBsWarps = kBsThreads / 32;
constexpr size_t kBsSmem = (size_t(kBucketCap) + 2 * size_t(kBsWarps) * 256 + 2 * 256 + 64) * 4;

// Counting sort of a bucket whose keys lie in [lo, lo + span), span <= 2^15:
// the sorted keys are fixed by how often each value occurs.  Histogram in
// shared memory (over the key buffer), exclusive scan, then every value is
// written as its run of copies: runs of up to 32 by the thread that owns the
// value, longer runs by a whole warp from a queue.
template <int KPT>
__device__ void bucket_count_sort(const uint32_t (&k)[KPT], int steps, uint32_t wbase,
                                  uint32_t wend, uint32_t lo, uint32_t span, uint32_t cnt,
                                  uint32_t* __restrict__ dst, uint32_t* sm) {
  uint32_t* s_c = sm;                   // [span] counts, then run starts
  uint32_t* s_q = sm + kBucketCap;      // queue of long runs: (value, start, length)
  uint32_t* s_misc = s_q + 3 * 1024;    // [0] queue length, [8..41] warp totals
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t span4 = (span + 3) & ~3u;
  for (uint32_t i = threadIdx.x; i < span4 / 4; i += kBsThreads)
    reinterpret_cast<uint4*>(s_c)[i] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) s_misc[0] = 0;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < KPT; ++i)
    if (i < steps && wbase + 32u * i < wend) atomicAdd(&s_c[k[i] - lo], 1u);
  __syncthreads();
  // exclusive scan of s_c[0, span): warp w scans the counters
  // [w*per, (w+1)*per) 32 at a time, after the totals of the earlier warps
  const uint32_t per = ((span + kBsWarps - 1) / kBsWarps + 31) & ~31u;
  const uint32_t w0 = min(span, warp * per), w1 = min(span, w0 + per);
  uint32_t tot = 0;
  for (uint32_t i = w0 + lane; i < w1; i += 32) tot += s_c[i];
  tot = warp_sum(tot);
  if (lane == 0) s_misc[8 + warp] = tot;
  __syncthreads();
  if (warp == 0) {
    const uint32_t t = s_misc[8 + lane];
    const uint32_t inc = warp_inclusive_scan(t);
    s_misc[8 + lane] = inc - t;
  }
  __syncthreads();
  uint32_t run = s_misc[8 + warp];
  for (uint32_t b0 = w0; b0 < w1; b0 += 32) {
    const uint32_t i = b0 + lane;
    const uint32_t c = i < w1 ? s_c[i] : 0u;
    const uint32_t inc = warp_inclusive_scan(c);
    if (i < w1) s_c[i] = run + inc - c;
    run += __shfl_sync(0xffffffffu, inc, 31);
  }
  __syncthreads();
  // expansion
  for (uint32_t v = threadIdx.x; v < span; v += kBsThreads) {
    const uint32_t o = s_c[v], e = v + 1 < span ? s_c[v + 1] : cnt;
    const uint32_t c = e - o;
    if (c > 32) {
      const uint32_t qi = atomicAdd(&s_misc[0], 1u);
      s_q[3 * qi] = lo + v;
      s_q[3 * qi + 1] = o;
      s_q[3 * qi + 2] = c;
    } else {
      for (uint32_t j = 0; j < c; ++j) dst[o + j] = lo + v;
    }
  }
  __syncthreads();
  const uint32_t nq = s_misc[0];
  for (uint32_t qi = warp; qi < nq; qi += kBsWarps) {
    const uint32_t val = s_q[3 * qi], o = s_q[3 * qi + 1], c = s_q[3 * qi + 2];
    for (uint32_t j = lane; j < c; j += 32) dst[o + j] = val;
  }
}

// A bucket of up to kBucketCap keys: keys in registers (warp w owns
// [w*32*KPT, (w+1)*32*KPT)), one stable LSD pass per 8 spanned bits with the
// onesweep ranking (warp_rank / warp_place), ending in s_keys.
__device__ void bucket_sort_small(const uint32_t* __restrict__ src, uint32_t cnt,
                                  uint32_t* __restrict__ dst, uint32_t* sm) {
  constexpr int KPT = kBsKpt, RADIX = 256;
  uint32_t* s_keys = sm;
  uint32_t* s_hist = s_keys + kBucketCap;
  uint32_t* s_match = s_hist + kBsWarps * RADIX;
  uint32_t* s_cnt = s_match + kBsWarps * RADIX;
  uint32_t* s_start = s_cnt + RADIX;
  uint32_t* s_warp = s_start + RADIX;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  // the bucket spread evenly over the warps: warp w holds [w*per, (w+1)*per)
  // (per a multiple of 32), so every warp runs only `steps` of its KPT steps
  const uint32_t per = ((cnt + kBsWarps - 1) / kBsWarps + 31) & ~31u;
  const int steps = int(per / 32);
  const uint32_t wbase = warp * per + lane;
  const uint32_t wend = min(cnt, (warp + 1) * per);  // end of this warp's keys
  uint32_t k[KPT];
  uint32_t mn = 0xffffffffu, mx = 0;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t idx = wbase + 32u * i;
    const bool v = i < steps && idx < wend;
    k[i] = v ? src[idx] : 0u;
    if (v) {
      mn = min(mn, k[i]);
      mx = max(mx, k[i]);
    }
  }
  // bits the bucket spans: only those below the common prefix are sorted
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
  const uint32_t lo = s_warp[40], hi = s_warp[41];
  const uint32_t diff = lo ^ hi;
  const int bits = diff ? 32 - __clz(diff) : 0;
  if (bits != 0 && hi - lo < kCountSpan) {
    bucket_count_sort(k, steps, wbase, wend, lo, hi - lo + 1, cnt, dst, sm);
    return;
  }
  if (bits == 0) {  // every key equal
#pragma unroll
    for (int i = 0; i < KPT; ++i)
      if (i < steps && wbase + 32u * i < wend) dst[wbase + 32u * i] = k[i];
    return;
  }
  uint32_t* wh = s_hist + warp * RADIX;
  uint32_t* wm = s_match + warp * RADIX;
  uint32_t rank2[RankPack<KPT>::kRegs];
  for (int shift = 0; shift < bits; shift += 8) {
    {
      const uint4 z = make_uint4(0, 0, 0, 0);
      for (int i = threadIdx.x; i < 2 * kBsWarps * RADIX / 4; i += kBsThreads)
        reinterpret_cast<uint4*>(s_hist)[i] = z;
    }
    __syncthreads();
    warp_rank<8, KPT, kRankAtomicOr, false>(k, rank2, shift, wbase, wend, wh, wm, steps);
    __syncthreads();
    if (threadIdx.x < RADIX) {
      uint32_t run = 0;
      for (int w = 0; w < kBsWarps; ++w) {
        const uint32_t c = s_hist[w * RADIX + threadIdx.x];
        s_hist[w * RADIX + threadIdx.x] = run;
        run += c;
      }
      s_cnt[threadIdx.x] = run;
    }
    __syncthreads();
    digit_exclusive_scan<8, kBsThreads>(s_cnt, s_start, s_warp);
    __syncthreads();
    for (int i = threadIdx.x; i < kBsWarps * RADIX; i += kBsThreads)
      s_hist[i] += s_start[i & (RADIX - 1)];
    __syncthreads();
    warp_place<8, KPT, false>(k, rank2, shift, wbase, wend, wh, s_keys, steps);
    __syncthreads();
    if (shift + 8 < bits) {
#pragma unroll
      for (int i = 0; i < KPT; ++i) {
        const uint32_t idx = wbase + 32u * i;
        k[i] = i < steps && idx < wend ? s_keys[idx] : 0u;
      }
    }
  }
  for (uint32_t p = threadIdx.x; p < cnt; p += kBsThreads) dst[p] = s_keys[p];
}

// A bucket above kBucketCap: stable LSD through global memory, ping-ponging
// between the bucket's region `a` and its output range `b`; every pass
// histograms the bucket, then places chunks of kBucketCap keys in order.
__device__ __noinline__ void bucket_sort_big(uint32_t* __restrict__ a, uint32_t cnt, uint32_t* __restrict__ b,
                                uint32_t* sm) {
  constexpr int KPT = kBsKpt, RADIX = 256;
  uint32_t* s_hist = sm + kBucketCap;
  uint32_t* s_match = s_hist + kBsWarps * RADIX;
  uint32_t* s_run = s_match + kBsWarps * RADIX;  // running digit starts across chunks
  uint32_t* s_warp = s_run + 2 * RADIX;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t mn = 0xffffffffu, mx = 0;
  for (uint32_t p = threadIdx.x; p < cnt; p += kBsThreads) {
    mn = min(mn, a[p]);
    mx = max(mx, a[p]);
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
  uint32_t* src = a;
  uint32_t* dst = b;
  uint32_t* wh = s_hist + warp * RADIX;
  uint32_t* wm = s_match + warp * RADIX;
  for (int shift = 0; shift < bits; shift += 8) {
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
      const uint32_t wbase = warp * 32u * KPT + lane;
      uint32_t k[KPT];
      uint32_t rank2[RankPack<KPT>::kRegs];
#pragma unroll
      for (int i = 0; i < KPT; ++i) {
        const uint32_t idx = wbase + 32u * i;
        k[i] = idx < ccount ? src[c0 + idx] : 0u;
      }
      {
        const uint4 z = make_uint4(0, 0, 0, 0);
        for (int i = threadIdx.x; i < 2 * kBsWarps * RADIX / 4; i += kBsThreads)
          reinterpret_cast<uint4*>(s_hist)[i] = z;
      }
      __syncthreads();
      warp_rank<8, KPT, kRankAtomicOr, false>(k, rank2, shift, wbase, ccount, wh, wm);
      __syncthreads();
      // per-warp starts = running start of the digit + earlier warps
      if (threadIdx.x < RADIX) {
        uint32_t run = s_run[threadIdx.x];
        for (int w = 0; w < kBsWarps; ++w) {
          const uint32_t c = s_hist[w * RADIX + threadIdx.x];
          s_hist[w * RADIX + threadIdx.x] = run;
          run += c;
        }
        s_run[threadIdx.x] = run;
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < KPT; ++i) {
        if (wbase + 32u * i < ccount) {
          const uint32_t pos = wh[(k[i] >> shift) & 255u] + RankPack<KPT>::get(rank2, i);
          if (pos < cnt) dst[pos] = k[i];
        }
      }
      __syncthreads();
    }
    uint32_t* t = src;
    src = dst;
    dst = t;
    __threadfence_block();
    __syncthreads();
  }
  if (src != b)
    for (uint32_t p = threadIdx.x; p < cnt; p += kBsThreads) b[p] = src[p];
}

// 5b. one CTA per bucket, in plan order
__global__ void __launch_bounds__(kBsThreads, 1)
    k_bucket_sort(uint32_t* __restrict__ region, uint32_t cap, const uint32_t* __restrict__ counts,
                  const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ order,
                  const LearnedPlan* __restrict__ plan, uint32_t* __restrict__ out) {
  pdl_enter();
  if (plan->fallback) return;  // a region overflowed: the gated onesweep sort writes `out`
  extern __shared__ __align__(16) uint32_t sm[];
  const uint32_t bk = order[blockIdx.x];
  const uint32_t cnt = counts[bk];
  if (cnt == 0 || cnt > cap) return;
  uint32_t* src = region + size_t(bk) * cap;
  uint32_t* dst = out + offsets[bk];
  if (cnt > kBucketCap) bucket_sort_big(src, cnt, dst, sm);
  else bucket_sort_small(src, cnt, dst, sm);
}

}  // namespace rwt

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

struct rw_tree_learned {
  uint32_t n_max = 0;
  uint32_t cap_max = 0;   // bucket region capacity for n_max keys
  uint32_t scap_max = 0;  // super-bucket region capacity for n_max keys
  int num_sms = 148;
  rw_tree_im_storage* sample_im = nullptr;  // onesweep scratch for the sample
  void* d_mem = nullptr;
  uint32_t *d_sample = nullptr, *d_sample_sorted = nullptr, *d_bounds = nullptr,
           *d_cursor = nullptr, *d_offsets = nullptr, *d_order = nullptr, *d_region = nullptr,
           *d_super_cursor = nullptr, *d_super_region = nullptr;
  float* d_params = nullptr;
  float* d_features = nullptr;
  rwt::LearnedPlan* d_plan = nullptr;
  rwt::LearnedPlan* h_plan = nullptr;
  uint32_t* d_mlp_err = nullptr;  // set when a boundary network wait ran out (sticky)
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
  const uint32_t blocks = (rwt::kBounds + 255) / 256;
  if (features) {  // training data (the per-boundary kernel writes the inputs)
    rwt::launch_pdl(rwt::k_boundaries, blocks, 256, 0, s, L->d_sample_sorted, L->group, L->d_bounds,
                                             L->d_features);
    RWL_CUDA(cudaGetLastError());
  }
  if (mlp) {
    const uint32_t ctas = (rwt::kBounds + rwt::kMlpTcRows - 1) / rwt::kMlpTcRows;
    rwt::launch_pdl(rwt::k_boundaries_mlp, ctas, rwt::kMlpTcThreads, 0, s, L->d_sample_sorted,
                    L->d_params, L->group, L->d_bounds, L->d_mlp_err);
    RWL_CUDA(cudaGetLastError());
    rwt::launch_pdl(rwt::k_bounds_monotone, 1, 1024, 0, s, L->d_bounds);
  } else if (!features) {
    rwt::launch_pdl(rwt::k_boundaries, blocks, 256, 0, s, L->d_sample_sorted, L->group, L->d_bounds,
                                             nullptr);
  }
  RWL_CUDA(cudaGetLastError());
  return RW_OK;
}

int front_half(rw_tree_learned* L, const uint32_t* keys, uint32_t n, bool mlp, bool features,
               cudaStream_t s) {
  rwt::launch_pdl(rwt::k_sample, rwt::kSample / 256, 256, 0, s, keys, n, L->d_sample);
  RWL_CUDA(cudaGetLastError());
  if (int rc = sort_sample(L, s)) return rc;
  return boundaries(L, mlp, features, s);
}

// both split passes into the bucket regions, and the plan; the plan is
// copied to the host (not waited for)
int scatter_and_plan(rw_tree_learned* L, const uint32_t* keys, uint32_t n, cudaStream_t s) {
  const uint32_t cap = rwt::region_cap(n), scap = rwt::super_cap(n);
  RWL_CUDA(cudaMemsetAsync(L->d_cursor, 0, 4 * rwt::kBuckets, s));
  RWL_CUDA(cudaMemsetAsync(L->d_super_cursor, 0, 4 * rwt::kSupers, s));
  RWL_CUDA(cudaMemsetAsync(L->d_plan, 0, sizeof(rwt::LearnedPlan), s));
  const uint32_t tiles1 = rwt::div_up(n, rwt::kSpTile);
  rwt::launch_pdl(rwt::k_split<8>, tiles1, rwt::kSpThreads, rwt::SplitCfg<8>::kSmem, s, 
      keys, n, nullptr, 0, tiles1, 1, L->d_bounds, L->d_super_cursor, L->d_super_region, scap);
  RWL_CUDA(cudaGetLastError());
  const uint32_t tps = rwt::div_up(scap, rwt::kSpTile);
  rwt::launch_pdl(rwt::k_split<4>, rwt::kSupers * tps, rwt::kSpThreads, rwt::SplitCfg<4>::kSmem, s, 
      L->d_super_region, 0, L->d_super_cursor, scap, tps, rwt::kSupers, L->d_bounds, L->d_cursor,
      L->d_region, cap);
  RWL_CUDA(cudaGetLastError());
  rwt::launch_pdl(rwt::k_bucket_plan, 1, 1024, 0, s, L->d_cursor, cap, L->d_super_cursor, scap, L->d_offsets,
                                        L->d_order, L->d_plan, L->d_mlp_err);
  RWL_CUDA(cudaGetLastError());
  RWL_CUDA(cudaMemcpyAsync(L->h_plan, L->d_plan, sizeof(rwt::LearnedPlan),
                           cudaMemcpyDeviceToHost, s));
  return RW_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

namespace rwt {

int learned_sort_enqueue(rw_tree_learned* L, const uint32_t* keys, uint32_t* sorted, uint32_t n,
                         int32_t mode, rw_tree_im_storage* fallback_im, bool clear_fallback,
                         cudaStream_t s) {
  if (n < kSample) {  // too few keys to sample: the onesweep sort, known on the host
    // the plan records the fallback, in stream order like a sampled run's
    RWL_CUDA(cudaMemsetAsync(L->d_plan, 0, sizeof(LearnedPlan), s));
    RWL_CUDA(cudaMemsetAsync(&L->d_plan->fallback, 1, 1, s));
    RWL_CUDA(cudaMemcpyAsync(L->h_plan, L->d_plan, sizeof(LearnedPlan), cudaMemcpyDeviceToHost,
                             s));
    return sort_enqueue_gated(fallback_im, keys, sorted, n, nullptr, clear_fallback, s);
  }
  if (int rc = front_half(L, keys, n, mode == RW_LEARNED_MLP, false, s)) return rc;
  if (int rc = scatter_and_plan(L, keys, n, s)) return rc;
  launch_pdl(k_bucket_sort, kBuckets, kBsThreads, kBsSmem, s, L->d_region, region_cap(n),
             L->d_cursor, L->d_offsets, L->d_order, L->d_plan, sorted);
  RWL_CUDA(cudaGetLastError());
  return sort_enqueue_gated(fallback_im, keys, sorted, n, &L->d_plan->fallback, clear_fallback, s);
}

uint32_t learned_capacity(const rw_tree_learned* L) { return L ? L->n_max : 0u; }

void learned_last_stats(const rw_tree_learned* L, rw_tree_learned_stats* out) {
  std::memset(out, 0, sizeof *out);
  out->max_bucket = L->h_plan->max_count;
  out->big_buckets = L->h_plan->n_big;
  out->fell_back = L->h_plan->fallback;
  out->mlp_timeout = L->h_plan->mlp_timeout;
}

}  // namespace rwt

extern "C" {

int rw_tree_learned_create(uint32_t n_max, rw_tree_learned** out) {
  if (!out || n_max < rwt::kSample || n_max >= RW_MAX_POINTS) return RW_ERR_ARG;
  *out = nullptr;
  auto* L = new rw_tree_learned();
  L->n_max = n_max;
  L->cap_max = rwt::region_cap(n_max);
  L->scap_max = rwt::super_cap(n_max);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&L->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (int rc = rw_tree_im_storage_create(rwt::kSample, 32, &L->sample_im)) {
    delete L;
    return rc;
  }
  auto up = [](size_t words) { return (words + 63) & ~size_t(63); };  // 256-byte pieces
  const size_t w_sample = up(rwt::kSample), w_b = up(rwt::kBuckets + 1),
               w_params = up(rwt::kMlpParams), w_feat = up(size_t(rwt::kBounds) * rwt::kMlpIn),
               w_plan = up(sizeof(rwt::LearnedPlan) / 4), w_err = up(1),
               w_region = size_t(rwt::kBuckets) * L->cap_max,
               w_super = size_t(rwt::kSupers) * L->scap_max;
  const size_t words =
      2 * w_sample + 5 * w_b + w_params + w_feat + w_plan + w_err + w_region + w_super;
  cudaError_t e = cudaMalloc(&L->d_mem, 4 * words);
  if (e == cudaSuccess) e = cudaMallocHost(&L->h_plan, sizeof(rwt::LearnedPlan));
  if (e != cudaSuccess) {
    rw_tree_learned_destroy(L);
    return lfail(e, "rw_tree_learned_create");
  }
  uint32_t* p = static_cast<uint32_t*>(L->d_mem);
  L->d_sample = p; p += w_sample;
  L->d_sample_sorted = p; p += w_sample;
  L->d_bounds = p; p += w_b;
  L->d_cursor = p; p += w_b;
  L->d_offsets = p; p += w_b;
  L->d_order = p; p += w_b;
  L->d_super_cursor = p; p += w_b;
  L->d_params = reinterpret_cast<float*>(p); p += w_params;
  L->d_features = reinterpret_cast<float*>(p); p += w_feat;
  L->d_plan = reinterpret_cast<rwt::LearnedPlan*>(p); p += w_plan;
  L->d_mlp_err = p; p += w_err;
  L->d_region = p; p += w_region;
  L->d_super_region = p;
  e = cudaMemset(L->d_mlp_err, 0, 4);
  if (e != cudaSuccess) {
    rw_tree_learned_destroy(L);
    return lfail(e, "rw_tree_learned_create");
  }
  cudaFuncSetAttribute(rwt::k_bucket_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       int(rwt::kBsSmem));
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
  if (!L || !d_keys || !h_counts || n < rwt::kSample || n > L->n_max || !aligned16(d_keys))
    return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = front_half(L, d_keys, n, mode == RW_LEARNED_MLP, false, s)) return rc;
  if (int rc = scatter_and_plan(L, d_keys, n, s)) return rc;
  RWL_CUDA(cudaMemcpyAsync(h_counts, L->d_cursor, 4 * rwt::kBuckets, cudaMemcpyDeviceToHost, s));
  RWL_CUDA(cudaStreamSynchronize(s));
  return RW_OK;
}

int rw_tree_learned_sort(rw_tree_learned* L, const uint32_t* d_keys, uint32_t* d_sorted,
                         uint32_t n, int32_t mode, rw_tree_im_storage* fallback_im,
                         rw_stream_t stream, rw_tree_learned_stats* stats) {
  if (!L || !d_keys || !d_sorted || n > L->n_max || n < 1 || !aligned16(d_keys) ||
      (mode != RW_LEARNED_MLP && mode != RW_LEARNED_SAMPLE_QUANTILES))
    return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (stats) std::memset(stats, 0, sizeof *stats);
  if (!fallback_im) {
    // no scratch for a fallback: the plan is read on the host and an
    // overflow is reported instead of sorted
    if (n < rwt::kSample) return RW_ERR_CAPACITY;
    if (int rc = front_half(L, d_keys, n, mode == RW_LEARNED_MLP, false, s)) return rc;
    if (int rc = scatter_and_plan(L, d_keys, n, s)) return rc;
    RWL_CUDA(cudaStreamSynchronize(s));
    if (stats) rwt::learned_last_stats(L, stats);
    if (L->h_plan->fallback) return RW_ERR_CAPACITY;
    rwt::launch_pdl(rwt::k_bucket_sort, rwt::kBuckets, rwt::kBsThreads, rwt::kBsSmem, s,
        L->d_region, rwt::region_cap(n), L->d_cursor, L->d_offsets, L->d_order, L->d_plan,
        d_sorted);
    RWL_CUDA(cudaGetLastError());
    return RW_OK;
  }
  if (int rc = rwt::learned_sort_enqueue(L, d_keys, d_sorted, n, mode, fallback_im, true, s))
    return rc;
  if (stats) {
    RWL_CUDA(cudaStreamSynchronize(s));
    rwt::learned_last_stats(L, stats);
  }
  return RW_OK;
}

}  // extern "C"
