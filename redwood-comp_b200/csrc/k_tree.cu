// Stages 3-7: unique compaction, Karras radix tree, edge count, exclusive
// scan, octree.
//
// Stage 3 replaces k_FindDups + host std::partial_sum + k_MoveDups
// (apps/tree/cuda/03_unique.cu, cu_dispatcher.cu:597-627) with three
// launches: per-tile head counts, one block scanning the tile counts, then a
// compaction of every tile at its scanned offset.
//
// Stage 4 builds the nodes of process_radix_tree_i (apps/tree/host/
// func_brt.hpp:45-138) from nearest smaller values: the radix tree is the
// Cartesian tree of the gap deltas, so each gap's node follows from the
// nearest strictly smaller gap on either side (k_radix_tree; the few gaps
// whose answer lies beyond the tile's window are searched for in the keys by
// the block at its end).  Node 0
// keeps the reference's own search over [0, n_brt-1] (brt_node, write_node);
// nodes i >= 1 are the true Karras nodes and each names its children once, so
// the parent writes are deterministic.
//
// The fused form computes stages 4 and 5 in one pass: the edge count of node i
// needs prefix_n[parent[i]], and the parent's prefix length is the larger of
// the two boundary deltas of i's key range (the parent splits at one end of
// it; when that split is the global minimum the parent is the root, whose
// prefix_n the reference computes over [0, n_brt-1]).
//
// Stage 6 run alone is a reduce, a one-block scan of the tile sums and a
// write.  In the fused pipeline its first two steps run on the octree's tiles
// and the octree kernel scans its own tile's counts on that prefix, writing
// the offsets as it uses them.
//
// Stage 7 follows process_oct_node (func_octree.hpp:28-112) in one pass per
// tile of nodes (k_octree): every row is written once, complete, with the
// links whose target row lies in the tile merged in shared memory; the links
// that leave the tile are applied afterwards with atomicMax/atomicOr
// (k_octree_far_links).  Sequential ascending-i execution leaves in every
// child slot the largest value written (node i writes only values in
// [off[i], off[i]+cnt[i]) and these ranges grow with i), and the node mask is
// an OR, so the result is the reference's sequential one.
#include <algorithm>

#include "internal.hpp"
#include "morton.cuh"

namespace rwt {

// ---------------------------------------------------------------------------
// stage 3: unique
// ---------------------------------------------------------------------------

// Exclusive scan of per-tile values E[0, tiles) in place (E[tiles] = total),
// one block; then each segment's total (its tiles per the tile map) into
// seg_total.  Between the per-tile count and the per-tile write launches of
// stages 3 and 6.
__global__ void __launch_bounds__(1024)
    k_tile_scan(uint32_t* __restrict__ E, uint32_t tiles, SegTable seg, TileMap map,
                uint32_t* __restrict__ seg_total) {
  pdl_enter();
  // rounds of 1,024 x J tiles; warp w scans its contiguous 32 x J slice with
  // coalesced loads (J warp scans with a running carry), then one warp scans
  // the 32 warp sums
  constexpr int J = 16;
  __shared__ uint32_t s_warp[33];
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t carry = 0;
  for (uint32_t c0 = 0; c0 < tiles; c0 += 1024u * J) {
    const uint32_t wb = c0 + warp * 32u * J + lane;
    uint32_t v[J];
#pragma unroll
    for (int j = 0; j < J; ++j) v[j] = wb + 32u * j < tiles ? E[wb + 32u * j] : 0u;
    uint32_t run = 0;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const uint32_t inc = warp_inclusive_scan(v[j]);
      const uint32_t x = v[j];
      v[j] = run + inc - x;  // exclusive within the warp's slice
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) s_warp[warp] = run;
    __syncthreads();
    if (warp == 0) {
      const uint32_t w = s_warp[lane];
      const uint32_t wi = warp_inclusive_scan(w);
      s_warp[lane] = wi - w;
      if (lane == 31) s_warp[32] = wi;
    }
    __syncthreads();
    const uint32_t wofs = carry + s_warp[warp];
#pragma unroll
    for (int j = 0; j < J; ++j)
      if (wb + 32u * j < tiles) E[wb + 32u * j] = wofs + v[j];
    carry += s_warp[32];
    __syncthreads();  // s_warp is reused by the next round
  }
  if (threadIdx.x == 0) E[tiles] = carry;
  __syncthreads();
  for (uint32_t sg = threadIdx.x; sg < seg.count; sg += 1024) {
    const uint32_t t0 = map.toff ? map.toff[sg] : 0u;
    const uint32_t t1 = map.toff ? map.toff[sg + 1] : tiles;
    seg_total[sg] = (t1 < tiles ? E[t1] : carry) - (t0 < tiles ? E[t0] : carry);
  }
}

// Stage 3 in three launches without a serial chain between tiles: (1) every
// tile counts its heads (a key is a head when it differs from its left
// neighbour in the segment, or starts the segment) into E[tile]; (2) one block
// turns E into its exclusive scan (E[tiles] = total) and writes each
// segment's n_unique; (3) every tile compacts its heads to segment begin +
// E[tile] - E[first tile of the segment].  Same result as
// cu_dispatcher.cu:597-627 (a std::unique over the sorted keys).
template <typename K>
__device__ __forceinline__ uint32_t tile_heads(const K* __restrict__ sorted, uint32_t sb,
                                               uint32_t n, uint32_t wbase,
                                               K (&keys)[kUniqueKpt],
                                               uint32_t (&heads)[kUniqueKpt]) {
  const uint32_t lane = lane_id();
  // every load first, so that all of them are in flight together
#pragma unroll
  for (int i = 0; i < kUniqueKpt; ++i) {
    const uint32_t idx = wbase + 32u * i + lane;
    keys[i] = idx < n ? sorted[idx] : K(0);
  }
  const K before = (lane == 0 && wbase > sb && wbase - 1 < n) ? sorted[wbase - 1] : K(0);
  K carry = K(0);
  uint32_t count = 0;
#pragma unroll
  for (int i = 0; i < kUniqueKpt; ++i) {
    const uint32_t idx = wbase + 32u * i + lane;
    const K k = keys[i];
    K left = __shfl_up_sync(0xffffffffu, k, 1);
    if (lane == 0) {
      if (i == 0)
        left = (wbase > sb && wbase - 1 < n) ? before : K(~k);
      else
        left = carry;
    }
    carry = __shfl_sync(0xffffffffu, k, 31);
    const bool head = idx < n && (idx == sb || k != left);
    heads[i] = __ballot_sync(0xffffffffu, head);
    count += __popc(heads[i]);
  }
  return count;
}

// The same head flags for a warp whose 32 * kUniqueKpt keys are all in the
// segment and start on a 16-byte boundary: vector j of lane l holds keys
// wbase + (32 j + l) V + [0, V) (V keys per 16 bytes); hm[j] bit e flags key e
// of that vector.
template <typename K>
struct UniqueVec {
  static constexpr int V = 16 / int(sizeof(K));
  static constexpr int NVEC = int(kUniqueKpt) / V;
};

template <typename K>
__device__ __forceinline__ bool unique_vec_ok(const K* sorted, uint32_t wbase, uint32_t n) {
  return wbase + 32u * kUniqueKpt <= n &&
         (reinterpret_cast<uintptr_t>(sorted + wbase) & 15u) == 0;
}

template <typename K>
__device__ __forceinline__ uint32_t tile_heads_vec(const K* __restrict__ sorted, uint32_t sb,
                                                   uint32_t wbase, K (&keys)[kUniqueKpt],
                                                   uint32_t (&hm)[UniqueVec<K>::NVEC]) {
  constexpr int V = UniqueVec<K>::V, NVEC = UniqueVec<K>::NVEC;
  const uint32_t lane = lane_id();
#pragma unroll
  for (int j = 0; j < NVEC; ++j) {
    const uint4 x = *reinterpret_cast<const uint4*>(sorted + wbase + (32u * j + lane) * V);
    const K* xk = reinterpret_cast<const K*>(&x);
#pragma unroll
    for (int e = 0; e < V; ++e) keys[j * V + e] = xk[e];
  }
  const K before = (lane == 0 && wbase > sb) ? sorted[wbase - 1] : K(0);
  K carry = K(0);
  uint32_t count = 0;
#pragma unroll
  for (int j = 0; j < NVEC; ++j) {
    const K last = keys[j * V + V - 1];
    K up = __shfl_up_sync(0xffffffffu, last, 1);
    if (lane == 0) up = j == 0 ? (wbase > sb ? before : K(~keys[0])) : carry;
    carry = __shfl_sync(0xffffffffu, last, 31);
    uint32_t m = 0;
#pragma unroll
    for (int e = 0; e < V; ++e) {
      const K prev = e == 0 ? up : keys[j * V + e - 1];
      const uint32_t idx = wbase + (32u * j + lane) * V + e;
      m |= uint32_t(idx == sb || keys[j * V + e] != prev) << e;
    }
    hm[j] = m;
    count += __popc(m);
  }
  return count;
}

template <typename K>
__global__ void __launch_bounds__(kUniqueThreads)
    k_unique_count(const K* __restrict__ sorted, SegTable seg, TileMap map,
                   uint32_t* __restrict__ E) {
  pdl_enter();
  constexpr int NW = kUniqueThreads / 32;
  __shared__ uint32_t s_warp[NW];
  const uint32_t tile = blockIdx.x, lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t first;
  const uint32_t c = tile_segment(seg, map, tile, &first);
  const uint32_t sb = seg_begin(seg, c);
  const uint32_t n = sb + seg_size(seg, c);
  const uint32_t wbase = sb + (tile - first) * kUniqueTile + warp * 32u * kUniqueKpt;
  K keys[kUniqueKpt];
  uint32_t count;
  if (unique_vec_ok(sorted, wbase, n)) {
    uint32_t hm[UniqueVec<K>::NVEC];
    count = warp_sum(tile_heads_vec(sorted, sb, wbase, keys, hm));
  } else {
    uint32_t heads[kUniqueKpt];
    count = tile_heads(sorted, sb, n, wbase, keys, heads);
  }
  if (lane == 0) s_warp[warp] = count;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < NW; ++w) t += s_warp[w];
    E[tile] = t;
  }
}

template <typename K>
__global__ void __launch_bounds__(kUniqueThreads)
    k_unique_write(const K* __restrict__ sorted, K* __restrict__ out, SegTable seg, TileMap map,
                   const uint32_t* __restrict__ E) {
  pdl_enter();
  constexpr int NW = kUniqueThreads / 32;
  __shared__ uint32_t s_warp[NW];
  const uint32_t tile = blockIdx.x, lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t first;
  const uint32_t c = tile_segment(seg, map, tile, &first);
  const uint32_t sb = seg_begin(seg, c);
  const uint32_t n = sb + seg_size(seg, c);
  const uint32_t wbase = sb + (tile - first) * kUniqueTile + warp * 32u * kUniqueKpt;
  K keys[kUniqueKpt];
  constexpr int V = UniqueVec<K>::V, NVEC = UniqueVec<K>::NVEC;
  const bool vec = unique_vec_ok(sorted, wbase, n);
  uint32_t heads[kUniqueKpt];  // scalar path: ballots; vector path: hm[j] in heads[j]
  uint32_t count;
  if (vec) {
    uint32_t hm[NVEC];
    count = warp_sum(tile_heads_vec(sorted, sb, wbase, keys, hm));
#pragma unroll
    for (int j = 0; j < NVEC; ++j) heads[j] = hm[j];
  } else {
    count = tile_heads(sorted, sb, n, wbase, keys, heads);
  }
  if (lane == 0) s_warp[warp] = count;
  __syncthreads();
  if (warp == 0) {
    const uint32_t cw = lane < NW ? s_warp[lane] : 0u;
    const uint32_t inc = warp_inclusive_scan(cw);
    if (lane < NW) s_warp[lane] = inc - cw;
  }
  __syncthreads();
  uint32_t pos = sb + (E[tile] - E[first]) + s_warp[warp];
  if (vec) {
#pragma unroll
    for (int j = 0; j < NVEC; ++j) {
      const uint32_t c = uint32_t(__popc(heads[j]));
      const uint32_t inc = warp_inclusive_scan(c);
      uint32_t dst = pos + inc - c;
#pragma unroll
      for (int e = 0; e < V; ++e) {
        if (((heads[j] >> e) & 1u) && dst < n) out[dst] = keys[j * V + e];
        dst += (heads[j] >> e) & 1u;
      }
      pos += __shfl_sync(0xffffffffu, inc, 31);
    }
  } else {
#pragma unroll
    for (int i = 0; i < kUniqueKpt; ++i) {
      const uint32_t dst = pos + __popc(heads[i] & lanemask_lt());
      if (((heads[i] >> lane) & 1u) && dst < n) out[dst] = keys[i];
      pos += __popc(heads[i]);
    }
  }
}

// ---------------------------------------------------------------------------
// stage 4: Karras radix tree node (func_brt.hpp:45-138)
// ---------------------------------------------------------------------------

__device__ __forceinline__ int log2_ceil_u(uint32_t x) {
  const uint32_t lower = 31u - uint32_t(__clz(x));
  return int(lower + ((uint32_t(1) << lower) < x));
}

struct BrtNode {
  int d, j, gamma, dnode;
};

// delta(a, b) > d, for codes whose top bit is clear (the reference asserts it,
// func_brt.hpp:30-31): clz(a ^ b) - 1 > d  <=>  a ^ b < 2^(W - 2 - d).  `lim`
// is that bound (0 when d >= W - 1: never true).
template <typename K>
__device__ __forceinline__ K delta_limit(int d) {
  constexpr int W = KeyTraits<K>::kWordBits;
  return (d >= 0 && d <= W - 2) ? (K(1) << (W - 2 - d)) : K(0);
}

// n = n_brt_nodes; keys live in [0, n].  Same searches as func_brt.hpp:45-138
// (power-of-two divisions written as shifts, delta comparisons as bounds).
template <typename K, typename KeyAt>
__device__ __forceinline__ BrtNode brt_node(int i, int n, const KeyAt& key) {
  const K ci = key(i);
  int d;
  if (i == 0) {
    d = 1;
  } else {
    const int diff = delta(ci, key(i + 1)) - delta(ci, key(i - 1));
    d = (diff > 0) - (diff < 0);
  }
  int l = 0;
  if (i == 0) {
    l = n - 1;
  } else {
    const K lim = delta_limit<K>(delta(ci, key(i - d)));
    int lmax = 2;
    while ((long long)i + (long long)lmax * d >= 0 && i + lmax * d <= n &&
           (ci ^ key(i + lmax * d)) < lim)
      lmax *= 2;
    const int lcut = (d == -1) ? i : n - i;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
      if (l + t <= lcut && (ci ^ key(i + (l + t) * d)) < lim) l += t;
  }
  BrtNode r;
  r.d = d;
  r.j = i + l * d;
  r.dnode = delta(ci, key(r.j));
  const K lim = delta_limit<K>(r.dnode);
  int s = 0;
  const int kmax = log2_ceil_u(uint32_t(l));  // divisor runs 2, 4, .. 2^kmax
  const int scut = (d == -1) ? i - 1 : n - i - 1;
  for (int k = 1; k <= kmax; ++k) {
    const uint32_t t = (uint32_t(l) + (1u << k) - 1u) >> k;
    if (uint32_t(s) + t <= uint32_t(scut) &&
        (ci ^ key(int(uint32_t(i) + (uint32_t(s) + t) * uint32_t(d)))) < lim)
      s += int(t);
  }
  r.gamma = i + s * d + min(d, 0);
  return r;
}

// Writes prefix_n / leaf flags / left_child of node i and its parent links.
// Node 0 writes parents[0] = 0 and a zero for each internal child of the
// true root of [0, n] (the reference's root covers only [0, n-1]; sequential
// execution on a zeroed buffer leaves exactly those entries 0, and no other
// node names them).  Every other entry is written once, by its true parent.
template <typename K, typename KeyAt>
__device__ __forceinline__ void write_node(int i, int n, const KeyAt& key,
                                           const BrtNode& r, uint8_t* prefix_n,
                                           uint8_t* hl, uint8_t* hr, int32_t* lc,
                                           int32_t* parents) {
  prefix_n[i] = uint8_t(r.dnode);
  const int lo = min(i, r.j), hi = max(i, r.j);
  const bool leaf_l = lo == r.gamma, leaf_r = hi == r.gamma + 1;
  hl[i] = leaf_l;
  hr[i] = leaf_r;
  lc[i] = r.gamma;
  if (i > 0) {
    if (!leaf_l) parents[r.gamma] = i;
    if (!leaf_r) parents[r.gamma + 1] = i;
  } else {
    parents[0] = 0;
    const int gamma_true = delta(key(n - 1), key(n)) < r.dnode ? n - 1 : r.gamma;
    if (gamma_true > 0) parents[gamma_true] = 0;
    if (gamma_true + 1 < n) parents[gamma_true + 1] = 0;
  }
}

// Edge count of node i >= 1 without reading parent[] (see file comment).
template <typename K, typename KeyAt>
__device__ __forceinline__ int fused_edge_count(int i, int n, const KeyAt& key,
                                                const BrtNode& r, int root_true_delta,
                                                int root_prefix) {
  const int lo = min(i, r.j), hi = max(i, r.j);
  const int dl = lo > 0 ? delta(key(lo - 1), key(lo)) : -1;
  const int dr = hi < n ? delta(key(hi), key(hi + 1)) : -1;
  const int pd = max(dl, dr);
  const int parent_prefix = pd == root_true_delta ? root_prefix : pd;
  return r.dnode / 3 - parent_prefix / 3;
}

__device__ __forceinline__ void seg_error(int32_t* seg_err, uint32_t c, int32_t code) {
  atomicCAS(reinterpret_cast<int*>(seg_err + c), 0, code);
}

// Key reads of node 0's searches: global memory only.
template <typename K>
struct GlobalKeys {
  const K* __restrict__ codes;
  __device__ __forceinline__ K operator()(int j) const { return codes[j]; }
};

// ---- stages 4 (+5) from nearest smaller values ----------------------------
//
// With D[k] = delta(key k, key k+1) for the n gaps k in [0, n), the binary
// radix tree of the keys is the Cartesian tree of D: the node that splits at
// gap g covers keys [L+1, R], where L < g and R > g are the nearest gaps with
// D strictly smaller than D[g] (-1 and n when there are none); its prefix
// length is D[g]; its parent splits at whichever of L, R has the larger D; and
// its Karras index (the one process_radix_tree_i gives it, func_brt.hpp:45-138)
// is R when it is its parent's left child and L+1 when it is the right child.
// Every node's outputs follow without a search: left_child = g, leaf flags
// g == L+1 and g+1 == R, the internal children's parent links, and the edge
// count from the parent's prefix max(D[L], D[R]).  The root (L = -1, R = n)
// is node 0, which keeps the reference's own computation over [0, n-1]
// (brt_node / write_node above).
//
// L and R per gap: in chunks of 32 gaps (one per lane) a bit-serial warp
// comparison of E = D + 1 (0 marks the walls at -1 and n) gives every lane
// the lanes with a smaller value, hence the nearest smaller in the chunk, and
// every value v the last / first position in the chunk below v.  Across the
// tile and a halo of kAnsvHalo chunks on either side, per-value bitmasks of
// the chunks whose minimum lies below v find the nearest such chunk in one
// clz / ffs, and its summary gives the answer; a gap whose nearest smaller
// lies beyond the halo (a node near the top of the tree) goes to a list in
// shared memory that the block resolves at its end with warp-cooperative
// searches of the keys.
constexpr int kAnsvHalo = 8;                                        // chunks per side
constexpr int kAnsvChunks = int(kTreeTile) / 32 + 2 * kAnsvHalo;   // chunks per window
constexpr int kAnsvWin = kAnsvChunks * 32;                           // gaps per window
constexpr int kAnsvTileChunks = int(kTreeTile) / 32;
constexpr int kAnsvRow = kAnsvTileChunks + 1;  // padded: lane v and chunk c in different banks
constexpr int kAnsvNone = -0x7fffffff;     // "no smaller gap found to the left"
constexpr int kAnsvNoneR = 0x7fffffff;     // "none to the right"

// Last / first position in a chunk of 32 E values (4-byte aligned) whose
// value is below e; the caller knows there is one.
__device__ __forceinline__ int chunk_last_below(const uint8_t* ce, int e) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(ce);
  const uint32_t ev = 0x01010101u * uint32_t(e);
  for (int q = 7; q > 0; --q) {
    const uint32_t below = __vcmpltu4(w[q], ev);  // 0xff in each byte below e
    if (below) return 4 * q + (31 - __clz(below)) / 8;
  }
  return (31 - __clz(__vcmpltu4(w[0], ev))) / 8;
}

__device__ __forceinline__ int chunk_first_below(const uint8_t* ce, int e) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(ce);
  const uint32_t ev = 0x01010101u * uint32_t(e);
  for (int q = 0; q < 7; ++q) {
    const uint32_t below = __vcmpltu4(w[q], ev);
    if (below) return 4 * q + (__ffs(below) - 1) / 8;
  }
  return 28 + (__ffs(__vcmpltu4(w[7], ev)) - 1) / 8;
}

template <typename K>
struct AnsvCfg {
  static constexpr int NV = sizeof(K) == 4 ? 32 : 64;  // values of E
  static constexpr int VB = sizeof(K) == 4 ? 5 : 6;    // bits of E
  static constexpr size_t kKeyBytes = (size_t(kAnsvWin) + 1) * sizeof(K);
  static constexpr int MW = (kAnsvChunks + 31) / 32;  // mask words per value
  static constexpr size_t kSmem = kKeyBytes + size_t(NV) * MW * 4 + 4 * size_t(kTreeTile) +
                                  size_t(kAnsvWin) + 2 * size_t(NV) * kAnsvRow +
                                  size_t(kAnsvChunks);
};

// Warp-cooperative search for the nearest smaller gaps of gap g beyond any
// window, both sides in lockstep: 32 probes per side and round (doubling
// distances, then 32-ary refinement), the two sides' loads issued together,
// so the pair costs about as many dependent loads as the longer side.
// Left: pred(a) = delta(key a, key g) > D is true from some a_min up to g;
// *first_key = a_min (the node's first key).  Right: pred(b) = delta(key g+1,
// key b) > D is true from g+1 up to some b_max <= n; *last_key = b_max.
template <typename K>
__device__ void coop_node_keys(const K* __restrict__ codes, int n, int g, int D,
                               int* first_key, int* last_key) {
  const uint32_t lane = lane_id();
  const K cl = codes[g], cr = codes[g + 1], lim = delta_limit<K>(D);
  const int pl = lane < 31 ? g - (1 << lane) : -1;
  const long long pr = lane < 31 ? (long long)g + 1 + (1ll << lane) : (long long)n + 1;
  const bool fl = pl >= 0 && (codes[pl] ^ cl) < lim;
  const bool fr = pr <= n && (codes[int(pr)] ^ cr) < lim;
  const int jl = __ffs(__ballot_sync(0xffffffffu, !fl)) - 1;  // a false probe exists
  const int jr = __ffs(__ballot_sync(0xffffffffu, !fr)) - 1;
  int llo = max(jl < 31 ? g - (1 << jl) : -1, -1);                // pred(llo) false
  int lhi = jl == 0 ? g : g - (1 << (jl - 1));                    // pred(lhi) true
  int rhi = jr < 31 ? int(min((long long)g + 1 + (1ll << jr), (long long)n + 1)) : n + 1;
  int rlo = jr == 0 ? g + 1 : g + 1 + (1 << (jr - 1));            // pred(rlo) true
  while (lhi - llo > 1 || rhi - rlo > 1) {
    const bool la = lhi - llo > 1, ra = rhi - rlo > 1;  // warp-uniform
    const int ls = la ? (lhi - llo + 31) / 32 : 0, rs = ra ? (rhi - rlo + 31) / 32 : 0;
    const int lq = llo + (int(lane) + 1) * ls, rq = rlo + (int(lane) + 1) * rs;
    const bool lin = la && lane < 31 && lq < lhi, rin = ra && lane < 31 && rq < rhi;
    const bool lt = lin && (codes[lq] ^ cl) < lim;
    const bool rt = rin && (codes[rq] ^ cr) < lim;
    const uint32_t mlt = __ballot_sync(0xffffffffu, lt), mli = __ballot_sync(0xffffffffu, lin);
    const uint32_t mrf = __ballot_sync(0xffffffffu, rin && !rt),
                   mri = __ballot_sync(0xffffffffu, rin);
    if (la) {
      if (mlt) {
        const int ft = __ffs(mlt) - 1;
        lhi = llo + (ft + 1) * ls;
        llo = ft > 0 ? llo + ft * ls : llo;
      } else {
        llo = llo + (32 - __clz(mli)) * ls;  // the last probe in range is false
      }
    }
    if (ra) {
      if (mrf) {
        const int ff = __ffs(mrf) - 1;
        rhi = rlo + (ff + 1) * rs;
        rlo = ff > 0 ? rlo + ff * rs : rlo;
      } else {
        rlo = rlo + (32 - __clz(mri)) * rs;  // every probe in range is true
      }
    }
  }
  *first_key = lhi;
  *last_key = rlo;
}

// Writes the node that splits at gap g, given its nearest smaller gaps L, R
// (see the ANSV comment below); the root (L = -1, R = n) is skipped.
// dl, dr: D of gaps L and R (-1 for the walls at -1 and n).
template <bool EDGES>
__device__ __forceinline__ void write_gap_node_d(int g, int D, int L, int R, int dl, int dr,
                                                 int root_true_delta, int root_prefix,
                                                 uint8_t* pn, uint8_t* l8, uint8_t* r8,
                                                 int32_t* lcs, int32_t* par, int32_t* ec) {
  const int i = dr > dl ? R : L + 1;  // left child of R's node, else right child of L's
  const bool leaf_l = g == L + 1, leaf_r = g + 1 == R;
  pn[i] = uint8_t(D);
  l8[i] = leaf_l;
  r8[i] = leaf_r;
  lcs[i] = g;
  if (!leaf_l) par[g] = i;
  if (!leaf_r) par[g + 1] = i;
  if (EDGES) {
    const int pd = max(dl, dr);
    const int pp = pd == root_true_delta ? root_prefix : pd;
    ec[i] = D / 3 - pp / 3;
  }
}

template <typename K, bool EDGES, typename DAt>
__device__ __forceinline__ void write_gap_node(int g, int n, int D, int L, int R, const DAt& d_at,
                                               int root_true_delta, int root_prefix,
                                               uint8_t* pn, uint8_t* l8, uint8_t* r8,
                                               int32_t* lcs, int32_t* par, int32_t* ec) {
  if (L < 0 && R >= n) return;
  write_gap_node_d<EDGES>(g, D, L, R, L >= 0 ? d_at(L) : -1, R < n ? d_at(R) : -1,
                          root_true_delta, root_prefix, pn, l8, r8, lcs, par, ec);
}

template <typename K, bool EDGES>
__global__ void __launch_bounds__(kTreeThreads, 8)  // 8 blocks (64 warps) per SM
    k_radix_tree(const K* __restrict__ codes_all, SegTable seg, TileMap map,
                 const uint32_t* __restrict__ n_unique, int32_t* __restrict__ seg_err,
                 uint8_t* __restrict__ prefix_n, uint8_t* __restrict__ hl,
                 uint8_t* __restrict__ hr, int32_t* __restrict__ lc,
                 int32_t* __restrict__ parents, int32_t* __restrict__ edge_count) {
  pdl_enter();
  using C = AnsvCfg<K>;
  constexpr int NV = C::NV, VB = C::VB, NW = kTreeThreads / 32;
  static_assert(kTreeFarPerTile >= 2 * uint32_t(NV), "far gaps of a tile: NV per side");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // positions inside a chunk are kept as lane indices (0xff: none)
  K* s_key = reinterpret_cast<K*>(smem_raw);                                   // [kAnsvWin + 1]
  uint32_t* s_mask = reinterpret_cast<uint32_t*>(smem_raw + C::kKeyBytes);     // [NV][MW]
  // the tile's gaps left to phase C: tile index | in-chunk left << 16 |
  // in-chunk right << 24 (lane indices, 0xff: none)
  uint32_t* s_pend = s_mask + NV * C::MW;                                      // [kTreeTile]
  uint8_t* s_e = reinterpret_cast<uint8_t*>(s_pend + kTreeTile);               // [kAnsvWin]
  // summaries of the tile's chunks only (a halo chunk is scanned when asked)
  uint8_t* s_last = s_e + kAnsvWin;                                            // [NV][kAnsvRow]
  uint8_t* s_first = s_last + NV * kAnsvRow;                                   // [NV][kAnsvRow]
  uint8_t* s_cmin = s_first + NV * kAnsvRow;                                   // [kAnsvChunks]

  uint32_t first;
  const uint32_t c = tile_segment(seg, map, blockIdx.x, &first);
  const uint32_t nu = *reinterpret_cast<const volatile uint32_t*>(n_unique + c);
  if (nu < 3 || nu == RW_COUNT_UNSET || nu > seg_size(seg, c)) {
    if (blockIdx.x == first && threadIdx.x == 0) seg_error(seg_err, c, RW_ERR_DEGENERATE);
    return;
  }
  const uint32_t sb = seg_begin(seg, c);
  const K* codes = codes_all + sb;
  const int n = int(nu - 1);  // gaps (= nodes); keys are [0, n]
  const int g0 = int(blockIdx.x - first) * int(kTreeTile);
  if (g0 >= n) return;
  const int wlo = g0 - kAnsvHalo * 32;  // first gap of the window
  uint8_t* pn = prefix_n + sb;
  uint8_t* l8 = hl + sb;
  uint8_t* r8 = hr + sb;
  int32_t* lcs = lc + sb;
  int32_t* par = parents + sb;

  int root_true_delta = 0, root_prefix = 0;
  if (EDGES) {
    root_true_delta = delta(codes[0], codes[n]);
    root_prefix = delta(codes[0], codes[n - 1]);
  }
  if (blockIdx.x == first && threadIdx.x == 0) {  // node 0, the reference's way
    const GlobalKeys<K> gk{codes};
    const BrtNode r = brt_node<K>(0, n, gk);
    write_node<K>(0, n, gk, r, pn, l8, r8, lcs, par);
    if (EDGES) edge_count[sb] = 0;
  }

  __shared__ uint32_t s_far[kTreeFarPerTile];  // the tile's gaps left to phase D
  __shared__ uint32_t s_far_n, s_pend_n;
  if (threadIdx.x == 0) {  // read after the barriers below
    s_far_n = 0;
    s_pend_n = 0;
  }

  // the window's keys [wlo, wlo + kAnsvWin]: one bulk copy when the window
  // lies inside the keys and starts on a 16-byte boundary (every interior
  // tile of a plain run), else key by key with zeros outside [0, n]
  static_assert((size_t(kAnsvWin) * sizeof(K)) % 16 == 0, "bulk copies move 16-byte units");
  __shared__ __align__(8) uint64_t s_bar;
  const bool bulk = wlo >= 0 && wlo + kAnsvWin <= n &&
                    (reinterpret_cast<uintptr_t>(codes + wlo) & 15u) == 0;
  if (bulk) {
    if (threadIdx.x == 0) bulk_barrier_init(&s_bar);
    __syncthreads();
    if (threadIdx.x == 0) {
      bulk_load(s_key, codes + wlo, uint32_t(kAnsvWin * sizeof(K)), &s_bar);
      s_key[kAnsvWin] = codes[wlo + kAnsvWin];
    }
    const bool landed = bulk_wait(&s_bar, kSpinLimit);
    if (__syncthreads_or(!landed)) {  // the whole block gives up together
      // report, and let the copy land before the block's shared memory goes
      if (threadIdx.x == 0) seg_error(seg_err, c, RW_ERR_TIMEOUT);
      bulk_wait(&s_bar, kSpinLimit);
      return;
    }
  } else {
    for (int j = threadIdx.x; j <= kAnsvWin; j += kTreeThreads) {
      const int k = wlo + j;
      s_key[j] = (k >= 0 && k <= n) ? codes[k] : K(0);
    }
  }
  __syncthreads();

  // phase A: per chunk, E, the nearest smaller inside the chunk, and the
  // chunk's summaries (last / first position with E below each value).  A gap
  // of the tile whose nearest smaller gaps on both sides lie in its own chunk
  // (about four in five on uniform keys) writes its node here, with the D of
  // both from its neighbours' lanes; the others go to the list of phase C.
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  static_assert(C::kKeyBytes % 4 == 0, "the masks follow the keys");
  // the halo chunks need only E and their minimum: a lookup that ends in one
  // scans its 32 values (phase C)
  static_assert(2 * kAnsvHalo % NW == 0, "whole rounds of halo chunks");
  for (int hc = int(warp); hc < 2 * kAnsvHalo; hc += NW) {
    const int ch = hc < kAnsvHalo ? hc : hc + kAnsvTileChunks;
    const int w = ch * 32 + int(lane);
    const int g = wlo + w;
    const int e = uint32_t(g) < uint32_t(n) ? KeyTraits<K>::clz(s_key[w] ^ s_key[w + 1]) : 0;
    s_e[w] = uint8_t(e);
    const uint32_t cmin = __reduce_min_sync(0xffffffffu, uint32_t(e));
    if (lane == 0) s_cmin[ch] = uint8_t(cmin);
  }
  // the tile's chunks two at a time per warp, so that their ballot chains
  // interleave
  static_assert(kAnsvTileChunks % (2 * NW) == 0, "whole pairs of chunks per warp");
  // lane v's threshold bits as masks (all ones where v has the bit), the same
  // for every chunk: kept in registers, since the kernel is bound by its
  // integer instructions
  uint32_t mlane[VB];
#pragma unroll
  for (int bt = 0; bt < VB; ++bt) mlane[bt] = 0u - ((lane >> bt) & 1u);
  for (int ch0 = kAnsvHalo + int(warp); ch0 < kAnsvHalo + kAnsvTileChunks; ch0 += 2 * NW) {
    int e[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int ch = ch0 + j * NW;
      const int w = ch * 32 + int(lane);  // window index of this lane's gap
      const int g = wlo + w;
      const bool real = uint32_t(g) < uint32_t(n);
      // distinct keys whose top bit is clear: E = delta + 1 = clz of the xor,
      // at least 1 for a real gap, so 0 marks walls only
      e[j] = real ? KeyTraits<K>::clz(s_key[w] ^ s_key[w + 1]) : 0;
      s_e[w] = uint8_t(e[j]);
      const uint32_t cmin = __reduce_min_sync(0xffffffffu, uint32_t(e[j]));
      if (lane == 0) s_cmin[ch] = uint8_t(cmin);
    }
    // bit-serial comparison of every lane's E against v = lane (and lane + 32
    // for 64-bit keys): lane v ends with the lanes whose E is below v; the
    // lanes below my own value are then lane e's result
    // (branch-free: with m = all ones where v has the bit, a lane stays equal
    // while its bit matches, eq &= ~(B ^ m), and falls below where v has the
    // bit and it has not, lt |= eq & ~B & m)
    uint32_t lt0[2] = {0, 0}, eq0[2] = {0xffffffffu, 0xffffffffu};  // below v = lane
    uint32_t lt1[2] = {0, 0}, eq1[2] = {0xffffffffu, 0xffffffffu};  // below v = lane + 32
#pragma unroll
    for (int bt = VB - 1; bt >= 0; --bt) {
      uint32_t B[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) B[j] = __ballot_sync(0xffffffffu, (e[j] >> bt) & 1);
      // v = lane + 32 has bit 5 set and lane's bits below it
      const uint32_t m0 = mlane[bt], m1 = bt == 5 ? 0xffffffffu : mlane[bt];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        lt0[j] |= eq0[j] & ~B[j] & m0;
        eq0[j] &= ~(B[j] ^ m0);
        if (NV > 32) {
          lt1[j] |= eq1[j] & ~B[j] & m1;
          eq1[j] &= ~(B[j] ^ m1);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int ch = ch0 + j * NW;
      const uint32_t from0 = __shfl_sync(0xffffffffu, lt0[j], e[j] & 31);
      const uint32_t from1 = NV > 32 ? __shfl_sync(0xffffffffu, lt1[j], e[j] & 31) : 0u;
      const uint32_t lt = (NV > 32 && e[j] >= 32) ? from1 : from0;
      {
        const int tg = (ch - kAnsvHalo) * 32 + int(lane);
        // lt never holds the lane itself; clz(0) = 32 and ffs(0) = 0 give -1
        const uint32_t lm = lt & lanemask_lt(), rm = lt & ~lm;
        const int lp = 31 - __clz(lm);
        const int rp = __ffs(rm) - 1;
        // E of the two nearest smaller lanes (a wall lane past the last gap
        // has E = 0, so D = -1 there as for the wall at n)
        const int el = __shfl_sync(0xffffffffu, e[j], lp & 31);
        const int er = __shfl_sync(0xffffffffu, e[j], rp & 31);
        const int g = g0 + tg;
        const bool real = g < n;
        const bool here = real && lp >= 0 && rp >= 0;
        if (here)
          write_gap_node_d<EDGES>(g, e[j] - 1, g - int(lane) + lp, g - int(lane) + rp, el - 1,
                                  er - 1, root_true_delta, root_prefix, pn, l8, r8, lcs, par,
                                  EDGES ? edge_count + sb : nullptr);
        const uint32_t pm = __ballot_sync(0xffffffffu, real && !here);
        if (pm) {
          uint32_t at = 0;
          if (lane == uint32_t(__ffs(pm) - 1)) at = atomicAdd(&s_pend_n, uint32_t(__popc(pm)));
          at = __shfl_sync(0xffffffffu, at, __ffs(pm) - 1) + __popc(pm & lanemask_lt());
          if (real && !here)
            s_pend[at] = uint32_t(tg) | uint32_t(lp & 0xff) << 16 | uint32_t(rp & 0xff) << 24;
        }
      }
      // an empty mask gives 0xff (none) by itself: 31 - clz(0) = ffs(0) - 1 = -1
      const int tc = ch - kAnsvHalo;  // the chunk's column among the tile's
      s_last[int(lane) * kAnsvRow + tc] = uint8_t(31 - __clz(lt0[j]));
      s_first[int(lane) * kAnsvRow + tc] = uint8_t(__ffs(lt0[j]) - 1);
      if (NV > 32) {
        s_last[(int(lane) + 32) * kAnsvRow + tc] = uint8_t(31 - __clz(lt1[j]));
        s_first[(int(lane) + 32) * kAnsvRow + tc] = uint8_t(__ffs(lt1[j]) - 1);
      }
    }
  }
  __syncthreads();

  // phase B: for every value v, a bitmask of the window's chunks whose
  // minimum lies below v (bit c of word c / 32)
  for (int v = int(warp); v < NV; v += NW) {
#pragma unroll
    for (int wd = 0; wd < C::MW; ++wd) {
      const int cidx = wd * 32 + int(lane);
      const uint32_t bits = __ballot_sync(0xffffffffu, cidx < kAnsvChunks && int(s_cmin[cidx]) < v);
      if (lane == 0) s_mask[v * C::MW + wd] = bits;
    }
  }
  __syncthreads();

  // phase C: every gap of the list writes its node; a gap whose nearest
  // smaller gap lies beyond the window goes to the far-search list
  const int wend = wlo + kAnsvWin - 1;  // last gap of the window
  auto d_at = [&](int p) -> int {       // D of gap p in [0, n)
    return (p >= wlo && p <= wend) ? int(s_e[p - wlo]) - 1 : delta(codes[p], codes[p + 1]);
  };
  const int np = int(s_pend_n);
  for (int q = int(threadIdx.x); q < np; q += kTreeThreads) {
    const uint32_t pw = s_pend[q];
    const int tg = int(pw & 0xffffu), lp = int((pw >> 16) & 0xffu), rp = int(pw >> 24);
    const int g = g0 + tg;
    const int ch = kAnsvHalo + tg / 32;
    const int e = s_e[g - wlo];
    // not inside its own chunk: the nearest chunk on that side whose minimum
    // is below e holds the answer in its summary
    const int cb = wlo + ch * 32;  // first gap of this chunk
    int L = lp != 0xff ? cb + lp : kAnsvNone;
    if (L == kAnsvNone) {
      for (int wd = (ch - 1) >> 5; wd >= 0; --wd) {
        uint32_t bits = s_mask[e * C::MW + wd];
        if (wd == (ch - 1) >> 5) bits &= 0xffffffffu >> (31 - ((ch - 1) & 31));
        if (bits) {
          const int c2 = wd * 32 + 31 - __clz(bits);
          L = wlo + c2 * 32 + (c2 >= kAnsvHalo ? int(s_last[e * kAnsvRow + c2 - kAnsvHalo])
                                               : chunk_last_below(s_e + c2 * 32, e));
          break;
        }
      }
    }
    int R = rp != 0xff ? cb + rp : kAnsvNoneR;
    if (R == kAnsvNoneR) {
      for (int wd = (ch + 1) >> 5; wd < C::MW; ++wd) {
        uint32_t bits = s_mask[e * C::MW + wd];
        if (wd == (ch + 1) >> 5) bits &= 0xffffffffu << ((ch + 1) & 31);
        if (bits) {
          const int c2 = wd * 32 + __ffs(bits) - 1;
          R = wlo + c2 * 32 +
              (c2 < kAnsvHalo + kAnsvTileChunks ? int(s_first[e * kAnsvRow + c2 - kAnsvHalo])
                                                : chunk_first_below(s_e + c2 * 32, e));
          break;
        }
      }
    }
    if (L == kAnsvNone || R == kAnsvNoneR) {
      // resolved by this block below.  The list cannot overflow: two gaps
      // whose nearest smaller gap on the left lies beyond the window never
      // share a value (if a < b did, every gap between them would be at least
      // that value, so the keys a+1 .. b would all have the bit at which keys
      // a and a+1 first differ set, while gap b needs key b to have it clear),
      // so the tile holds at most NV such gaps, and NV more on the right
      const uint32_t local = atomicAdd(&s_far_n, 1u);
      if (local < kTreeFarPerTile) s_far[local] = uint32_t(g);
      else seg_error(seg_err, c, RW_ERR_CAPACITY);  // not reachable, see above
      continue;
    }
    write_gap_node<K, EDGES>(g, n, e - 1, max(L, -1), min(R, n), d_at, root_true_delta,
                             root_prefix, pn, l8, r8, lcs, par,
                             EDGES ? edge_count + sb : nullptr);
  }
  __syncthreads();

  // phase D: the tile's gaps whose nearest smaller gap lies beyond the
  // window, one warp per gap (the warp-cooperative search of the keys in
  // global memory); their latency overlaps the other resident blocks' work
  const uint32_t nf = min(s_far_n, kTreeFarPerTile);
  auto d_glob = [&](int p) -> int { return delta(codes[p], codes[p + 1]); };
  for (uint32_t f = warp; f < nf; f += NW) {
    const int g = int(s_far[f]);
    const int D = delta(codes[g], codes[g + 1]);
    int first_key, last_key;
    coop_node_keys<K>(codes, n, g, D, &first_key, &last_key);
    if (lane == 0)
      write_gap_node<K, EDGES>(g, n, D, first_key - 1, last_key, d_glob, root_true_delta,
                               root_prefix, pn, l8, r8, lcs, par,
                               EDGES ? edge_count + sb : nullptr);
  }
}

// ---------------------------------------------------------------------------
// stage 5: edge count (func_edge.hpp:9-16, 05_edge_count.cu:16-29)
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256)
    k_edge_count(const uint8_t* __restrict__ prefix_n, const int32_t* __restrict__ parents,
                 int32_t* __restrict__ ec, SegTable seg, TileMap map,
                 const uint32_t* __restrict__ n_unique) {
  pdl_enter();
  uint32_t first;
  const uint32_t c = tile_segment(seg, map, blockIdx.x, &first);
  const uint32_t nu = n_unique[c];
  if (nu < 3 || nu == RW_COUNT_UNSET || nu > seg_size(seg, c)) return;
  const int n = int(nu - 1);
  const uint32_t sb = seg_begin(seg, c);
  const int base = int(blockIdx.x - first) * kOctTile;
  for (int q = 0; q < kOctNpt; ++q) {
    const int i = base + q * kOctThreads + int(threadIdx.x);
    if (i >= n) break;
    const int p = parents[sb + i];
    // parents[] holds node indices in [0, n) after stage 4; anything else is a
    // caller error and reads node 0 instead of leaving the buffer
    ec[sb + i] = prefix_n[sb + i] / 3 - prefix_n[sb + (uint32_t(p) < uint32_t(n) ? p : 0)] / 3;
  }
}

// ---------------------------------------------------------------------------
// stage 6: exclusive scan of the edge counts
// ---------------------------------------------------------------------------

// Stage 6 in three launches (no serial chain between tiles): (1) every tile
// sums its edge counts into E[tile]; (2) one block scans E (E[tiles] = total)
// and writes each segment's node count; (3) every tile writes its exclusive
// offsets from E[tile] - E[the segment's first tile].
// Tiles past a segment's nodes (the tile map is sized by points) count zero.
__device__ __forceinline__ bool scan_tile(const SegTable& seg, const TileMap& map,
                                          const uint32_t* n_unique, uint32_t tile,
                                          uint32_t* c, uint32_t* firstt, uint32_t* n,
                                          uint32_t* j) {
  *c = tile_segment(seg, map, tile, firstt);
  const uint32_t nu = *reinterpret_cast<const volatile uint32_t*>(n_unique + *c);
  const bool valid = nu >= 3 && nu != RW_COUNT_UNSET && nu <= seg_size(seg, *c);
  *n = valid ? nu - 1 : 0;
  *j = tile - *firstt;
  return *j < (*n + kScanTile - 1) / kScanTile;
}

__device__ __forceinline__ void scan_load(const int32_t* ec, uint32_t first, uint32_t n,
                                          bool vec, int32_t (&v)[kScanKpt]) {
  if (vec) {
#pragma unroll
    for (int q = 0; q < kScanKpt / 4; ++q) {
      const int4 x = reinterpret_cast<const int4*>(ec + first)[q];
      v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < kScanKpt; ++q) v[q] = first + q < n ? ec[first + q] : 0;
  }
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_reduce(const int32_t* __restrict__ ec_all, SegTable seg, TileMap map,
                  const uint32_t* __restrict__ n_unique, uint32_t* __restrict__ E) {
  pdl_enter();
  constexpr int NW = kScanThreads / 32;
  __shared__ uint32_t s_warp[NW];
  const uint32_t tile = blockIdx.x;
  uint32_t c, firstt, n, j;
  uint32_t local = 0;
  if (scan_tile(seg, map, n_unique, tile, &c, &firstt, &n, &j)) {
    const uint32_t sb = seg_begin(seg, c);
    const uint32_t first = j * kScanTile + threadIdx.x * kScanKpt;
    int32_t v[kScanKpt];
    scan_load(ec_all + sb, first, n, first + kScanKpt <= n && (sb & 3u) == 0, v);
#pragma unroll
    for (int q = 0; q < kScanKpt; ++q) local += uint32_t(v[q]);
  }
  local = warp_sum(local);
  if (lane_id() == 0) s_warp[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < NW; ++w) t += s_warp[w];
    E[tile] = t;
  }
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_write(const int32_t* __restrict__ ec_all, int32_t* __restrict__ off_all,
                 SegTable seg, TileMap map, const uint32_t* __restrict__ n_unique,
                 const uint32_t* __restrict__ E) {
  pdl_enter();
  __shared__ uint32_t s_warp[kScanThreads / 32 + 1];
  const uint32_t tile = blockIdx.x;
  uint32_t c, firstt, n, j;
  if (!scan_tile(seg, map, n_unique, tile, &c, &firstt, &n, &j)) return;  // whole CTA
  const uint32_t sb = seg_begin(seg, c);
  const uint32_t first = j * kScanTile + threadIdx.x * kScanKpt;
  const bool vec = first + kScanKpt <= n && (sb & 3u) == 0;
  int32_t v[kScanKpt];
  scan_load(ec_all + sb, first, n, vec, v);
  uint32_t local = 0;
#pragma unroll
  for (int q = 0; q < kScanKpt; ++q) local += uint32_t(v[q]);
  uint32_t total;
  uint32_t run = (E[tile] - E[firstt]) +
                 block_exclusive_scan<kScanThreads>(local, s_warp, &total);
  int32_t* off = off_all + sb;
  if (vec) {
#pragma unroll
    for (int q = 0; q < kScanKpt / 4; ++q) {
      int4 x;
      x.x = int32_t(run); run += uint32_t(v[4 * q]);
      x.y = int32_t(run); run += uint32_t(v[4 * q + 1]);
      x.z = int32_t(run); run += uint32_t(v[4 * q + 2]);
      x.w = int32_t(run); run += uint32_t(v[4 * q + 3]);
      reinterpret_cast<int4*>(off + first)[q] = x;
    }
  } else {
#pragma unroll
    for (int q = 0; q < kScanKpt; ++q) {
      if (first + q < n) off[first + q] = int32_t(run);
      run += uint32_t(v[q]);
    }
  }
}

// ---------------------------------------------------------------------------
// stage 7: octree rows and links (func_octree.hpp:28-112)
// ---------------------------------------------------------------------------

struct OctOut {
  int32_t* children;
  float4* corner;
  float* cell_size;
  int32_t* node_mask;
  int32_t* leaf_mask;
  const uint32_t* oct_off;  // [segments + 1] row offsets; null with one segment
  uint32_t capacity;        // rows with one segment
};

struct OctSeg {
  uint32_t row0, cap, m;
  int n;        // radix-tree nodes
  bool counts;  // the counts are valid (the edge offsets can be made)
  bool ok;      // ... and the octree fits its rows
};

// The segment's octree rows and counts; reports a too small octree.
__device__ __forceinline__ OctSeg oct_segment(const SegTable& seg, const OctOut& o,
                                              const uint32_t* n_unique,
                                              const uint32_t* n_octree, int32_t* seg_err,
                                              uint32_t c, bool report) {
  OctSeg r{};
  const uint32_t nu = *reinterpret_cast<const volatile uint32_t*>(n_unique + c);
  r.ok = nu >= 3 && nu != RW_COUNT_UNSET && nu <= seg_size(seg, c);
  if (!r.ok) return r;
  r.n = int(nu - 1);
  r.m = *reinterpret_cast<const volatile uint32_t*>(n_octree + c);
  r.row0 = o.oct_off ? o.oct_off[c] : 0u;
  r.cap = o.oct_off ? o.oct_off[c + 1] - o.oct_off[c] : o.capacity;
  r.counts = true;
  if (uint64_t(r.m) + 1 > r.cap) {
    if (report) seg_error(seg_err, c, RW_ERR_CAPACITY);
    r.ok = false;
  }
  return r;
}

// Nearest ancestor of node c that owns rows: parents are followed while the
// count is zero, at most 31 steps as in the reference (func_octree.hpp:80-92).
// Returns -1 when a parent index is outside [0, n).
__device__ __forceinline__ int link_parent(const int32_t* __restrict__ parents,
                                           const int32_t* __restrict__ ec, int c, int n) {
  int rp = parents[c];
  if (uint32_t(rp) >= uint32_t(n)) return -1;
  int counter = 0;
  while (ec[rp] == 0) {
    rp = parents[rp];
    if (uint32_t(rp) >= uint32_t(n)) return -1;
    if (++counter > 30) break;
  }
  return rp;
}

// The link of node c (count cnt > 0) into the global rows: child slot of the
// chain's top row (level prefix_n[c] / 3 - cnt + 1) in row offset[rp]
// (func_octree.hpp:94-102).  The reference overwrites in ascending node
// order; the value off[c] + cnt - 1 grows with c, so the maximum is the last
// write.
template <typename K>
__device__ __forceinline__ void link_global(const K* __restrict__ codes,
                                            const uint8_t* __restrict__ prefix_n,
                                            const int32_t* __restrict__ off, int c, int cnt,
                                            int rp, const OctSeg& os, const OctOut& o) {
  constexpr int B = KeyTraits<K>::kCodeBits;
  const int oct_parent = off[rp];
  const int top = prefix_n[c] / 3 - cnt + 1;
  const int slot = int((codes[c] >> (B - 3 * top)) & K(7));
  if (uint32_t(oct_parent) < os.cap) {
    const size_t r = size_t(os.row0) + uint32_t(oct_parent);
    atomicMax(o.children + 8 * r + slot, off[c] + cnt - 1);
    atomicOr(o.node_mask + r, 1 << slot);
  }
}

// A far link (16 bytes): segment, node, kind << 30 | counter << 3 | slot,
// link value.  kFarFromParent: the walk starts at parents[node] (node = the
// linking node); kFarFromStep: node is the last ancestor reached inside the
// tile, count 0, the walk continues at parents[node] with counter + 1;
// kFarFinal: node is the ancestor whose row takes the link.  kFarLocal is
// used inside k_octree only.
constexpr uint32_t kFarFromParent = 0, kFarFromStep = 1, kFarFinal = 2, kFarLocal = 3;

// Stage 7 in one pass over a tile of radix-tree nodes (func_octree.hpp:28-112).
//
// Rows [off[i], off[i] + cnt[i]) belong to node i (i >= 1); the offsets are
// an exclusive scan of non-negative counts, so a tile of nodes owns one
// contiguous run of rows, and the owner of row p is the last node whose
// first row is <= p.  Row off+k sits at level L - k (L = prefix_n[i] / 3);
// for k > 0 its one child is the chain row off+k-1 (func_octree.hpp:56-78).
// A row with k = 0 gets its children only from links: the chain's top row
// p = off[c] + cnt[c] - 1 of node c is named in row off[rp] of c's nearest
// ancestor rp that owns rows (func_octree.hpp:80-111).  When rp lies in the
// tile and owns rows, that row is a k = 0 row of the tile: the link is
// merged in shared memory and every row is written once, complete.  Other
// links go to the far list (node, segment), applied after this kernel with
// global atomics; a list that overflows makes the far kernel apply every
// link again (the atomics are idempotent).
//
// Threads take the tile's rows in turn (row r by thread r mod threads), so
// that every lane has a row; the owner comes from a binary search over the
// tile's first rows.
//
// Node 0 owns no row; tile 0 writes the root initialisation when there is
// no octree row at all (07_octree.cu:188-198) and clears the spare row m
// that a link may name.
//
// With OFFS the offsets are not read but made here (stage 6's write folded
// into stage 7): tile_prefix holds the exclusive scan of every tile's count
// sum (k_node_sums, k_tile_scan), the block scans its tile's counts on top
// of it and writes them to off_all.
template <typename K, bool OFFS>
__global__ void __launch_bounds__(kOctThreads, 8)  // 8 blocks per SM with 32-bit keys
    k_octree(const K* __restrict__ codes_all, const uint8_t* __restrict__ prefix_all,
             const int32_t* __restrict__ parents_all, const int32_t* __restrict__ ec_all,
             int32_t* __restrict__ off_all, const uint32_t* __restrict__ tile_prefix,
             SegTable seg, TileMap map, const uint32_t* __restrict__ n_unique,
             const uint32_t* __restrict__ n_octree, int32_t* __restrict__ seg_err,
             float min_coord, float range, OctOut o, uint32_t* __restrict__ far,
             uint32_t far_cap, uint32_t* __restrict__ far_n) {
  pdl_enter();
  constexpr int B = KeyTraits<K>::kCodeBits;
  constexpr int kTile = int(kOctTile);
  constexpr int kRowCap = kTile;  // rows whose owner is kept
  static_assert(kTile < 0xfff && (kTile & (kTile - 1)) == 0, "12-bit parents, 2^k tile");
  // k = 0 row of each node: child slot values relative to the tile's first
  // row, plus one (0: no child; the nonzero slots are the node mask)
  __shared__ uint4 s_child[kTile];  // 8 x u16
  // first row of each node relative to the tile's first row (a tile's rows
  // number at most kTile times the largest count, 21 levels; 0xffff past the
  // tile's nodes); [kTile]: end of the tile's rows
  __shared__ uint16_t s_off[kTile + 2];
  __shared__ K s_code[kTile];
  // per node: (count class << 12) | tile-relative parent (0xfff: outside);
  // class 0: count 0, 1: count > 0, 2: count < 0
  __shared__ uint16_t s_node[kTile];
  __shared__ uint8_t s_level[kTile];  // prefix_n / 3
  __shared__ uint16_t s_owner[kRowCap];
  __shared__ uint32_t s_wsum[4 * (kOctThreads / 32) + 1];
  static_assert(kTile == 4 * kOctThreads && 4 * (kOctThreads / 32) == 32,
                "four groups of 256 nodes, 32 warp sums");

  uint32_t first;
  const uint32_t c = tile_segment(seg, map, blockIdx.x, &first);
  const OctSeg os = oct_segment(seg, o, n_unique, n_octree, seg_err, c,
                                blockIdx.x == first && threadIdx.x == 0);
  // with OFFS a too small octree still gets its edge offsets (stage 6's
  // output), as when stage 6 runs on its own
  if (OFFS ? !os.counts : !os.ok) return;
  const int n = os.n;
  const int tile0 = int(blockIdx.x - first) * kTile;
  if (tile0 >= n) return;
  const uint32_t sb = seg_begin(seg, c);
  const K* codes = codes_all + sb;
  const uint8_t* prefix_n = prefix_all + sb;
  const int32_t* parents = parents_all + sb;
  const int32_t* ec = ec_all + sb;
  int32_t* off = off_all + sb;
  const uint32_t m = os.m;
  const int tile_end = min(tile0 + kTile, n);
  const int tid = int(threadIdx.x);

  // thread tid: nodes tile0 + tid + 256 q, q < 4 (coalesced loads)
  int ev[4], ov[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int t = tid + q * kOctThreads;
    const int i = tile0 + t;
    const bool valid = i < tile_end;
    ev[q] = valid ? ec[i] : 0;
    const int pa = valid ? parents[i] : -1;
    const int pr = pa >= tile0 && pa < tile_end ? pa - tile0 : 0xfff;
    s_node[t] = uint16_t((ev[q] == 0 ? 0 : ev[q] > 0 ? 1 : 2) << 12 | pr);
    ov[q] = (!OFFS && valid) ? off[i] : 0;
    s_code[t] = valid ? codes[i] : K(0);
    s_level[t] = valid ? uint8_t(prefix_n[i] / 3) : uint8_t(0);
    s_child[t] = make_uint4(0, 0, 0, 0);
  }
  uint32_t rows_end = 0;
  int rbase = 0;  // the tile's first row
  if (OFFS) {
    // exclusive scan of the counts in node order, as stage 6 computes it: a
    // warp scan per group of 32 nodes, then one warp scans the 32 group sums
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t inc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      inc[q] = warp_inclusive_scan(uint32_t(ev[q]));
      if (lane == 31) s_wsum[q * (kOctThreads / 32) + warp] = inc[q];
    }
    __syncthreads();
    if (warp == 0) {
      const uint32_t v = s_wsum[lane];
      const uint32_t wi = warp_inclusive_scan(v);
      s_wsum[lane] = wi - v;
      if (lane == 31) s_wsum[32] = wi;
    }
    __syncthreads();
    const uint32_t base = tile_prefix[blockIdx.x] - tile_prefix[first];
    rbase = int(base);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ov[q] = int32_t(base + s_wsum[q * (kOctThreads / 32) + warp] + inc[q] - uint32_t(ev[q]));
      const int i = tile0 + tid + q * kOctThreads;
      if (i < tile_end) off[i] = ov[q];
    }
    rows_end = base + s_wsum[32];
  } else {
    rbase = off[tile0];
  }
  if (!os.ok) return;  // the whole block: no octree row is written
  // relative rows kept in [0, 0xfffe] (offsets made by stage 6 stay far inside)
  auto rel16 = [&](int v) -> uint16_t { return uint16_t(min(max(v - rbase, 0), 0xfffe)); };
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int t = tid + q * kOctThreads;
    s_off[t] = tile0 + t < tile_end ? rel16(ov[q]) : uint16_t(0xffff);
  }
  if (tid == 0) {
    s_off[kTile] = rel16(OFFS ? int(rows_end) : (tile_end < n ? off[tile_end] : int(m)));
    if (tile0 == 0) {
      const size_t rm = size_t(os.row0) + m;
      int4* row = reinterpret_cast<int4*>(o.children + 8 * rm);
      row[0] = make_int4(0, 0, 0, 0);
      row[1] = make_int4(0, 0, 0, 0);
      o.node_mask[rm] = 0;
      o.leaf_mask[rm] = 0;
      if (m == 0) {
        const int root_level = prefix_n[0] / 3;
        const K pre = codes[0] >> (B - 3 * root_level);
        o.corner[os.row0] = decode<K>(K(pre << (B - 3 * root_level)), min_coord, range);
        o.cell_size[os.row0] = range;
      }
    }
  }
  __syncthreads();
  if (tile_end < tile0 + kTile && tid == 0) s_off[tile_end - tile0] = s_off[kTile];
  __syncthreads();

  const int rend = min(rbase + int(s_off[kTile]), int(m));  // rows [rbase, rend)
  const int root_level = prefix_n[0] / 3;
  auto owner_of = [&](int r) -> int {  // last node whose first row is <= rbase + r
    int t = 0;
#pragma unroll
    for (int step = kTile / 2; step >= 1; step >>= 1)
      if (int(s_off[t + step]) <= r) t += step;
    return t;
  };

  // links, from the chain top rows; the walk of link_parent over the tile's
  // counts and parents.  A walk that leaves the tile, ends on a node without
  // rows or gives up, and a value that does not fit 16 bits, go to the far
  // list with the walk's state (FarLink), where k_octree_far_links finishes
  // the walk in global memory and merges with atomics.  Several links may
  // name one slot (the reference keeps the last, the largest value): the
  // 16-bit maximum is taken with compare-and-swap on the slot's word.
  for (int r = tid; rbase + r < rend; r += kOctThreads) {
    const int p = rbase + r;
    const int t = owner_of(r);
    if (r < kRowCap) s_owner[r] = uint16_t(t);
    if (r != int(s_off[t + 1]) - 1) continue;  // not the top row of its chain
    const int level = int(s_level[t]) - (r - int(s_off[t]));  // the top row's level
    const int slot = int((s_code[t] >> (B - 3 * level)) & K(7));
    int rp = int(s_node[t] & 0xfffu), counter = 0, x = t;
    uint32_t kind = kFarFromParent;
    if (rp != 0xfff) {
      for (;;) {
        const uint32_t w = s_node[rp];
        if (w >> 12) {
          kind = (w >> 12) == 1 ? kFarLocal : kFarFinal;
          break;
        }
        const int nx = int(w & 0xfffu);
        if (nx == 0xfff) {  // the parent lies outside the tile
          kind = kFarFromStep;
          x = rp;
          break;
        }
        rp = nx;
        if (++counter > 30) {
          kind = kFarFinal;
          break;
        }
      }
    }
    if (kind == kFarLocal) {
      bool done = false;
      if (r < 0xffff) {
        uint32_t* wp = reinterpret_cast<uint32_t*>(&s_child[rp]) + (slot >> 1);
        const int sh = 16 * (slot & 1);
        const uint32_t rel = uint32_t(r) + 1u;  // the link value is p itself
        uint32_t cur = *reinterpret_cast<volatile uint32_t*>(wp);
        for (int tries = 0; tries < 64 && !done; ++tries) {  // each failure is another's success
          if (((cur >> sh) & 0xffffu) >= rel) {
            done = true;
          } else {
            const uint32_t nv = (cur & ~(0xffffu << sh)) | (rel << sh);
            const uint32_t prev = atomicCAS(wp, cur, nv);
            done = prev == cur;
            cur = prev;
          }
        }
      }
      if (done) continue;
      kind = kFarFinal;
    }
    const uint32_t at = atomicAdd(far_n, 1u);
    if (at < far_cap) {
      const int node = kind == kFarFinal ? tile0 + rp : tile0 + x;
      reinterpret_cast<uint4*>(far)[at] =
          make_uint4(c, uint32_t(node), kind << 30 | uint32_t(counter) << 3 | uint32_t(slot),
                     uint32_t(p));
    }
  }
  __syncthreads();

  // rows
  for (int r = tid; rbase + r < rend; r += kOctThreads) {
    const int p = rbase + r;
    const int t = r < kRowCap ? int(s_owner[r]) : owner_of(r);
    const size_t rp = size_t(os.row0) + uint32_t(p);
    const int k = r - int(s_off[t]);
    const int level = int(s_level[t]) - k;
    const K code = s_code[t];
    const K pre = code >> (B - 3 * level);
    o.corner[rp] = decode<K>(K(pre << (B - 3 * level)), min_coord, range);
    // range / 2^s, s = level - root_level in [0, 21]: the product with the
    // exact reciprocal 2^-s is the same correctly rounded value
    o.cell_size[rp] =
        __fmul_rn(range, __uint_as_float(uint32_t(127 - (level - root_level)) << 23));
    int4* row = reinterpret_cast<int4*>(o.children + 8 * rp);
    if (k == 0) {
      const uint4 a = s_child[t];
      const uint32_t wv[4] = {a.x, a.y, a.z, a.w};
      int32_t child[8];
      uint32_t mask = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const uint32_t v = (wv[q >> 1] >> (16 * (q & 1))) & 0xffffu;
        child[q] = v ? int32_t(v) - 1 + rbase : 0;
        mask |= uint32_t(v != 0) << q;
      }
      row[0] = make_int4(child[0], child[1], child[2], child[3]);
      row[1] = make_int4(child[4], child[5], child[6], child[7]);
      o.node_mask[rp] = int32_t(mask);
    } else {
      int32_t child[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      const int slot = int((code >> (B - 3 * (level + 1))) & K(7));
      child[slot] = p - 1;
      row[0] = make_int4(child[0], child[1], child[2], child[3]);
      row[1] = make_int4(child[4], child[5], child[6], child[7]);
      o.node_mask[rp] = 1 << slot;
    }
    o.leaf_mask[rp] = 0;
  }
}

// Sum of the edge counts of every tile of kOctTile nodes (the tiles of
// k_octree), for k_tile_scan: stage 6's reduce on the octree's tiles.  A block
// takes four tiles, 64 threads each; thread j of a tile adds the 16-byte
// vectors j, j + 64, j + 128 and j + 192 of it (a sum needs no order, so the
// warps read consecutive vectors).
__global__ void __launch_bounds__(kOctThreads)
    k_node_sums(const int32_t* __restrict__ ec_all, SegTable seg, TileMap map,
                const uint32_t* __restrict__ n_unique, uint32_t* __restrict__ E) {
  pdl_enter();
  constexpr int kVecs = int(kOctTile) / 4 / 64;  // 16-byte vectors per thread
  static_assert(kOctThreads == 256 && kVecs * 4 * 64 == int(kOctTile), "four tiles of 64 threads");
  __shared__ uint32_t s_warp[kOctThreads / 32];
  const uint32_t g = threadIdx.x >> 6;  // tile of this thread's group
  const uint32_t tile = 4 * blockIdx.x + g;
  uint32_t local = 0;
  if (tile < map.n_tiles) {
    uint32_t first;
    const uint32_t c = tile_segment(seg, map, tile, &first);
    const uint32_t nu = *reinterpret_cast<const volatile uint32_t*>(n_unique + c);
    const bool ok = nu >= 3 && nu != RW_COUNT_UNSET && nu <= seg_size(seg, c);
    const int n = ok ? int(nu - 1) : 0;
    const int tb = int(tile - first) * int(kOctTile);
    const int j = int(threadIdx.x & 63u);
    const int32_t* ec = ec_all + seg_begin(seg, c);
    if (tb + int(kOctTile) <= n && (reinterpret_cast<uintptr_t>(ec + tb) & 15u) == 0) {
      int4 x[kVecs];
#pragma unroll
      for (int q = 0; q < kVecs; ++q) x[q] = reinterpret_cast<const int4*>(ec + tb)[q * 64 + j];
#pragma unroll
      for (int q = 0; q < kVecs; ++q)
        local += uint32_t(x[q].x) + uint32_t(x[q].y) + uint32_t(x[q].z) + uint32_t(x[q].w);
    } else {
      for (int q = 0; q < kVecs; ++q)
        for (int e = 0; e < 4; ++e) {
          const int i = tb + (q * 64 + j) * 4 + e;
          if (i < n) local += uint32_t(ec[i]);
        }
    }
  }
  local = warp_sum(local);
  if (lane_id() == 0) s_warp[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x < 4 && 4 * blockIdx.x + threadIdx.x < map.n_tiles)
    E[4 * blockIdx.x + threadIdx.x] = s_warp[2 * threadIdx.x] + s_warp[2 * threadIdx.x + 1];
}

// Links that k_octree left to the far list, with global atomics; when the
// list overflowed, every node's link again (blocks stride over all tiles).
template <typename K>
__global__ void __launch_bounds__(256)
    k_octree_far_links(const K* __restrict__ codes_all, const uint8_t* __restrict__ prefix_all,
                       const int32_t* __restrict__ parents_all,
                       const int32_t* __restrict__ ec_all, const int32_t* __restrict__ off_all,
                       SegTable seg, TileMap map, const uint32_t* __restrict__ n_unique,
                       const uint32_t* __restrict__ n_octree, int32_t* __restrict__ seg_err,
                       OctOut o, const uint32_t* __restrict__ far, uint32_t far_cap,
                       const uint32_t* __restrict__ far_n) {
  pdl_enter();
  const uint32_t count = *far_n;
  if (count <= far_cap) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < count;
         w += gridDim.x * blockDim.x) {
      // the walk is a chain of dependent loads: every step loads the count,
      // the parent and the offset of its node together, and the first step
      // goes out with the segment's counts (k_octree wrote only nodes of the
      // segment, in [0, n), into the list)
      const uint4 f = reinterpret_cast<const uint4*>(far)[w];
      const uint32_t c = f.x, kind = f.z >> 30, slot = f.z & 7u;
      const uint32_t sb = seg_begin(seg, c);
      const int32_t* parents = parents_all + sb;
      const int32_t* ec = ec_all + sb;
      const int32_t* off = off_all + sb;
      int rp = int(f.y);
      const int first = kind != kFarFinal ? parents[rp] : rp;
      const OctSeg os = oct_segment(seg, o, n_unique, n_octree, seg_err, c, false);
      if (!os.ok) continue;
      const int n = os.n;
      int oct_parent;
      if (kind != kFarFinal) {  // the rest of link_parent's walk
        int counter = int((f.z >> 3) & 31u);
        rp = first;
        if (uint32_t(rp) >= uint32_t(n)) continue;
        bool stop = kind == kFarFromStep && ++counter > 30;
        int cnt = ec[rp], par = parents[rp];
        oct_parent = off[rp];
        while (!stop && cnt == 0) {
          rp = par;
          if (uint32_t(rp) >= uint32_t(n)) break;
          stop = ++counter > 30;
          cnt = ec[rp];
          par = parents[rp];
          oct_parent = off[rp];
        }
        if (uint32_t(rp) >= uint32_t(n)) continue;
      } else {
        oct_parent = off[rp];
      }
      if (uint32_t(oct_parent) < os.cap) {
        const size_t r = size_t(os.row0) + uint32_t(oct_parent);
        atomicMax(o.children + 8 * r + slot, int32_t(f.w));
        atomicOr(o.node_mask + r, 1 << slot);
      }
    }
    return;
  }
  for (uint32_t tile = blockIdx.x; tile < map.n_tiles; tile += gridDim.x) {
    uint32_t first;
    const uint32_t c = tile_segment(seg, map, tile, &first);
    const OctSeg os = oct_segment(seg, o, n_unique, n_octree, seg_err, c, false);
    if (!os.ok) continue;
    const uint32_t sb = seg_begin(seg, c);
    const int32_t* ec = ec_all + sb;
    const int base = int(tile - first) * int(kOctTile);
    for (int q = int(threadIdx.x); q < int(kOctTile); q += int(blockDim.x)) {
      const int i = base + q;
      if (i >= os.n) break;
      if (i == 0) continue;
      const int cnt = ec[i];
      if (cnt <= 0) continue;
      const int rp = link_parent(parents_all + sb, ec, i, os.n);
      if (rp < 0) continue;
      link_global<K>(codes_all + sb, prefix_all + sb, off_all + sb, i, cnt, rp, os, o);
    }
  }
}

// ---------------------------------------------------------------------------
// options outside the reference contract (rw_tree_im_storage_set_options)
// ---------------------------------------------------------------------------

// RW_TREE_OPT_GEOMETRIC_DELTA, 32-bit keys: prefix_n[i] -= 1.  The tree's
// shape depends only on comparisons between deltas, so building it with the
// reference's clz - 1 and lowering every prefix by one gives exactly the tree
// of the clz - 2 delta (every node of distinct 30-bit keys has prefix >= 1).
__global__ void __launch_bounds__(256)
    k_prefix_shift(uint8_t* __restrict__ prefix_n, const uint32_t* __restrict__ n_unique) {
  pdl_enter();
  const uint32_t nu = *n_unique;
  if (nu < 3 || nu == RW_COUNT_UNSET) return;
  const uint32_t n = nu - 1;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    prefix_n[i] = uint8_t(prefix_n[i] - 1u);
}

// RW_TREE_OPT_LINK_LEAVES: process_link_leaf (func_octree.hpp:114-163) for
// every radix-tree node, as if run in ascending order after stage 7.  Leaf
// `side` of node i goes to slot (leaf code at level prefix_n[i]/3 + 1) & 7 of
// the bottom octree row of the nearest ancestor-or-self with octree rows.
// The walk stops after 31 steps (the reference CPU walk has no bound and
// never ends at a root without rows; its CUDA left-leaf walk stops there),
// and a negative level shift (32-bit keys, prefix_n = 30) is taken modulo
// the word width, as an x86 build of the reference does.  Returns false when
// the node has no such leaf or the row is out of range.
template <typename K>
__device__ __forceinline__ bool leaf_target(int i, int side, int n, const K* __restrict__ codes,
                                            const uint8_t* __restrict__ pn,
                                            const uint8_t* __restrict__ hl,
                                            const uint8_t* __restrict__ hr,
                                            const int32_t* __restrict__ lc,
                                            const int32_t* __restrict__ par,
                                            const int32_t* __restrict__ ec,
                                            const int32_t* __restrict__ off, uint32_t rows,
                                            uint32_t* slot, int* leaf) {
  if (!(side ? hr[i] : hl[i])) return false;
  constexpr int B = KeyTraits<K>::kCodeBits, W = KeyTraits<K>::kWordBits;
  const int lf = min(max(lc[i] + side, 0), n);  // keys are [0, n]
  const int level = pn[i] / 3 + 1;
  const uint32_t which = uint32_t(codes[lf] >> ((B - 3 * level) & (W - 1))) & 7u;
  int rt = i;
  for (int step = 0; step < 31 && ec[rt] == 0; ++step) {
    const int p = par[rt];
    rt = uint32_t(p) < uint32_t(n) ? p : 0;
  }
  const int bottom = off[rt];
  if (uint32_t(bottom) >= rows) return false;
  *slot = uint32_t(bottom) * 8u + which;
  *leaf = lf;
  return true;
}

// Pass 1: every writer claims its slot with atomicMin of -(2 i + side) - 2,
// so the slot ends holding the claim of the last writer in sequential order
// (claims are negative, the rows' node links are not); set_leaf's clear of
// the leaf-mask bit commutes and is applied here.
template <typename K>
__global__ void __launch_bounds__(256)
    k_leaf_claim(const K* __restrict__ codes, const uint8_t* __restrict__ pn,
                 const uint8_t* __restrict__ hl, const uint8_t* __restrict__ hr,
                 const int32_t* __restrict__ lc, const int32_t* __restrict__ par,
                 const int32_t* __restrict__ ec, const int32_t* __restrict__ off,
                 int32_t* __restrict__ children, int32_t* __restrict__ leaf_mask,
                 const uint32_t* __restrict__ n_unique, uint32_t rows) {
  pdl_enter();
  const uint32_t nu = *n_unique;
  if (nu < 3 || nu == RW_COUNT_UNSET) return;
  const int n = int(nu - 1);
  for (int i = int(blockIdx.x * blockDim.x + threadIdx.x); i < n; i += int(gridDim.x * blockDim.x))
    for (int side = 0; side < 2; ++side) {
      uint32_t slot;
      int leaf;
      if (!leaf_target<K>(i, side, n, codes, pn, hl, hr, lc, par, ec, off, rows, &slot, &leaf))
        continue;
      atomicMin(children + slot, int(-(int64_t(2 * i + side) + 2)));
      atomicAnd(leaf_mask + slot / 8u, ~(1 << (slot & 7u)));
    }
}

// Pass 2: the writer whose claim survived stores its leaf index.
template <typename K>
__global__ void __launch_bounds__(256)
    k_leaf_write(const K* __restrict__ codes, const uint8_t* __restrict__ pn,
                 const uint8_t* __restrict__ hl, const uint8_t* __restrict__ hr,
                 const int32_t* __restrict__ lc, const int32_t* __restrict__ par,
                 const int32_t* __restrict__ ec, const int32_t* __restrict__ off,
                 int32_t* __restrict__ children, const uint32_t* __restrict__ n_unique,
                 uint32_t rows) {
  pdl_enter();
  const uint32_t nu = *n_unique;
  if (nu < 3 || nu == RW_COUNT_UNSET) return;
  const int n = int(nu - 1);
  for (int i = int(blockIdx.x * blockDim.x + threadIdx.x); i < n; i += int(gridDim.x * blockDim.x))
    for (int side = 0; side < 2; ++side) {
      uint32_t slot;
      int leaf;
      if (!leaf_target<K>(i, side, n, codes, pn, hl, hr, lc, par, ec, off, rows, &slot, &leaf))
        continue;
      // a loser reads the winner's claim or its leaf index, never its own claim
      if (children[slot] == int(-(int64_t(2 * i + side) + 2))) children[slot] = leaf;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

namespace {


template <typename K>
cudaError_t unique_t(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s) {
  const uint32_t tiles = pl.unique_map.n_tiles;
  if (!tiles) return cudaSuccess;
  const K* sorted = static_cast<const K*>(b.alt);
  launch_pdl(k_unique_count<K>, tiles, kUniqueThreads, 0, s, sorted, pl.seg, pl.unique_map,
                                                     sc.unique_desc);
  launch_pdl(k_tile_scan, 1, 1024, 0, s, sc.unique_desc, tiles, pl.seg, pl.unique_map, pl.n_unique);
  launch_pdl(k_unique_write<K>, tiles, kUniqueThreads, 0, s, sorted, static_cast<K*>(b.keys), pl.seg,
                                                     pl.unique_map, sc.unique_desc);
  return cudaGetLastError();
}

template <typename K>
cudaError_t tree_t(const Bufs& b, const Scratch& sc, const Plan& pl, bool edges,
                   cudaStream_t s) {
  const uint32_t tiles = pl.tree_map.n_tiles;
  if (!tiles) return cudaSuccess;
  const K* codes = static_cast<const K*>(b.keys);
  constexpr size_t smem = AnsvCfg<K>::kSmem;
  const auto kern = edges ? k_radix_tree<K, true> : k_radix_tree<K, false>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  // eight blocks of 32-bit keys need nearly all of the SM's shared memory
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             int(cudaSharedmemCarveoutMaxShared));
  if (e != cudaSuccess) return e;
  if (edges)
    launch_pdl(k_radix_tree<K, true>, tiles, kTreeThreads, smem, s, codes, pl.seg, pl.tree_map,
               pl.n_unique, pl.seg_err, b.prefix_n, b.hl, b.hr, b.lc, b.parents, b.edge_count);
  else
    launch_pdl(k_radix_tree<K, false>, tiles, kTreeThreads, smem, s, codes, pl.seg, pl.tree_map,
               pl.n_unique, pl.seg_err, b.prefix_n, b.hl, b.hr, b.lc, b.parents,
               static_cast<int32_t*>(nullptr));
  return cudaGetLastError();
}

template <typename K>
cudaError_t octree_t(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s,
                     cudaEvent_t* marks, bool fused_offsets) {
  OctOut o{b.children, b.corner, b.cell_size, b.node_mask, b.leaf_mask, pl.oct_off,
           pl.oct_capacity};
  const K* codes = static_cast<const K*>(b.keys);
  const uint32_t tiles = pl.node_map.n_tiles;
  uint32_t* far_n = sc.tile_ctr + kCtrLinks;
  // the fused pipeline clears every counter when it starts; stage 7 run alone
  // clears its own (a memset between two kernels would also end the
  // programmatic launch chain)
  cudaError_t e = fused_offsets ? cudaSuccess : cudaMemsetAsync(far_n, 0, sizeof(uint32_t), s);
  // eight blocks of 32-bit keys need nearly all of the SM's shared memory
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fused_offsets ? k_octree<K, true> : k_octree<K, false>,
                             cudaFuncAttributePreferredSharedMemoryCarveout,
                             int(cudaSharedmemCarveoutMaxShared));
  if (e != cudaSuccess) return e;
  if (tiles) {
    if (fused_offsets)
      launch_pdl(k_octree<K, true>, tiles, kOctThreads, 0, s, 
          codes, b.prefix_n, b.parents, b.edge_count, b.edge_offset, sc.scan_desc, pl.seg,
          pl.node_map, pl.n_unique, pl.n_octree, pl.seg_err, b.min_coord, b.range, o,
          sc.tree_far, sc.tree_far_cap, far_n);
    else
      launch_pdl(k_octree<K, false>, tiles, kOctThreads, 0, s, 
          codes, b.prefix_n, b.parents, b.edge_count, b.edge_offset, nullptr, pl.seg,
          pl.node_map, pl.n_unique, pl.n_octree, pl.seg_err, b.min_coord, b.range, o,
          sc.tree_far, sc.tree_far_cap, far_n);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (marks) cudaEventRecord(marks[0], s);
  if (tiles)
    launch_pdl(k_octree_far_links<K>, std::max(1, sc.num_sms * 8), 256, 0, s, 
        codes, b.prefix_n, b.parents, b.edge_count, b.edge_offset, pl.seg, pl.node_map,
        pl.n_unique, pl.n_octree, pl.seg_err, o, sc.tree_far, sc.tree_far_cap, far_n);
  e = cudaGetLastError();
  if (e == cudaSuccess && marks) cudaEventRecord(marks[1], s);
  return e;
}

}  // namespace

cudaError_t launch_unique(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s) {
  return b.key_bits == 32 ? unique_t<uint32_t>(b, sc, pl, s) : unique_t<uint64_t>(b, sc, pl, s);
}

cudaError_t launch_prefix_shift(const Bufs& b, const Scratch& sc, const Plan& pl,
                                cudaStream_t s) {
  if (pl.seg.count != 1) return cudaErrorInvalidValue;
  launch_pdl(k_prefix_shift, std::max(1, sc.num_sms * 4), 256, 0, s, b.prefix_n, pl.n_unique);
  return cudaGetLastError();
}

namespace {
template <typename K>
cudaError_t leaf_links_t(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s) {
  const K* codes = static_cast<const K*>(b.keys);
  const int grid = std::max(1, sc.num_sms * 4);
  launch_pdl(k_leaf_claim<K>, grid, 256, 0, s, codes, b.prefix_n, b.hl, b.hr, b.lc, b.parents,
             b.edge_count, b.edge_offset, b.children, b.leaf_mask, pl.n_unique,
             pl.oct_capacity);
  launch_pdl(k_leaf_write<K>, grid, 256, 0, s, codes, b.prefix_n, b.hl, b.hr, b.lc, b.parents,
             b.edge_count, b.edge_offset, b.children, pl.n_unique, pl.oct_capacity);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_leaf_links(const Bufs& b, const Scratch& sc, const Plan& pl,
                              cudaStream_t s) {
  if (pl.seg.count != 1) return cudaErrorInvalidValue;
  return b.key_bits == 32 ? leaf_links_t<uint32_t>(b, sc, pl, s)
                          : leaf_links_t<uint64_t>(b, sc, pl, s);
}

cudaError_t launch_unique_raw(const void* sorted, void* out, uint32_t n, int key_bits,
                              uint32_t* counts, DevStatus* status, int num_sms,
                              cudaStream_t s) {
  Bufs b;
  b.key_bits = key_bits;
  b.alt = const_cast<void*>(sorted);
  b.keys = out;
  Scratch sc;
  sc.num_sms = num_sms;
  sc.unique_desc = counts;
  sc.status = status;
  const Plan pl = single_plan(n, 0, status, 0);
  return launch_unique(b, sc, pl, s);
}

cudaError_t launch_radix_tree(const Bufs& b, const Scratch& sc, const Plan& pl, bool edges,
                              cudaStream_t s) {
  return b.key_bits == 32 ? tree_t<uint32_t>(b, sc, pl, edges, s)
                          : tree_t<uint64_t>(b, sc, pl, edges, s);
}

cudaError_t launch_edge_count(const Bufs& b, const Scratch& sc, const Plan& pl,
                              cudaStream_t s) {
  (void)sc;
  if (!pl.node_map.n_tiles) return cudaSuccess;
  launch_pdl(k_edge_count, pl.node_map.n_tiles, kOctThreads, 0, s, 
      b.prefix_n, b.parents, b.edge_count, pl.seg, pl.node_map, pl.n_unique);
  return cudaGetLastError();
}

cudaError_t launch_edge_scan(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s) {
  const uint32_t tiles = pl.scan_map.n_tiles;
  if (!tiles) return cudaSuccess;
  launch_pdl(k_scan_reduce, tiles, kScanThreads, 0, s, b.edge_count, pl.seg, pl.scan_map, pl.n_unique,
                                               sc.scan_desc);
  launch_pdl(k_tile_scan, 1, 1024, 0, s, sc.scan_desc, tiles, pl.seg, pl.scan_map, pl.n_octree);
  launch_pdl(k_scan_write, tiles, kScanThreads, 0, s, b.edge_count, b.edge_offset, pl.seg,
                                              pl.scan_map, pl.n_unique, sc.scan_desc);
  return cudaGetLastError();
}

cudaError_t launch_edge_sums(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s) {
  const uint32_t tiles = pl.node_map.n_tiles;
  if (!tiles) return cudaSuccess;
  launch_pdl(k_node_sums, div_up(tiles, 4), kOctThreads, 0, s, b.edge_count, pl.seg, pl.node_map,
                                                      pl.n_unique, sc.scan_desc);
  launch_pdl(k_tile_scan, 1, 1024, 0, s, sc.scan_desc, tiles, pl.seg, pl.node_map, pl.n_octree);
  return cudaGetLastError();
}

cudaError_t launch_octree(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s,
                          cudaEvent_t* marks, bool fused_offsets) {
  return b.key_bits == 32 ? octree_t<uint32_t>(b, sc, pl, s, marks, fused_offsets)
                          : octree_t<uint64_t>(b, sc, pl, s, marks, fused_offsets);
}

Plan single_plan(uint32_t n, uint32_t oct_capacity, DevStatus* status, uint32_t sort_tile) {
  Plan pl;
  pl.seg = SegTable{1u, n, nullptr};
  pl.point_map = TileMap{div_up(n, kPointTile), nullptr};
  pl.sort_map = TileMap{sort_tile ? div_up(n, sort_tile) : 0u, nullptr};
  pl.unique_map = TileMap{div_up(n, kUniqueTile), nullptr};
  pl.tree_map = TileMap{div_up(n, kTreeTile), nullptr};
  pl.scan_map = TileMap{div_up(n, kScanTile), nullptr};
  pl.node_map = TileMap{div_up(n, kOctTile), nullptr};
  pl.n_unique = &status->n_unique;
  pl.n_octree = &status->n_octree_nodes;
  pl.seg_err = &status->err;
  pl.oct_off = nullptr;
  pl.oct_capacity = oct_capacity;
  return pl;
}

}  // namespace rwt
