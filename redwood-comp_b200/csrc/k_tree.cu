// Stages 3-7: unique compaction, Karras radix tree, edge count, exclusive
// scan, octree.
//
// Stage 3 replaces k_FindDups + host std::partial_sum + k_MoveDups
// (apps/tree/cuda/03_unique.cu, cu_dispatcher.cu:597-627) with one kernel:
// ballot head flags, a block scan and a warp-cooperative decoupled look-back.
//
// Stage 4 is process_radix_tree_i of apps/tree/host/func_brt.hpp:45-138,
// one thread per node.  The parent writes are made deterministic (see
// write_node): nodes i >= 1 are the true Karras nodes and each names its
// children once; node 0 (whose range the reference limits to [0, n_brt-1])
// only writes the entries that sequential execution on a zeroed buffer gives.
//
// The fused form computes stages 4 and 5 in one pass: the edge count of node i
// needs prefix_n[parent[i]], and the parent's prefix length is the larger of
// the two boundary deltas of i's key range (the parent splits at one end of
// it; when that split is the global minimum the parent is the root, whose
// prefix_n the reference computes over [0, n_brt-1]), so no second pass over
// parent[] is needed.  Stage 6 stays a separate single-pass scan: chaining it
// to the tree's tiles would make every tile wait for the slowest one.
//
// Stage 7 follows process_oct_node (func_octree.hpp:28-112) in two kernels:
// one writes every octree row in full (corner, cell_size, the chain child and
// zeros elsewhere) from the radix-tree node that owns it, the next adds the
// links from each chain's top node to its parent row with atomicMax/atomicOr.
// Sequential ascending-i execution leaves in every child slot the largest
// value written (node i writes only values in [off[i], off[i]+cnt[i]) and
// these ranges grow with i), and the node mask is an OR, so the result is the
// reference's sequential one.
#include <algorithm>

#include "internal.hpp"
#include "morton.cuh"

namespace rwt {

__device__ __forceinline__ uint32_t count_of(Count c) {
  return c.ptr ? *reinterpret_cast<const volatile uint32_t*>(c.ptr) : c.value;
}

// ---------------------------------------------------------------------------
// stage 3: unique
// ---------------------------------------------------------------------------

template <typename K>
__global__ void __launch_bounds__(kUniqueThreads)
    k_unique(const K* __restrict__ sorted, K* __restrict__ out, uint32_t n,
             uint32_t* __restrict__ desc, uint32_t* __restrict__ tile_ctr,
             DevStatus* __restrict__ st) {
  constexpr int KPT = kUniqueKpt, NW = kUniqueThreads / 32;
  __shared__ uint32_t s_warp[NW + 1];
  __shared__ uint32_t s_tile, s_excl;
  const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  const uint32_t n_tiles = (n + kUniqueTile - 1) / kUniqueTile;
  while (true) {
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= n_tiles) break;
    const uint32_t wbase = tile * kUniqueTile + warp * 32u * KPT;
    K keys[KPT];
    uint32_t heads[KPT];
    K carry = K(0);
    uint32_t count = 0;
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      const uint32_t idx = wbase + 32u * i + lane;
      const K k = idx < n ? sorted[idx] : K(0);
      K left = __shfl_up_sync(0xffffffffu, k, 1);
      if (lane == 0) {
        if (i == 0)
          left = (wbase > 0 && wbase - 1 < n) ? sorted[wbase - 1] : K(~k);
        else
          left = carry;
      }
      carry = __shfl_sync(0xffffffffu, k, 31);
      const bool head = idx < n && (idx == 0 || k != left);
      heads[i] = __ballot_sync(0xffffffffu, head);
      keys[i] = k;
      count += __popc(heads[i]);
    }
    if (lane == 0) s_warp[warp] = count;
    __syncthreads();
    if (warp == 0) {
      const uint32_t c = lane < NW ? s_warp[lane] : 0u;
      const uint32_t inc = warp_inclusive_scan(c);
      if (lane < NW) s_warp[lane] = inc - c;
      const uint32_t total = __shfl_sync(0xffffffffu, inc, NW - 1);
      uint32_t excl = 0;
      if (tile == 0) {
        if (lane == 0) st_relaxed(desc, kFlagInc | (total << 2));
      } else {
        if (lane == 0) st_relaxed(desc + tile, kFlagAgg | (total << 2));
        excl = warp_lookback(desc, tile, st, kSiteUnique);
        if (lane == 0) st_relaxed(desc + tile, kFlagInc | ((excl + total) << 2));
      }
      if (lane == 0) {
        s_excl = excl;
        if (tile == n_tiles - 1) st->n_unique = excl + total;
      }
    }
    __syncthreads();
    uint32_t pos = s_excl + s_warp[warp];
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      const uint32_t dst = pos + __popc(heads[i] & lanemask_lt());
      if (((heads[i] >> lane) & 1u) && dst < n) out[dst] = keys[i];
      pos += __popc(heads[i]);
    }
    __syncthreads();
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

// Key reads of the radix-tree search go through a shared-memory window of the
// tile's keys plus a halo on either side; probes outside it read global memory.
template <typename K>
struct KeyWindow {
  const K* __restrict__ codes;
  const K* win;  // shared memory
  int lo;        // global index of win[0]
  int len;
  __device__ __forceinline__ K operator()(int j) const {
    const int r = j - lo;
    return uint32_t(r) < uint32_t(len) ? win[r] : codes[j];
  }
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

// One CTA per tile of kTreeTile nodes; node base + q*kTreeThreads + tid for
// q < kTreeNpt (striped, so every store instruction of a warp is contiguous).
// With EDGES the kernel also writes edge_count (stages 4 and 5 in one pass);
// tiles are independent, so no CTA ever waits for another.
template <typename K, bool EDGES>
__global__ void __launch_bounds__(kTreeThreads)
    k_radix_tree(const K* __restrict__ codes, Count n_unique_c,
                 uint8_t* __restrict__ prefix_n, uint8_t* __restrict__ hl,
                 uint8_t* __restrict__ hr, int32_t* __restrict__ lc,
                 int32_t* __restrict__ parents, int32_t* __restrict__ edge_count,
                 DevStatus* __restrict__ st) {
  constexpr int NPT = kTreeNpt, HALO = kTreeHalo;
  constexpr int WIN = kTreeTile + 2 * HALO;
  __shared__ K s_win[WIN];
  const uint32_t nu = count_of(n_unique_c);
  if (nu < 3 || nu == RW_COUNT_UNSET) {
    if (blockIdx.x == 0 && threadIdx.x == 0) report_error(st, RW_ERR_DEGENERATE, kSiteTree);
    return;
  }
  const int n = int(nu - 1);
  const int base = int(blockIdx.x) * kTreeTile;
  if (base >= n) return;
  const int wlo = base - HALO;
  for (int j = threadIdx.x; j < WIN; j += kTreeThreads) {
    const int g = wlo + j;
    s_win[j] = (g >= 0 && g <= n) ? codes[g] : K(0);
  }
  __syncthreads();
  const KeyWindow<K> key{codes, s_win, wlo, WIN};
  int root_true_delta = 0, root_prefix = 0;
  if (EDGES) {
    root_true_delta = delta(codes[0], codes[n]);
    root_prefix = delta(codes[0], codes[n - 1]);
  }
#pragma unroll 1
  for (int q = 0; q < NPT; ++q) {
    const int i = base + q * kTreeThreads + int(threadIdx.x);
    if (i >= n) break;
    const BrtNode r = brt_node<K>(i, n, key);
    write_node<K>(i, n, key, r, prefix_n, hl, hr, lc, parents);
    if (EDGES)
      edge_count[i] =
          i > 0 ? fused_edge_count<K>(i, n, key, r, root_true_delta, root_prefix) : 0;
  }
}

// ---------------------------------------------------------------------------
// stage 5: edge count (func_edge.hpp:9-16, 05_edge_count.cu:16-29)
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256)
    k_edge_count(const uint8_t* __restrict__ prefix_n,
                 const int32_t* __restrict__ parents, int32_t* __restrict__ ec,
                 Count n_unique_c) {
  const int n = int(count_of(n_unique_c)) - 1;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int p = parents[i];
    // parents[] holds node indices in [0, n) after stage 4; anything else is a
    // caller error and reads node 0 instead of leaving the buffer
    ec[i] = prefix_n[i] / 3 - prefix_n[uint32_t(p) < uint32_t(n) ? p : 0] / 3;
  }
}

// ---------------------------------------------------------------------------
// stage 6: exclusive scan of the edge counts
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kScanThreads)
    k_edge_scan(const int32_t* __restrict__ ec, int32_t* __restrict__ off,
                Count n_unique_c, uint32_t* __restrict__ desc,
                uint32_t* __restrict__ tile_ctr, DevStatus* __restrict__ st) {
  constexpr int KPT = kScanKpt, NW = kScanThreads / 32;
  __shared__ uint32_t s_warp[NW + 1];
  __shared__ uint32_t s_tile, s_excl;
  const uint32_t n = count_of(n_unique_c) - 1;
  const uint32_t n_tiles = (n + kScanTile - 1) / kScanTile;
  const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  while (true) {
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= n_tiles) break;
    const uint32_t first = tile * kScanTile + tid * KPT;
    int32_t v[KPT];
    uint32_t local = 0;
    if (first + KPT <= n) {
#pragma unroll
      for (int q = 0; q < KPT / 4; ++q) {
        const int4 x = reinterpret_cast<const int4*>(ec + first)[q];
        v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < KPT; ++q) v[q] = first + q < n ? ec[first + q] : 0;
    }
#pragma unroll
    for (int q = 0; q < KPT; ++q) local += uint32_t(v[q]);
    uint32_t total;
    const uint32_t ex = block_exclusive_scan<kScanThreads>(local, s_warp, &total);
    if (warp == 0) {
      uint32_t excl = 0;
      if (tile == 0) {
        if (lane == 0) st_relaxed(desc, kFlagInc | (total << 2));
      } else {
        if (lane == 0) st_relaxed(desc + tile, kFlagAgg | (total << 2));
        excl = warp_lookback(desc, tile, st, kSiteScan);
        if (lane == 0) st_relaxed(desc + tile, kFlagInc | ((excl + total) << 2));
      }
      if (lane == 0) {
        s_excl = excl;
        if (tile == n_tiles - 1) st->n_octree_nodes = excl + total;
      }
    }
    __syncthreads();
    uint32_t run = s_excl + ex;
    if (first + KPT <= n) {
#pragma unroll
      for (int q = 0; q < KPT / 4; ++q) {
        int4 x;
        x.x = int32_t(run); run += uint32_t(v[4 * q]);
        x.y = int32_t(run); run += uint32_t(v[4 * q + 1]);
        x.z = int32_t(run); run += uint32_t(v[4 * q + 2]);
        x.w = int32_t(run); run += uint32_t(v[4 * q + 3]);
        reinterpret_cast<int4*>(off + first)[q] = x;
      }
    } else {
#pragma unroll
      for (int q = 0; q < KPT; ++q) {
        if (first + q < n) off[first + q] = int32_t(run);
        run += uint32_t(v[q]);
      }
    }
    __syncthreads();
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
  uint32_t capacity;
};

// Rows [off[i], off[i] + cnt[i]) belong to radix-tree node i (i >= 1).  Row
// off+k sits at level L - k (L = prefix_n[i] / 3); for k > 0 its one chain
// child is row off+k-1 (func_octree.hpp:56-78).  Node 0 owns no row; its
// thread writes the root initialisation when there is no octree node at all
// (07_octree.cu:188-198) and clears the spare row m that a top link may name.
template <typename K>
__global__ void __launch_bounds__(256)
    k_octree_rows(const K* __restrict__ codes, const uint8_t* __restrict__ prefix_n,
                  const int32_t* __restrict__ ec, const int32_t* __restrict__ off,
                  Count n_unique_c, Count n_oct_c, float min_coord, float range,
                  OctOut o, DevStatus* __restrict__ st) {
  constexpr int B = KeyTraits<K>::kCodeBits;
  const uint32_t nu = count_of(n_unique_c);
  if (nu < 3 || nu == RW_COUNT_UNSET) return;
  const int n = int(nu - 1);
  const uint32_t m = count_of(n_oct_c);
  if (uint64_t(m) + 1 > o.capacity) {
    if (blockIdx.x == 0 && threadIdx.x == 0) report_error(st, RW_ERR_CAPACITY, kSiteOctree);
    return;
  }
  const int root_level = prefix_n[0] / 3;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (i == 0) {
      int4* row = reinterpret_cast<int4*>(o.children + 8 * size_t(m));
      row[0] = make_int4(0, 0, 0, 0);
      row[1] = make_int4(0, 0, 0, 0);
      o.node_mask[m] = 0;
      o.leaf_mask[m] = 0;
      if (m == 0) {
        const K pre = codes[0] >> (B - 3 * root_level);
        o.corner[0] = decode<K>(K(pre << (B - 3 * root_level)), min_coord, range);
        o.cell_size[0] = range;
      }
      continue;
    }
    const int cnt = ec[i];
    if (cnt <= 0) continue;
    const int base = off[i];
    const K code = codes[i];
    const int li = prefix_n[i] / 3;
    for (int k = 0; k < cnt; ++k) {
      const int p = base + k;
      if (uint32_t(p) >= m) break;  // rows of a consistent scan lie below m
      const int level = li - k;
      const K pre = code >> (B - 3 * level);
      o.corner[p] = decode<K>(K(pre << (B - 3 * level)), min_coord, range);
      o.cell_size[p] = __fdiv_rn(range, float(1 << (level - root_level)));
      int32_t child[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      int32_t mask = 0;
      if (k > 0) {
        const int slot = int((code >> (B - 3 * (level + 1))) & K(7));
        child[slot] = p - 1;
        mask = 1 << slot;
      }
      int4* row = reinterpret_cast<int4*>(o.children + 8 * size_t(p));
      row[0] = make_int4(child[0], child[1], child[2], child[3]);
      row[1] = make_int4(child[4], child[5], child[6], child[7]);
      o.node_mask[p] = mask;
      o.leaf_mask[p] = 0;
    }
  }
}

// Link of each chain's top row to the row of the nearest ancestor that owns
// rows (func_octree.hpp:80-111; the walk gives up after 31 steps as there).
template <typename K>
__global__ void __launch_bounds__(256)
    k_octree_links(const K* __restrict__ codes, const uint8_t* __restrict__ prefix_n,
                   const int32_t* __restrict__ parents, const int32_t* __restrict__ ec,
                   const int32_t* __restrict__ off, Count n_unique_c, Count n_oct_c,
                   OctOut o) {
  constexpr int B = KeyTraits<K>::kCodeBits;
  const uint32_t nu = count_of(n_unique_c);
  if (nu < 3 || nu == RW_COUNT_UNSET) return;
  const int n = int(nu - 1);
  const uint32_t m = count_of(n_oct_c);
  if (uint64_t(m) + 1 > o.capacity) return;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x + 1; i < n; i += stride) {
    const int cnt = ec[i];
    if (cnt <= 0) continue;
    int rp = parents[i];
    if (uint32_t(rp) >= uint32_t(n)) continue;
    int counter = 0;
    while (ec[rp] == 0) {
      rp = parents[rp];
      if (uint32_t(rp) >= uint32_t(n)) break;
      if (++counter > 30) break;
    }
    if (uint32_t(rp) >= uint32_t(n)) continue;
    const int oct_parent = off[rp];
    const int top = prefix_n[i] / 3 - cnt + 1;
    const int slot = int((codes[i] >> (B - 3 * top)) & K(7));
    if (uint32_t(oct_parent) < o.capacity) {
      atomicMax(o.children + 8 * size_t(oct_parent) + slot, off[i] + cnt - 1);
      atomicOr(o.node_mask + oct_parent, 1 << slot);
    }
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

namespace {

int persistent_blocks(rw_tree_im_storage* im, int per_sm) {
  return im->num_sms * per_sm;
}

template <typename K>
cudaError_t unique_t(const rw_tree_app_data& app, rw_tree_im_storage* im,
                     cudaStream_t s) {
  const uint32_t tiles = div_up(app.n_input, kUniqueTile);
  const int blocks = std::max(1, std::min<int>(tiles, persistent_blocks(im, 8)));
  k_unique<K><<<blocks, kUniqueThreads, 0, s>>>(
      static_cast<const K*>(app.u_morton_keys_alt), static_cast<K*>(app.u_morton_keys),
      app.n_input, im->d_unique_desc, im->d_tile_ctr + kCtrUnique, im->d_status);
  return cudaGetLastError();
}

template <typename K>
cudaError_t tree_t(const rw_tree_app_data& app, rw_tree_im_storage* im,
                   Count nu, bool edges, cudaStream_t s) {
  const uint32_t tiles = std::max(1u, div_up(app.n_input, kTreeTile));
  const K* codes = static_cast<const K*>(app.u_morton_keys);
  if (edges)
    k_radix_tree<K, true><<<tiles, kTreeThreads, 0, s>>>(
        codes, nu, app.brt_prefix_n, app.brt_has_leaf_left, app.brt_has_leaf_right,
        app.brt_left_child, app.brt_parents, app.u_edge_count, im->d_status);
  else
    k_radix_tree<K, false><<<tiles, kTreeThreads, 0, s>>>(
        codes, nu, app.brt_prefix_n, app.brt_has_leaf_left, app.brt_has_leaf_right,
        app.brt_left_child, app.brt_parents, nullptr, im->d_status);
  return cudaGetLastError();
}

template <typename K>
cudaError_t octree_t(const rw_tree_app_data& app, rw_tree_im_storage* im,
                     Count nu, Count nm, cudaStream_t s, cudaEvent_t* marks) {
  OctOut o{app.oct_children, reinterpret_cast<float4*>(app.oct_corner),
           app.oct_cell_size, app.oct_child_node_mask, app.oct_child_leaf_mask,
           app.oct_capacity};
  const K* codes = static_cast<const K*>(app.u_morton_keys);
  const int blocks = std::max(1, std::min<int>(div_up(app.n_input, 256),
                                               persistent_blocks(im, 8)));
  k_octree_rows<K><<<blocks, 256, 0, s>>>(codes, app.brt_prefix_n, app.u_edge_count,
                                          app.u_edge_offset, nu, nm, app.min_coord,
                                          app.range, o, im->d_status);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (marks) cudaEventRecord(marks[0], s);
  k_octree_links<K><<<blocks, 256, 0, s>>>(codes, app.brt_prefix_n, app.brt_parents,
                                           app.u_edge_count, app.u_edge_offset, nu,
                                           nm, o);
  e = cudaGetLastError();
  if (e == cudaSuccess && marks) cudaEventRecord(marks[1], s);
  return e;
}

}  // namespace

cudaError_t launch_unique(const rw_tree_app_data& app, rw_tree_im_storage* im,
                          cudaStream_t s) {
  return app.key_bits == 32 ? unique_t<uint32_t>(app, im, s)
                            : unique_t<uint64_t>(app, im, s);
}

cudaError_t launch_unique_raw(const void* sorted, void* out, uint32_t n, int key_bits,
                              uint32_t* desc, uint32_t* tile_ctr, DevStatus* status,
                              int num_sms, cudaStream_t s) {
  const uint32_t tiles = div_up(n, kUniqueTile);
  const int blocks = std::max(1, std::min<int>(tiles, num_sms * 8));
  if (key_bits == 32)
    k_unique<uint32_t><<<blocks, kUniqueThreads, 0, s>>>(
        static_cast<const uint32_t*>(sorted), static_cast<uint32_t*>(out), n, desc,
        tile_ctr, status);
  else
    k_unique<uint64_t><<<blocks, kUniqueThreads, 0, s>>>(
        static_cast<const uint64_t*>(sorted), static_cast<uint64_t*>(out), n, desc,
        tile_ctr, status);
  return cudaGetLastError();
}

cudaError_t launch_radix_tree(const rw_tree_app_data& app, rw_tree_im_storage* im,
                              Count nu, bool edges, cudaStream_t s) {
  return app.key_bits == 32 ? tree_t<uint32_t>(app, im, nu, edges, s)
                            : tree_t<uint64_t>(app, im, nu, edges, s);
}

cudaError_t launch_edge_count(const rw_tree_app_data& app, rw_tree_im_storage* im,
                              Count nu, cudaStream_t s) {
  const int blocks = std::max(1, std::min<int>(div_up(app.n_input, 256),
                                               persistent_blocks(im, 8)));
  k_edge_count<<<blocks, 256, 0, s>>>(app.brt_prefix_n, app.brt_parents,
                                      app.u_edge_count, nu);
  return cudaGetLastError();
}

cudaError_t launch_edge_scan(const rw_tree_app_data& app, rw_tree_im_storage* im,
                             Count nu, cudaStream_t s) {
  const uint32_t tiles = div_up(app.n_input, kScanTile);
  const int blocks = std::max(1, std::min<int>(tiles, persistent_blocks(im, 8)));
  k_edge_scan<<<blocks, kScanThreads, 0, s>>>(app.u_edge_count, app.u_edge_offset, nu,
                                              im->d_scan_desc, im->d_tile_ctr + kCtrScan,
                                              im->d_status);
  return cudaGetLastError();
}

cudaError_t launch_octree(const rw_tree_app_data& app, rw_tree_im_storage* im,
                          Count nu, Count nm, cudaStream_t s, cudaEvent_t* marks) {
  return app.key_bits == 32 ? octree_t<uint32_t>(app, im, nu, nm, s, marks)
                            : octree_t<uint64_t>(app, im, nu, nm, s, marks);
}

}  // namespace rwt
