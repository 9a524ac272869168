// Host-side internals shared by the kernel translation units and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "common.cuh"
#include "rw_tree.h"

// Scratch for one pipeline instance (the reference's cuda::ImStorage,
// apps/tree/cuda/im_storage.cuh:10-42, with the look-back state this design
// needs).  The "zero region" is one allocation cleared before every run.
struct rw_tree_im_storage {
  uint32_t n_cap = 0;   // largest n_input this scratch serves
  int32_t key_bits = 32;
  int device = 0;
  int num_sms = 148;

  // sort configuration (radix bits, passes, tile) fixed at creation
  int radix_bits = 8;
  int passes = 4;
  int sort_variant = 0;      // index into the onesweep variant menu (k_keys.cu)
  uint32_t sort_tile = 0;
  uint32_t sort_tiles = 0;  // tiles per pass at n_cap

  void* d_tmp_keys = nullptr;  // [n_cap] ping-pong buffer of the sort
  uint32_t* d_tree_far = nullptr;  // far links of the octree
  uint32_t tree_far_cap = 0;       // entries (16 bytes each)

  // zero region
  void* d_zero = nullptr;
  size_t zero_bytes = 0;
  uint32_t* d_ghist = nullptr;      // [passes][radix]
  uint32_t* d_skew = nullptr;       // [1]: the top sort pass's digits are skewed
  uint32_t* d_sort_desc = nullptr;  // [passes][sort_tiles + 1][radix]
  uint32_t* d_unique_desc = nullptr;
  uint32_t* d_scan_desc = nullptr;
  uint32_t* d_tile_ctr = nullptr;   // [kCounters]
  rwt::DevStatus* d_status = nullptr;
  size_t sort_zero_off = 0, sort_zero_bytes = 0;  // ghist + sort_desc

  rwt::DevStatus* h_status = nullptr;  // pinned mirror

  // optional learned-CDF sort for stage 2 (32-bit keys); not owned
  rw_tree_learned* learned = nullptr;
  int32_t learned_mode = 0;
  rw_tree_learned_stats learned_stats{};

  // RW_TREE_OPT_* bits (0: the reference's own behaviour)
  int32_t options = 0;
};

namespace rwt {

enum : int { kCtrUnique = 0, kCtrScan = 1, kCtrTree = 2, kCtrLinks = 3, kCtrSortBase = 4,
             kCtrSortClassStride = 8, kMaxSortClasses = 4, kCounters = 64 };

// Tile sizes of the kernels (points or nodes per tile).
constexpr uint32_t kPointTile = 4096;  // Morton / histogram
constexpr uint32_t kUniqueThreads = 256, kUniqueKpt = 16;
constexpr uint32_t kUniqueTile = kUniqueThreads * kUniqueKpt;
constexpr uint32_t kScanThreads = 256, kScanKpt = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanKpt;
constexpr int kTreeThreads = 256;
constexpr uint32_t kTreeTile = 2048;  // radix-tree nodes (key gaps) per tile
constexpr int kOctThreads = 256, kOctNpt = 4;
constexpr uint32_t kOctTile = kOctThreads * kOctNpt;

// Boundary MLP of the learned sort: kMlpIn -> kMlpHidden -> kMlpHidden -> 1.
constexpr int kMlpIn = 16, kMlpHidden = 64;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden +
                           kMlpHidden + kMlpHidden + 1;

inline uint32_t div_up(uint64_t a, uint64_t b) { return uint32_t((a + b - 1) / b); }

// A count either known on the host (value) or produced on the device (ptr).
struct Count {
  const uint32_t* ptr;
  uint32_t value;
};

// Device buffers of one pipeline run: one AppData, or a batch of clouds
// stored back to back (octree rows at per-cloud row offsets).
struct Bufs {
  int key_bits = 32;
  float min_coord = 0.0f, range = 1024.0f;
  const float4* points = nullptr;
  void* keys = nullptr;
  void* alt = nullptr;
  void* tmp = nullptr;  // ping-pong buffer of the sort
  uint8_t* prefix_n = nullptr;
  uint8_t* hl = nullptr;
  uint8_t* hr = nullptr;
  int32_t* lc = nullptr;
  int32_t* parents = nullptr;
  int32_t* edge_count = nullptr;
  int32_t* edge_offset = nullptr;
  int32_t* children = nullptr;
  float4* corner = nullptr;
  float* cell_size = nullptr;
  int32_t* node_mask = nullptr;
  int32_t* leaf_mask = nullptr;
};

// Scratch: histograms, descriptors, tickets, status.
struct Scratch {
  int num_sms = 148;
  int radix_bits = 8;
  int passes = 4;
  int sort_variant = 0;
  uint32_t* ghist = nullptr;      // [segments][passes][radix]
  // [segments]: 1 when the segment's top-pass digits are skewed enough that
  // ballots rank them faster than shared-memory atomics (k_sort_init sets it,
  // the kRankMixed variants read it)
  uint32_t* skew = nullptr;
  uint32_t* sort_desc = nullptr;  // [passes][sort_rows][radix]
  uint32_t sort_rows = 0;         // rows per pass: sort tiles + segments
  uint32_t* unique_desc = nullptr;
  uint32_t* scan_desc = nullptr;
  uint32_t* tile_ctr = nullptr;
  DevStatus* status = nullptr;
  // polls of a look-back wait before it gives up with RW_ERR_TIMEOUT
  uint32_t spin_limit = kSpinLimit;
  // when set, the sort's kernels (digit histograms, set-up, passes) do their
  // work only if *gate != 0, read on the device: a fallback sort enqueued
  // ahead of the decision that needs it
  const uint32_t* gate = nullptr;
  // tree_far_cap entries of 16 bytes: the octree's far links
  uint32_t* tree_far = nullptr;
  uint32_t tree_far_cap = 0;
};

// Entries of the radix tree's far-search list per tile: the gaps of a tile
// with no smaller gap inside its window have strictly decreasing (left side)
// or increasing (right side) prefix lengths, so there are at most 64 per side.
constexpr uint32_t kTreeFarPerTile = 128;

// Segments and the tile map of every kernel, plus per-segment results.
struct Plan {
  SegTable seg{};
  TileMap point_map{}, sort_map{}, unique_map{}, tree_map{}, scan_map{}, node_map{};
  uint32_t* n_unique = nullptr;  // [segments]
  uint32_t* n_octree = nullptr;  // [segments]
  int32_t* seg_err = nullptr;    // [segments] first error of each segment
  const uint32_t* oct_off = nullptr;  // [segments + 1] octree row offsets
  uint32_t oct_capacity = 0;          // rows when there is one segment
};

// ---- onesweep variant menu (k_keys.cu) --------------------------------------
uint32_t sort_tile_for(int key_bits, int radix_bits);
uint32_t sort_variant_tile(int idx);
int sort_variant_count();
int sort_variant_info(int idx, int* key_bits, int* radix_bits, int* threads, int* kpt,
                      int* rank);
int default_sort_variant(int key_bits, int radix_bits);

// ---- launchers (each returns the launch's cudaError_t) --------------------
// Stage 1 (encode) and/or the sort's digit histograms (hist).
cudaError_t launch_keys(const Bufs& b, const Scratch& sc, const Plan& pl, bool encode,
                        bool hist, cudaStream_t s);
// Init rows + every pass; `marks`, when given, gets one event after the init
// kernel and one after each pass (profiling only).
cudaError_t launch_sort_passes(const Bufs& b, const Scratch& sc, const Plan& pl,
                               cudaStream_t s, cudaEvent_t* marks = nullptr);
// The onesweep sort of keys[0, n) into out on `im`'s scratch, with every
// kernel gated on *gate (see Scratch::gate); `clear` zeroes the scratch's
// zero region first (not needed when a pipeline cleared it and has not used
// it since).  For the learned sort's device-decided fallback.
int sort_enqueue_gated(rw_tree_im_storage* im, const void* keys, void* out, uint32_t n,
                       const uint32_t* gate, bool clear, cudaStream_t s);

// The learned-CDF sort of keys[0, n) into sorted, enqueued without any host
// wait: the bucket sort and a gated onesweep fallback on fallback_im (needed)
// are both enqueued and the plan's overflow word picks one on the device.
// The plan is copied to pinned host memory; learned_last_stats reads it once
// the stream has passed this sort.
int learned_sort_enqueue(rw_tree_learned* L, const uint32_t* keys, uint32_t* sorted, uint32_t n,
                         int32_t mode, rw_tree_im_storage* fallback_im, bool clear_fallback,
                         cudaStream_t s);
void learned_last_stats(const rw_tree_learned* L, rw_tree_learned_stats* out);
uint32_t learned_capacity(const rw_tree_learned* L);  // n_max it was created for

// Test hook of the bounded look-back wait: the digit histograms of b.keys,
// then pass 0 of the sort into b.alt with tile 0 left out, so that every
// other tile's look-back waits on a row nothing publishes and gives up after
// spin_limit polls (RW_ERR_TIMEOUT in the status word).  Needs >= 2 tiles.
cudaError_t launch_sort_lookback_probe(const Bufs& b, const Scratch& sc, const Plan& pl,
                                       uint32_t spin_limit, cudaStream_t s);
cudaError_t launch_unique(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s);
// The unique kernels on caller-given scratch: `counts` holds one word per
// kUniqueTile keys plus one and, like *status, must be zero.
cudaError_t launch_unique_raw(const void* sorted, void* out, uint32_t n, int key_bits,
                              uint32_t* counts, DevStatus* status, int num_sms,
                              cudaStream_t s);
// Stage 4 alone (edges = false) or stages 4 and 5 in one pass (edges = true).
cudaError_t launch_radix_tree(const Bufs& b, const Scratch& sc, const Plan& pl, bool edges,
                              cudaStream_t s);
cudaError_t launch_edge_count(const Bufs& b, const Scratch& sc, const Plan& pl,
                              cudaStream_t s);
cudaError_t launch_edge_scan(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s);
// The first half of stage 6 on the octree's tiles: each tile's count sum,
// scanned into sc.scan_desc, and the octree row counts.  launch_octree with
// fused_offsets then makes and writes the offsets itself.
cudaError_t launch_edge_sums(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s);
cudaError_t launch_octree(const Bufs& b, const Scratch& sc, const Plan& pl, cudaStream_t s,
                          cudaEvent_t* marks = nullptr, bool fused_offsets = false);

// Options outside the reference contract (RW_TREE_OPT_*), single cloud only:
// prefix_n[0, n_brt) -= 1 after stage 4 (the clz - 2 delta of 32-bit keys),
// and the leaf links after stage 7.
cudaError_t launch_prefix_shift(const Bufs& b, const Scratch& sc, const Plan& pl,
                                cudaStream_t s);
cudaError_t launch_leaf_links(const Bufs& b, const Scratch& sc, const Plan& pl,
                              cudaStream_t s);

// Text returned by rw_tree_last_error (this thread).
void set_last_error(const std::string& msg);

// One-segment plan for n points (tile maps computed arithmetically); counts
// and errors go to `status`.
Plan single_plan(uint32_t n, uint32_t oct_capacity, DevStatus* status, uint32_t sort_tile);

}  // namespace rwt
