// Host-side internals shared by the kernel translation units and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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

  // zero region
  void* d_zero = nullptr;
  size_t zero_bytes = 0;
  uint32_t* d_ghist = nullptr;      // [passes][radix]
  uint32_t* d_sort_desc = nullptr;  // [passes][sort_tiles + 1][radix]
  uint32_t* d_unique_desc = nullptr;
  uint32_t* d_scan_desc = nullptr;
  uint32_t* d_tile_ctr = nullptr;   // [kCounters]
  rwt::DevStatus* d_status = nullptr;
  size_t sort_zero_off = 0, sort_zero_bytes = 0;  // ghist + sort_desc

  rwt::DevStatus* h_status = nullptr;  // pinned mirror
};

namespace rwt {

enum : int { kCtrUnique = 0, kCtrScan = 1, kCtrTree = 2, kCtrSortBase = 4,
             kCounters = 32 };

// Tiles for the single-value chained scans (unique, edge-offset scan, fused
// radix tree).
constexpr uint32_t kUniqueThreads = 256, kUniqueKpt = 16;
constexpr uint32_t kUniqueTile = kUniqueThreads * kUniqueKpt;
constexpr uint32_t kScanThreads = 256, kScanKpt = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanKpt;
constexpr int kTreeThreads = 256, kTreeNpt = 4, kTreeHalo = 256;
constexpr uint32_t kTreeTile = kTreeThreads * kTreeNpt;

inline uint32_t div_up(uint64_t a, uint64_t b) { return uint32_t((a + b - 1) / b); }

// A count either known on the host (value) or produced on the device (ptr).
struct Count {
  const uint32_t* ptr;
  uint32_t value;
};

// ---- onesweep variant menu (k_keys.cu) --------------------------------------
uint32_t sort_tile_for(int key_bits, int radix_bits);
int sort_variant_count();
int sort_variant_info(int idx, int* key_bits, int* radix_bits, int* threads, int* kpt,
                      int* rank);
int default_sort_variant(int key_bits, int radix_bits);

// ---- launchers (each returns the launch's cudaError_t) --------------------

cudaError_t launch_morton(const rw_tree_app_data& app, rw_tree_im_storage* im,
                          bool with_histogram, cudaStream_t s);
cudaError_t launch_histogram(const rw_tree_app_data& app, rw_tree_im_storage* im,
                             cudaStream_t s);
// `marks`, when given, gets one event recorded after sort_init and after each
// pass (profiling only).
cudaError_t launch_sort_passes(const rw_tree_app_data& app,
                               rw_tree_im_storage* im, cudaStream_t s,
                               cudaEvent_t* marks = nullptr);
cudaError_t launch_unique(const rw_tree_app_data& app, rw_tree_im_storage* im,
                          cudaStream_t s);
// The unique kernel on caller-given scratch: `desc` holds one word per
// kUniqueTile keys and, like *tile_ctr and *status, must be zero.
cudaError_t launch_unique_raw(const void* sorted, void* out, uint32_t n, int key_bits,
                              uint32_t* desc, uint32_t* tile_ctr, DevStatus* status,
                              int num_sms, cudaStream_t s);
// Stage 4 alone (edges = false) or stages 4 and 5 in one pass (edges = true).
cudaError_t launch_radix_tree(const rw_tree_app_data& app,
                              rw_tree_im_storage* im, Count n_unique,
                              bool edges, cudaStream_t s);
cudaError_t launch_edge_count(const rw_tree_app_data& app,
                              rw_tree_im_storage* im, Count n_unique,
                              cudaStream_t s);
cudaError_t launch_edge_scan(const rw_tree_app_data& app,
                             rw_tree_im_storage* im, Count n_unique,
                             cudaStream_t s);
cudaError_t launch_octree(const rw_tree_app_data& app, rw_tree_im_storage* im,
                          Count n_unique, Count n_octree, cudaStream_t s,
                          cudaEvent_t* marks = nullptr);

}  // namespace rwt
