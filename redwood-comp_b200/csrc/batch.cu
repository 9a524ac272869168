// Batched tree pipeline: many point clouds of uneven size, stored back to
// back, run through the same seven stages with one launch per kernel for the
// whole batch (each kernel walks a tile map whose tiles never straddle two
// clouds).  Counts stay on the device; the whole sequence is captured into a
// CUDA graph once per buffer set and replayed.  Every cloud's outputs equal
// those of a plain run on that cloud alone.  No reference counterpart: the
// reference builds one cloud per call (apps/tree/pipe_main_baseline.cpp:55-92).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "internal.hpp"

struct rw_tree_batch {
  uint32_t n_clouds = 0;
  uint32_t n_total = 0;
  int32_t key_bits = 32;
  int device = 0;
  int num_sms = 148;
  int radix_bits = 8;
  int passes = 4;
  int sort_variant = 0;

  std::vector<uint32_t> h_pt_off, h_oct_off;
  uint32_t oct_rows = 0;

  // device tables, one allocation: pt_off, oct_off and the tile offsets of
  // every kernel, each [n_clouds + 1]
  uint32_t* d_tables = nullptr;
  uint32_t *d_pt_off = nullptr, *d_oct_off = nullptr, *d_point_toff = nullptr,
           *d_unique_toff = nullptr, *d_tree_toff = nullptr,
           *d_scan_toff = nullptr, *d_node_toff = nullptr;
  uint32_t point_tiles = 0, unique_tiles = 0, tree_tiles = 0,
           scan_tiles = 0, node_tiles = 0;
  uint32_t sort_rows = 0;  // rows per pass (stride), room for kMaxSortClasses classes

  // size classes of the sort: clouds with n_c <= class_max[k] (first match)
  // run variant class_variant[k]; each class has its own tile map and rows
  uint32_t n_classes = 1;
  uint32_t class_max[rwt::kMaxSortClasses] = {0xffffffffu};
  int class_variant[rwt::kMaxSortClasses] = {0};
  uint32_t class_tiles[rwt::kMaxSortClasses] = {0};
  uint32_t class_base[rwt::kMaxSortClasses] = {0};  // first descriptor row
  uint32_t* d_class_toff = nullptr;                  // [kMaxSortClasses][n_clouds + 1]

  void* d_tmp_keys = nullptr;
  uint32_t* d_tree_far = nullptr;  // far lists of the radix tree, then of the octree
  uint32_t tree_far_cap = 0;
  void* d_zero = nullptr;
  size_t zero_bytes = 0;
  uint32_t *d_ghist = nullptr, *d_skew = nullptr, *d_sort_desc = nullptr,
           *d_unique_desc = nullptr,
           *d_scan_desc = nullptr, *d_tile_ctr = nullptr;
  rwt::DevStatus* d_status = nullptr;
  uint32_t *d_n_unique = nullptr, *d_n_octree = nullptr;
  int32_t* d_seg_err = nullptr;

  uint32_t* h_results = nullptr;  // pinned: n_unique[C], n_octree[C], seg_err[C], status

  // optional learned-CDF sort for stage 2, one sort per cloud (not owned)
  rw_tree_learned* learned = nullptr;
  int32_t learned_mode = 0;
  rw_tree_im_storage* learned_fallback = nullptr;

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  rw_tree_batch_buffers graph_bufs{};
  cudaStream_t graph_stream = nullptr;
};

namespace {

int fail(cudaError_t e, const char* what) {
  rwt::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return RW_ERR_CUDA;
}

#define RWB_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return fail(e_, #call);       \
  } while (0)

int code_bits(int32_t key_bits) { return key_bits == 32 ? 30 : 63; }

// tile offsets of a kernel with tile size `tile`
std::vector<uint32_t> tile_offsets(const std::vector<uint32_t>& pt_off, uint32_t tile) {
  std::vector<uint32_t> t(pt_off.size(), 0);
  for (size_t c = 0; c + 1 < pt_off.size(); ++c)
    t[c + 1] = t[c] + rwt::div_up(pt_off[c + 1] - pt_off[c], tile);
  return t;
}

// Tile maps and descriptor rows of the sort's size classes.
int upload_classes(rw_tree_batch* b) {
  const size_t tab = size_t(b->n_clouds) + 1;
  std::vector<uint32_t> all;
  all.reserve(rwt::kMaxSortClasses * tab);
  uint32_t base = 0;
  for (uint32_t k = 0; k < rwt::kMaxSortClasses; ++k) {
    std::vector<uint32_t> t(tab, 0);
    if (k < b->n_classes) {
      const uint32_t tile = rwt::sort_variant_tile(b->class_variant[k]);
      for (uint32_t c = 0; c < b->n_clouds; ++c) {
        const uint32_t n = b->h_pt_off[c + 1] - b->h_pt_off[c];
        uint32_t cls = b->n_classes - 1;
        for (uint32_t j = 0; j < b->n_classes; ++j)
          if (n <= b->class_max[j]) {
            cls = j;
            break;
          }
        t[c + 1] = t[c] + (cls == k ? rwt::div_up(n, tile) : 0u);
      }
      b->class_tiles[k] = t.back();
      b->class_base[k] = base;
      base += t.back() + b->n_clouds;
    }
    all.insert(all.end(), t.begin(), t.end());
  }
  if (base > b->sort_rows) return RW_ERR_ARG;
  RWB_CUDA(cudaMemcpy(b->d_class_toff, all.data(), 4 * all.size(), cudaMemcpyHostToDevice));
  return RW_OK;
}

rwt::Bufs bufs_of(const rw_tree_batch* b, const rw_tree_batch_buffers* u) {
  rwt::Bufs x;
  x.key_bits = b->key_bits;
  x.min_coord = 0.0f;
  x.range = 1024.0f;
  x.points = reinterpret_cast<const float4*>(u->points);
  x.keys = u->morton_keys;
  x.alt = u->morton_keys_alt;
  x.tmp = b->d_tmp_keys;
  x.prefix_n = u->prefix_n;
  x.hl = u->has_leaf_left;
  x.hr = u->has_leaf_right;
  x.lc = u->left_child;
  x.parents = u->parents;
  x.edge_count = u->edge_count;
  x.edge_offset = u->edge_offset;
  x.children = u->children;
  x.corner = reinterpret_cast<float4*>(u->corner);
  x.cell_size = u->cell_size;
  x.node_mask = u->child_node_mask;
  x.leaf_mask = u->child_leaf_mask;
  return x;
}

rwt::Scratch scratch_of(const rw_tree_batch* b) {
  rwt::Scratch sc;
  sc.num_sms = b->num_sms;
  sc.radix_bits = b->radix_bits;
  sc.passes = b->passes;
  sc.sort_variant = b->sort_variant;
  sc.ghist = b->d_ghist;
  sc.skew = b->d_skew;
  sc.sort_desc = b->d_sort_desc;
  sc.sort_rows = b->sort_rows;
  sc.unique_desc = b->d_unique_desc;
  sc.scan_desc = b->d_scan_desc;
  sc.tile_ctr = b->d_tile_ctr;
  sc.status = b->d_status;
  sc.tree_far = b->d_tree_far;
  sc.tree_far_cap = b->tree_far_cap;
  return sc;
}

rwt::Plan plan_of(const rw_tree_batch* b) {
  rwt::Plan pl;
  pl.seg = rwt::SegTable{b->n_clouds, b->n_total, b->d_pt_off};
  pl.point_map = rwt::TileMap{b->point_tiles, b->d_point_toff};
  pl.sort_map = rwt::TileMap{b->class_tiles[0], b->d_class_toff};
  pl.unique_map = rwt::TileMap{b->unique_tiles, b->d_unique_toff};
  pl.tree_map = rwt::TileMap{b->tree_tiles, b->d_tree_toff};
  pl.scan_map = rwt::TileMap{b->scan_tiles, b->d_scan_toff};
  pl.node_map = rwt::TileMap{b->node_tiles, b->d_node_toff};
  pl.n_unique = b->d_n_unique;
  pl.n_octree = b->d_n_octree;
  pl.seg_err = b->d_seg_err;
  pl.oct_off = b->d_oct_off;
  pl.oct_capacity = 0;
  return pl;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int check_bufs(const rw_tree_batch_buffers* u) {
  if (!u || !u->points || !u->morton_keys || !u->morton_keys_alt || !u->edge_count ||
      !u->edge_offset || !u->prefix_n || !u->has_leaf_left || !u->has_leaf_right ||
      !u->left_child || !u->parents || !u->children || !u->corner || !u->cell_size ||
      !u->child_node_mask || !u->child_leaf_mask)
    return RW_ERR_ARG;
  if (!aligned16(u->points) || !aligned16(u->morton_keys) || !aligned16(u->morton_keys_alt) ||
      !aligned16(u->edge_count) || !aligned16(u->edge_offset) || !aligned16(u->children) ||
      !aligned16(u->corner))
    return RW_ERR_ARG;
  return RW_OK;
}

void release_graph(rw_tree_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

void release_stream(rw_tree_batch* b) {
  if (b->graph_stream) cudaStreamDestroy(b->graph_stream);
  b->graph_stream = nullptr;
}

}  // namespace

extern "C" {

int rw_tree_batch_create(const uint32_t* cloud_sizes, uint32_t n_clouds, int32_t key_bits,
                         int32_t radix_bits, float octree_ratio, rw_tree_batch** out) {
  if (!out || !cloud_sizes || n_clouds < 1 || (key_bits != 32 && key_bits != 64) ||
      (radix_bits != 0 && radix_bits != 8 && radix_bits != 10 && radix_bits != 11) || !(octree_ratio < 64.0f))
    return RW_ERR_ARG;
  const float ratio = octree_ratio > 0.0f ? octree_ratio : 0.6f;
  *out = nullptr;
  uint64_t total = 0;
  for (uint32_t c = 0; c < n_clouds; ++c) {
    if (cloud_sizes[c] < 1) return RW_ERR_ARG;
    total += cloud_sizes[c];
  }
  if (total >= RW_MAX_POINTS) return RW_ERR_ARG;
  {
    uint64_t rows = 0;
    for (uint32_t c = 0; c < n_clouds; ++c) rows += uint64_t(float(cloud_sizes[c]) * ratio) + 1;
    if (rows >= RW_MAX_POINTS * uint64_t(8)) return RW_ERR_ARG;
  }
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count < 1) return RW_ERR_NO_DEVICE;

  auto* b = new rw_tree_batch();
  b->n_clouds = n_clouds;
  b->n_total = uint32_t(total);
  b->key_bits = key_bits;
  cudaGetDevice(&b->device);
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
  b->radix_bits = radix_bits ? radix_bits : 8;
  b->passes = (code_bits(key_bits) + b->radix_bits - 1) / b->radix_bits;
  b->sort_variant = rwt::default_sort_variant(key_bits, b->radix_bits);
  b->class_variant[0] = b->sort_variant;

  b->h_pt_off.assign(n_clouds + 1, 0);
  b->h_oct_off.assign(n_clouds + 1, 0);
  for (uint32_t c = 0; c < n_clouds; ++c) {
    b->h_pt_off[c + 1] = b->h_pt_off[c] + cloud_sizes[c];
    // rows = floor(n_c * ratio) in float, the formula of app_data.hpp:28
    const float rows = float(cloud_sizes[c]) * ratio;
    b->h_oct_off[c + 1] = b->h_oct_off[c] + std::max(1u, uint32_t(rows));
  }
  b->oct_rows = b->h_oct_off.back();

  const auto point_t = tile_offsets(b->h_pt_off, rwt::kPointTile);
  const auto unique_t = tile_offsets(b->h_pt_off, rwt::kUniqueTile);
  const auto tree_t = tile_offsets(b->h_pt_off, rwt::kTreeTile);
  const auto scan_t = tile_offsets(b->h_pt_off, rwt::kScanTile);
  const auto node_t = tile_offsets(b->h_pt_off, rwt::kOctTile);
  const auto min_sort_t =
      tile_offsets(b->h_pt_off, rwt::sort_tile_for(key_bits, b->radix_bits));
  b->point_tiles = point_t.back();
  b->unique_tiles = unique_t.back();
  b->tree_tiles = tree_t.back();
  b->scan_tiles = scan_t.back();
  b->node_tiles = node_t.back();
  b->sort_rows = min_sort_t.back() + rwt::kMaxSortClasses * n_clouds;

  const size_t tab = size_t(n_clouds) + 1;
  const size_t radix = size_t(1) << b->radix_bits;
  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t ghist_b = align(size_t(n_clouds) * b->passes * radix * 4);
  const size_t sdesc_b = align(size_t(b->passes) * b->sort_rows * radix * 4);
  const size_t udesc_b = align((size_t(b->unique_tiles) + 1) * 4);
  const size_t cdesc_b = align((size_t(std::max(b->scan_tiles, b->node_tiles)) + 1) * 4);
  const size_t ctr_b = align(rwt::kCounters * 4);
  const size_t st_b = align(sizeof(rwt::DevStatus));
  const size_t per_b = align(size_t(n_clouds) * 4);
  b->zero_bytes = ghist_b + sdesc_b + udesc_b + cdesc_b + ctr_b + st_b + 4 * per_b;

  const size_t ks = key_bits == 32 ? 4 : 8;
  cudaError_t e = cudaMalloc(&b->d_tables, (8 + rwt::kMaxSortClasses) * tab * 4);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_tmp_keys, ks * total);
  b->tree_far_cap = b->tree_tiles * rwt::kTreeFarPerTile;
  if (e == cudaSuccess) e = cudaMalloc(&b->d_tree_far, size_t(b->tree_far_cap) * 16);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_zero, b->zero_bytes);
  if (e == cudaSuccess) e = cudaMallocHost(&b->h_results, (3 * size_t(n_clouds) + 4) * 4);
  if (e != cudaSuccess) {
    rw_tree_batch_destroy(b);
    return fail(e, "rw_tree_batch_create");
  }
  uint32_t* t = b->d_tables;
  b->d_pt_off = t;
  b->d_oct_off = t + tab;
  b->d_point_toff = t + 2 * tab;
  // t + 3 * tab: the smallest-tile sort map (sizing only)
  b->d_unique_toff = t + 4 * tab;
  b->d_tree_toff = t + 5 * tab;
  b->d_scan_toff = t + 6 * tab;
  b->d_node_toff = t + 7 * tab;
  b->d_class_toff = t + 8 * tab;
  char* z = static_cast<char*>(b->d_zero);
  size_t o = 0;
  b->d_ghist = reinterpret_cast<uint32_t*>(z + o); o += ghist_b;
  b->d_sort_desc = reinterpret_cast<uint32_t*>(z + o); o += sdesc_b;
  b->d_unique_desc = reinterpret_cast<uint32_t*>(z + o); o += udesc_b;
  b->d_scan_desc = reinterpret_cast<uint32_t*>(z + o); o += cdesc_b;
  b->d_tile_ctr = reinterpret_cast<uint32_t*>(z + o); o += ctr_b;
  b->d_status = reinterpret_cast<rwt::DevStatus*>(z + o); o += st_b;
  b->d_n_unique = reinterpret_cast<uint32_t*>(z + o); o += per_b;
  b->d_n_octree = reinterpret_cast<uint32_t*>(z + o); o += per_b;
  b->d_seg_err = reinterpret_cast<int32_t*>(z + o); o += per_b;
  b->d_skew = reinterpret_cast<uint32_t*>(z + o); o += per_b;

  std::vector<uint32_t> all;
  all.reserve(8 * tab);
  const std::vector<uint32_t>* parts[] = {&b->h_pt_off, &b->h_oct_off, &point_t, &min_sort_t,
                                          &unique_t,     &tree_t,       &scan_t,  &node_t};
  for (const auto* v : parts) all.insert(all.end(), v->begin(), v->end());
  e = cudaMemcpy(b->d_tables, all.data(), 4 * all.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->d_zero, 0, b->zero_bytes);
  if (e != cudaSuccess || upload_classes(b) != RW_OK) {
    rw_tree_batch_destroy(b);
    return RW_ERR_CUDA;
  }
  *out = b;
  return RW_OK;
}

int rw_tree_batch_destroy(rw_tree_batch* b) {
  if (!b) return RW_OK;
  release_graph(b);
  release_stream(b);
  if (b->d_tables) cudaFree(b->d_tables);
  if (b->d_tmp_keys) cudaFree(b->d_tmp_keys);
  if (b->d_tree_far) cudaFree(b->d_tree_far);
  if (b->d_zero) cudaFree(b->d_zero);
  if (b->h_results) cudaFreeHost(b->h_results);
  delete b;
  return RW_OK;
}

uint32_t rw_tree_batch_total_points(const rw_tree_batch* b) { return b ? b->n_total : 0; }

uint32_t rw_tree_batch_octree_rows(const rw_tree_batch* b) { return b ? b->oct_rows : 0; }

int rw_tree_batch_offsets(const rw_tree_batch* b, uint32_t* point_offsets,
                          uint32_t* octree_offsets) {
  if (!b) return RW_ERR_ARG;
  if (point_offsets) std::memcpy(point_offsets, b->h_pt_off.data(), 4 * b->h_pt_off.size());
  if (octree_offsets) std::memcpy(octree_offsets, b->h_oct_off.data(), 4 * b->h_oct_off.size());
  return RW_OK;
}

int rw_tree_batch_set_sort_variant(rw_tree_batch* b, int32_t idx) {
  const uint32_t all = 0xffffffffu;
  return rw_tree_batch_set_classes(b, 1, &all, &idx);
}

int rw_tree_batch_set_classes(rw_tree_batch* b, uint32_t n_classes, const uint32_t* max_points,
                              const int32_t* variants) {
  if (!b || n_classes < 1 || n_classes > uint32_t(rwt::kMaxSortClasses) || !max_points ||
      !variants)
    return RW_ERR_ARG;
  for (uint32_t k = 0; k < n_classes; ++k) {
    int kb, rb, th, kpt, rk;
    if (rwt::sort_variant_info(variants[k], &kb, &rb, &th, &kpt, &rk) != 0) return RW_ERR_ARG;
    if (kb != b->key_bits || rb != b->radix_bits) return RW_ERR_ARG;
    if (k > 0 && max_points[k] <= max_points[k - 1]) return RW_ERR_ARG;
  }
  // keep the current classes to restore them if the new ones do not fit
  const uint32_t old_n = b->n_classes;
  uint32_t old_max[rwt::kMaxSortClasses];
  int old_var[rwt::kMaxSortClasses];
  std::memcpy(old_max, b->class_max, sizeof old_max);
  std::memcpy(old_var, b->class_variant, sizeof old_var);
  b->n_classes = n_classes;
  for (uint32_t k = 0; k < n_classes; ++k) {
    b->class_max[k] = max_points[k];
    b->class_variant[k] = variants[k];
  }
  b->class_max[n_classes - 1] = 0xffffffffu;  // the last class takes the rest
  if (int rc = upload_classes(b)) {
    b->n_classes = old_n;
    std::memcpy(b->class_max, old_max, sizeof old_max);
    std::memcpy(b->class_variant, old_var, sizeof old_var);
    upload_classes(b);
    return rc;
  }
  b->sort_variant = variants[0];
  release_graph(b);  // the captured graph used the previous classes
  return RW_OK;
}

int rw_tree_batch_set_learned(rw_tree_batch* b, rw_tree_learned* learned, int32_t mode,
                              rw_tree_im_storage* fallback_im) {
  if (!b || (mode != RW_LEARNED_MLP && mode != RW_LEARNED_SAMPLE_QUANTILES)) return RW_ERR_ARG;
  if (learned) {
    uint32_t largest = 0;
    for (uint32_t c = 0; c < b->n_clouds; ++c)
      largest = std::max(largest, b->h_pt_off[c + 1] - b->h_pt_off[c]);
    if (b->key_bits != 32 || !fallback_im || rwt::learned_capacity(learned) < largest ||
        fallback_im->key_bits != 32 || fallback_im->n_cap < largest)
      return RW_ERR_ARG;
  }
  b->learned = learned;
  b->learned_mode = mode;
  b->learned_fallback = learned ? fallback_im : nullptr;
  release_graph(b);  // the captured graph used the other stage 2
  return RW_OK;
}

int rw_tree_batch_enqueue(rw_tree_batch* b, const rw_tree_batch_buffers* u, rw_stream_t stream) {
  if (!b) return RW_ERR_ARG;
  if (int rc = check_bufs(u)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const auto x = bufs_of(b, u);
  const auto sc = scratch_of(b);
  const auto pl = plan_of(b);
  RWB_CUDA(cudaMemsetAsync(b->d_zero, 0, b->zero_bytes, s));
  if (b->learned) {
    // stage 1 without the digit histograms, then every cloud's learned sort
    // (asynchronous: its onesweep fallback is decided on the device), back to
    // back on the stream
    RWB_CUDA(rwt::launch_keys(x, sc, pl, true, false, s));
    const uint32_t* keys = static_cast<const uint32_t*>(x.keys);
    uint32_t* alt = static_cast<uint32_t*>(x.alt);
    for (uint32_t c = 0; c < b->n_clouds; ++c) {
      const uint32_t p0 = b->h_pt_off[c], nc = b->h_pt_off[c + 1] - p0;
      if (int rc = rwt::learned_sort_enqueue(b->learned, keys + p0, alt + p0, nc, b->learned_mode,
                                             b->learned_fallback, true, s))
        return rc;
    }
  }
  if (!b->learned) RWB_CUDA(rwt::launch_keys(x, sc, pl, true, true, s));
  const size_t radix = size_t(1) << b->radix_bits;
  for (uint32_t k = 0; k < b->n_classes && !b->learned; ++k) {
    if (!b->class_tiles[k]) continue;
    rwt::Scratch sk = sc;
    sk.sort_variant = b->class_variant[k];
    sk.sort_desc = b->d_sort_desc + size_t(b->class_base[k]) * radix;
    sk.tile_ctr = b->d_tile_ctr + k * rwt::kCtrSortClassStride;
    rwt::Plan pk = pl;
    pk.sort_map = rwt::TileMap{b->class_tiles[k], b->d_class_toff + k * (size_t(b->n_clouds) + 1)};
    RWB_CUDA(rwt::launch_sort_passes(x, sk, pk, s));
  }
  RWB_CUDA(rwt::launch_unique(x, sc, pl, s));
  RWB_CUDA(rwt::launch_radix_tree(x, sc, pl, true, s));
  RWB_CUDA(rwt::launch_edge_sums(x, sc, pl, s));
  RWB_CUDA(rwt::launch_octree(x, sc, pl, s, nullptr, true));
  const size_t c = b->n_clouds;
  RWB_CUDA(cudaMemcpyAsync(b->h_results, b->d_n_unique, 4 * c, cudaMemcpyDeviceToHost, s));
  RWB_CUDA(cudaMemcpyAsync(b->h_results + c, b->d_n_octree, 4 * c, cudaMemcpyDeviceToHost, s));
  RWB_CUDA(cudaMemcpyAsync(b->h_results + 2 * c, b->d_seg_err, 4 * c, cudaMemcpyDeviceToHost, s));
  RWB_CUDA(cudaMemcpyAsync(b->h_results + 3 * c, b->d_status, sizeof(rwt::DevStatus),
                           cudaMemcpyDeviceToHost, s));
  return RW_OK;
}

int rw_tree_batch_graph_launch(rw_tree_batch* b, const rw_tree_batch_buffers* u,
                               rw_stream_t stream) {
  if (!b) return RW_ERR_ARG;
  if (int rc = check_bufs(u)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const bool same = b->exec && std::memcmp(&b->graph_bufs, u, sizeof *u) == 0;
  if (!same) {
    release_graph(b);
    // captured on a stream of our own: the caller's may be the legacy default
    // stream, which cannot be captured; the graph is then launched into it
    if (!b->graph_stream)
      RWB_CUDA(cudaStreamCreateWithFlags(&b->graph_stream, cudaStreamNonBlocking));
    RWB_CUDA(cudaStreamBeginCapture(b->graph_stream, cudaStreamCaptureModeThreadLocal));
    const int rc = rw_tree_batch_enqueue(b, u, reinterpret_cast<rw_stream_t>(b->graph_stream));
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->graph_stream, &g);
    if (rc != RW_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(e, "cudaStreamEndCapture");
    b->graph = g;
    RWB_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    b->graph_bufs = *u;
  }
  RWB_CUDA(cudaGraphLaunch(b->exec, s));
  return RW_OK;
}

int rw_tree_batch_finish(rw_tree_batch* b, rw_stream_t stream, uint32_t* n_unique,
                         uint32_t* n_octree_nodes, int32_t* status) {
  if (!b) return RW_ERR_ARG;
  RWB_CUDA(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)));
  const size_t c = b->n_clouds;
  if (n_unique) std::memcpy(n_unique, b->h_results, 4 * c);
  if (n_octree_nodes) std::memcpy(n_octree_nodes, b->h_results + c, 4 * c);
  if (status) std::memcpy(status, b->h_results + 2 * c, 4 * c);
  rwt::DevStatus st;
  std::memcpy(&st, b->h_results + 3 * c, sizeof st);
  return st.err == RW_ERR_TIMEOUT ? RW_ERR_TIMEOUT : RW_OK;
}

}  // extern "C"
