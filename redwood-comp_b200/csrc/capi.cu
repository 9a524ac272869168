// C ABI of the tree pipeline (declared in include/rw_tree.h).
//
// The per-stage calls mirror cuda::run_stage1..7 (apps/tree/cuda/
// cu_dispatcher.cu:501-752): each is synchronous and updates the counts of the
// app struct.  The pipeline calls run the same work with fused kernels and
// device-resident counts, without any host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "internal.hpp"

namespace {

thread_local std::string g_last_error;

int cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return RW_ERR_CUDA;
}

#define RW_CUDA(call)                                         \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);       \
  } while (0)

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

size_t key_size(int32_t key_bits) { return key_bits == 32 ? 4 : 8; }

int code_bits(int32_t key_bits) { return key_bits == 32 ? 30 : 63; }

// Common argument checks.  `need` lists the buffers a stage touches.
enum Need : unsigned {
  kPoints = 1, kKeys = 2, kAlt = 4, kBrt = 8, kEdge = 16, kOct = 32
};

int check(const rw_tree_app_data* app, const rw_tree_im_storage* im, unsigned need) {
  if (!app || !im) return RW_ERR_ARG;
  if (app->key_bits != 32 && app->key_bits != 64) return RW_ERR_ARG;
  if (app->key_bits != im->key_bits) return RW_ERR_ARG;
  if (app->n_input < 1 || app->n_input >= RW_MAX_POINTS || app->n_input > im->n_cap)
    return RW_ERR_ARG;
  if ((need & kPoints) && !(app->u_input_points && aligned16(app->u_input_points)))
    return RW_ERR_ARG;
  if ((need & kKeys) && !(app->u_morton_keys && aligned16(app->u_morton_keys)))
    return RW_ERR_ARG;
  if ((need & kAlt) && !(app->u_morton_keys_alt && aligned16(app->u_morton_keys_alt)))
    return RW_ERR_ARG;
  if ((need & kBrt) && !(app->brt_prefix_n && app->brt_has_leaf_left &&
                         app->brt_has_leaf_right && app->brt_left_child &&
                         app->brt_parents))
    return RW_ERR_ARG;
  if ((need & kEdge) && !(app->u_edge_count && app->u_edge_offset &&
                          aligned16(app->u_edge_count) && aligned16(app->u_edge_offset)))
    return RW_ERR_ARG;
  if ((need & kOct) &&
      !(app->oct_children && app->oct_corner && app->oct_cell_size &&
        app->oct_child_node_mask && app->oct_child_leaf_mask &&
        aligned16(app->oct_children) && aligned16(app->oct_corner)))
    return RW_ERR_ARG;
  return RW_OK;
}

rwt::Bufs bufs_of(const rw_tree_app_data& a, const rw_tree_im_storage* im) {
  rwt::Bufs b;
  b.key_bits = a.key_bits;
  b.min_coord = a.min_coord;
  b.range = a.range;
  b.points = reinterpret_cast<const float4*>(a.u_input_points);
  b.keys = a.u_morton_keys;
  b.alt = a.u_morton_keys_alt;
  b.tmp = im->d_tmp_keys;
  b.prefix_n = a.brt_prefix_n;
  b.hl = a.brt_has_leaf_left;
  b.hr = a.brt_has_leaf_right;
  b.lc = a.brt_left_child;
  b.parents = a.brt_parents;
  b.edge_count = a.u_edge_count;
  b.edge_offset = a.u_edge_offset;
  b.children = a.oct_children;
  b.corner = reinterpret_cast<float4*>(a.oct_corner);
  b.cell_size = a.oct_cell_size;
  b.node_mask = a.oct_child_node_mask;
  b.leaf_mask = a.oct_child_leaf_mask;
  return b;
}

rwt::Scratch scratch_of(const rw_tree_im_storage* im) {
  rwt::Scratch sc;
  sc.num_sms = im->num_sms;
  sc.radix_bits = im->radix_bits;
  sc.passes = im->passes;
  sc.sort_variant = im->sort_variant;
  sc.ghist = im->d_ghist;
  sc.skew = im->d_skew;
  sc.sort_desc = im->d_sort_desc;
  sc.sort_rows = im->sort_tiles + 1;
  sc.unique_desc = im->d_unique_desc;
  sc.scan_desc = im->d_scan_desc;
  sc.tile_ctr = im->d_tile_ctr;
  sc.status = im->d_status;
  sc.tree_far = im->d_tree_far;
  sc.tree_far_cap = im->tree_far_cap;
  return sc;
}

rwt::Plan plan_of(const rw_tree_app_data& a, const rw_tree_im_storage* im) {
  return rwt::single_plan(a.n_input, a.oct_capacity, im->d_status,
                          rwt::sort_variant_tile(im->sort_variant));
}

// Device status := the host's counts of `app`, error word cleared (for the
// per-stage calls whose kernels read the counts on the device).
int upload_counts(const rw_tree_app_data* app, rw_tree_im_storage* im, cudaStream_t s) {
  RW_CUDA(cudaStreamSynchronize(s));  // the pinned mirror may still be in use
  im->h_status->n_unique = app->n_unique;
  im->h_status->n_octree_nodes = app->n_octree_nodes;
  im->h_status->err = 0;
  im->h_status->err_site = 0;
  RW_CUDA(cudaMemcpyAsync(im->d_status, im->h_status, sizeof(rwt::DevStatus),
                          cudaMemcpyHostToDevice, s));
  return RW_OK;
}

bool geometric_delta(const rw_tree_im_storage* im) {
  return (im->options & RW_TREE_OPT_GEOMETRIC_DELTA) && im->key_bits == 32;
}

int clear_all(rw_tree_im_storage* im, cudaStream_t s) {
  RW_CUDA(cudaMemsetAsync(im->d_zero, 0, im->zero_bytes, s));
  return RW_OK;
}

// Waits for the stream, copies the device status and maps its error word.
int sync_status(rw_tree_im_storage* im, cudaStream_t s) {
  RW_CUDA(cudaMemcpyAsync(im->h_status, im->d_status, sizeof(rwt::DevStatus),
                          cudaMemcpyDeviceToHost, s));
  RW_CUDA(cudaStreamSynchronize(s));
  if (im->h_status->err != 0) {
    char buf[96];
    std::snprintf(buf, sizeof buf, "device error %d at site %u", im->h_status->err,
                  im->h_status->err_site);
    g_last_error = buf;
    return im->h_status->err;
  }
  return RW_OK;
}

}  // namespace

namespace rwt {
void set_last_error(const std::string& msg) { g_last_error = msg; }

int sort_enqueue_gated(rw_tree_im_storage* im, const void* keys, void* out, uint32_t n,
                       const uint32_t* gate, bool clear, cudaStream_t s) {
  // internal callers pass key ranges of a batch, which start anywhere: the
  // sort's kernels load and store keys one at a time, so only the word
  // alignment of the key type is needed
  if (!im || !keys || !out || n < 1 || n > im->n_cap || n >= RW_MAX_POINTS) return RW_ERR_ARG;
  rw_tree_app_data app;
  rw_tree_app_data_init(&app, n, im->key_bits);
  app.u_morton_keys = const_cast<void*>(keys);
  app.u_morton_keys_alt = out;
  if (clear)
    if (int rc = clear_all(im, s)) return rc;
  const auto b = bufs_of(app, im);
  auto sc = scratch_of(im);
  sc.gate = gate;
  const auto pl = plan_of(app, im);
  RW_CUDA(launch_keys(b, sc, pl, false, true, s));
  RW_CUDA(launch_sort_passes(b, sc, pl, s));
  return RW_OK;
}
}  // namespace rwt

extern "C" {

uint32_t rw_tree_octree_capacity(uint32_t n_input) {
  const float rows = float(n_input) * 0.6f;
  return uint32_t(rows);
}

void rw_tree_app_data_init(rw_tree_app_data* app, uint32_t n_input, int32_t key_bits) {
  std::memset(app, 0, sizeof *app);
  app->n_input = n_input;
  app->oct_capacity = rw_tree_octree_capacity(n_input);
  app->key_bits = key_bits;
  app->min_coord = 0.0f;
  app->range = 1024.0f;
  app->n_unique = app->n_brt_nodes = app->n_octree_nodes = RW_COUNT_UNSET;
}

const char* rw_tree_last_error(void) { return g_last_error.c_str(); }

const char* rw_tree_version(void) { return "rw_tree 0.1 sm_100a"; }

int rw_tree_im_storage_create(uint32_t n_input, int32_t key_bits,
                              rw_tree_im_storage** out) {
  return rw_tree_im_storage_create_ex(n_input, key_bits, 0, out);
}

int rw_tree_im_storage_create_ex(uint32_t n_input, int32_t key_bits,
                                 int32_t radix_bits, rw_tree_im_storage** out) {
  if (!out || n_input < 1 || n_input >= RW_MAX_POINTS ||
      (key_bits != 32 && key_bits != 64) ||
      (radix_bits != 0 && radix_bits != 8 && radix_bits != 10 && radix_bits != 11))
    return RW_ERR_ARG;
  *out = nullptr;
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count < 1) {
    g_last_error = "no CUDA device";
    return RW_ERR_NO_DEVICE;
  }
  int device = 0, sms = 0;
  RW_CUDA(cudaGetDevice(&device));
  RW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  auto* im = new rw_tree_im_storage();
  im->n_cap = n_input;
  im->key_bits = key_bits;
  im->device = device;
  im->num_sms = sms;
  im->radix_bits = radix_bits == 0 ? 8 : radix_bits;
  im->passes = (code_bits(key_bits) + im->radix_bits - 1) / im->radix_bits;
  im->sort_variant = rwt::default_sort_variant(key_bits, im->radix_bits);
  im->sort_tile = rwt::sort_tile_for(key_bits, im->radix_bits);
  im->sort_tiles = rwt::div_up(n_input, im->sort_tile);
  const size_t radix = size_t(1) << im->radix_bits;

  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t ghist_b = align(size_t(im->passes) * radix * 4);
  const size_t skew_b = align(4);
  const size_t sdesc_b = align(size_t(im->passes) * (im->sort_tiles + 1) * radix * 4);
  const size_t udesc_b = align((size_t(rwt::div_up(n_input, rwt::kUniqueTile)) + 1) * 4);
  // stage 6's tiles, or the octree's (smaller) ones in the fused pipeline
  const size_t cdesc_b = align((size_t(rwt::div_up(n_input, rwt::kOctTile)) + 1) * 4);
  static_assert(rwt::kOctTile <= rwt::kScanTile, "scan descriptors sized by the octree tiles");
  const size_t ctr_b = align(rwt::kCounters * 4);
  const size_t st_b = align(sizeof(rwt::DevStatus));
  im->zero_bytes = ghist_b + skew_b + sdesc_b + udesc_b + cdesc_b + ctr_b + st_b;

  cudaError_t e = cudaMalloc(&im->d_zero, im->zero_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&im->d_tmp_keys, key_size(key_bits) * n_input);
  im->tree_far_cap = rwt::div_up(n_input, rwt::kTreeTile) * rwt::kTreeFarPerTile;
  if (e == cudaSuccess) e = cudaMalloc(&im->d_tree_far, size_t(im->tree_far_cap) * 16);
  if (e == cudaSuccess) e = cudaMallocHost(&im->h_status, sizeof(rwt::DevStatus));
  if (e != cudaSuccess) {
    rw_tree_im_storage_destroy(im);
    return cuda_fail(e, "rw_tree_im_storage_create");
  }
  char* z = static_cast<char*>(im->d_zero);
  size_t o = 0;
  im->d_ghist = reinterpret_cast<uint32_t*>(z + o); o += ghist_b;
  im->d_skew = reinterpret_cast<uint32_t*>(z + o); o += skew_b;
  im->d_sort_desc = reinterpret_cast<uint32_t*>(z + o); o += sdesc_b;
  im->d_unique_desc = reinterpret_cast<uint32_t*>(z + o); o += udesc_b;
  im->d_scan_desc = reinterpret_cast<uint32_t*>(z + o); o += cdesc_b;
  im->d_tile_ctr = reinterpret_cast<uint32_t*>(z + o); o += ctr_b;
  im->d_status = reinterpret_cast<rwt::DevStatus*>(z + o);
  std::memset(im->h_status, 0, sizeof(rwt::DevStatus));
  e = cudaMemset(im->d_zero, 0, im->zero_bytes);
  if (e != cudaSuccess) {
    rw_tree_im_storage_destroy(im);
    return cuda_fail(e, "rw_tree_im_storage_create");
  }
  *out = im;
  return RW_OK;
}

int rw_tree_sort_variant_count(void) { return rwt::sort_variant_count(); }

int rw_tree_sort_variant_info(int32_t idx, int32_t* key_bits, int32_t* radix_bits,
                              int32_t* threads, int32_t* keys_per_thread,
                              int32_t* rank_mode) {
  if (!key_bits || !radix_bits || !threads || !keys_per_thread || !rank_mode)
    return RW_ERR_ARG;
  return rwt::sort_variant_info(idx, key_bits, radix_bits, threads, keys_per_thread,
                                rank_mode) == 0
             ? RW_OK
             : RW_ERR_ARG;
}

int rw_tree_im_storage_set_sort_variant(rw_tree_im_storage* im, int32_t idx) {
  int kb, rb, th, kpt, rk;
  if (!im || rwt::sort_variant_info(idx, &kb, &rb, &th, &kpt, &rk) != 0) return RW_ERR_ARG;
  if (kb != im->key_bits || rb != im->radix_bits) return RW_ERR_ARG;
  im->sort_variant = idx;
  return RW_OK;
}

int rw_tree_im_storage_set_options(rw_tree_im_storage* im, int32_t options) {
  if (!im || (options & ~(RW_TREE_OPT_GEOMETRIC_DELTA | RW_TREE_OPT_LINK_LEAVES)))
    return RW_ERR_ARG;
  im->options = options;
  return RW_OK;
}

int rw_tree_im_storage_destroy(rw_tree_im_storage* im) {
  if (!im) return RW_OK;
  if (im->d_zero) cudaFree(im->d_zero);
  if (im->d_tmp_keys) cudaFree(im->d_tmp_keys);
  if (im->d_tree_far) cudaFree(im->d_tree_far);
  if (im->h_status) cudaFreeHost(im->h_status);
  delete im;
  return RW_OK;
}

int rw_tree_im_storage_clear(rw_tree_im_storage* im, rw_stream_t stream) {
  if (!im) return RW_ERR_ARG;
  return clear_all(im, reinterpret_cast<cudaStream_t>(stream));
}

// ---- stage 1: Morton codes (cu_dispatcher.cu:501-522) -----------------------
int rw_tree_run_stage1(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream) {
  if (int rc = check(app, im, kPoints | kKeys)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  RW_CUDA(rwt::launch_keys(bufs_of(*app, im), scratch_of(im), plan_of(*app, im), true, false,
                           s));
  RW_CUDA(cudaStreamSynchronize(s));
  return RW_OK;
}

// ---- stage 2: sort (cu_dispatcher.cu:528-591) ---------------------------------
int rw_tree_run_stage2(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream) {
  if (int rc = check(app, im, kKeys | kAlt)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = clear_all(im, s)) return rc;
  const auto b = bufs_of(*app, im);
  const auto sc = scratch_of(im);
  const auto pl = plan_of(*app, im);
  if (im->learned) {
    if (int rc = rw_tree_learned_sort(im->learned, static_cast<const uint32_t*>(b.keys),
                                      static_cast<uint32_t*>(b.alt), app->n_input,
                                      im->learned_mode, im, stream, &im->learned_stats))
      return rc;
    return sync_status(im, s);
  }
  RW_CUDA(rwt::launch_keys(b, sc, pl, false, true, s));
  RW_CUDA(rwt::launch_sort_passes(b, sc, pl, s));
  return sync_status(im, s);
}

int rw_tree_sort_enqueue(rw_tree_app_data* app, rw_tree_im_storage* im, rw_stream_t stream) {
  if (int rc = check(app, im, kKeys | kAlt)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = clear_all(im, s)) return rc;
  const auto b = bufs_of(*app, im);
  const auto sc = scratch_of(im);
  const auto pl = plan_of(*app, im);
  RW_CUDA(rwt::launch_keys(b, sc, pl, false, true, s));
  RW_CUDA(rwt::launch_sort_passes(b, sc, pl, s));
  return RW_OK;
}

int rw_tree_sort_profile(rw_tree_app_data* app, rw_tree_im_storage* im, rw_stream_t stream,
                         int32_t reps, float* kernel_ms, int32_t max_kernels,
                         int32_t* n_kernels) {
  if (int rc = check(app, im, kKeys | kAlt)) return rc;
  if (!kernel_ms || reps < 1) return RW_ERR_ARG;
  const int n_k = 2 + im->passes;  // histogram, sort_init, one per pass
  if (max_kernels < n_k || n_k + 1 > 64) return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const auto b = bufs_of(*app, im);
  const auto sc = scratch_of(im);
  const auto pl = plan_of(*app, im);
  cudaEvent_t ev[64];
  for (int i = 0; i <= n_k; ++i) RW_CUDA(cudaEventCreate(&ev[i]));
  for (int i = 0; i < n_k; ++i) kernel_ms[i] = 0.0f;
  int rc = RW_OK;
  for (int r = 0; r < reps && rc == RW_OK; ++r) {
    rc = clear_all(im, s);
    if (rc != RW_OK) break;
    cudaEventRecord(ev[0], s);
    cudaError_t e = rwt::launch_keys(b, sc, pl, false, true, s);
    cudaEventRecord(ev[1], s);
    if (e == cudaSuccess) e = rwt::launch_sort_passes(b, sc, pl, s, ev + 2);
    if (e != cudaSuccess) {
      rc = cuda_fail(e, "rw_tree_sort_profile");
      break;
    }
    rc = sync_status(im, s);
    for (int i = 0; rc == RW_OK && i < n_k; ++i) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      kernel_ms[i] += ms / float(reps);
    }
  }
  for (int i = 0; i <= n_k; ++i) cudaEventDestroy(ev[i]);
  if (n_kernels) *n_kernels = n_k;
  return rc;
}

int rw_tree_sort_lookback_probe(rw_tree_app_data* app, rw_tree_im_storage* im,
                                uint32_t spin_limit, rw_stream_t stream) {
  if (int rc = check(app, im, kKeys | kAlt)) return rc;
  if (spin_limit == 0) return RW_ERR_ARG;
  if (rwt::div_up(app->n_input, rwt::sort_variant_tile(im->sort_variant)) < 2)
    return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = clear_all(im, s)) return rc;
  RW_CUDA(rwt::launch_sort_lookback_probe(bufs_of(*app, im), scratch_of(im), plan_of(*app, im),
                                          spin_limit, s));
  return sync_status(im, s);
}

// ---- stage 3: unique (cu_dispatcher.cu:597-627) -------------------------------
int rw_tree_run_stage3(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream) {
  if (int rc = check(app, im, kKeys | kAlt)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = clear_all(im, s)) return rc;
  RW_CUDA(rwt::launch_unique(bufs_of(*app, im), scratch_of(im), plan_of(*app, im), s));
  if (int rc = sync_status(im, s)) return rc;
  app->n_unique = im->h_status->n_unique;
  app->n_brt_nodes = app->n_unique - 1;
  return RW_OK;
}

// ---- stage 4: radix tree (cu_dispatcher.cu:633-648) ---------------------------
int rw_tree_run_stage4(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream) {
  if (int rc = check(app, im, kKeys | kBrt)) return rc;
  if (app->n_unique == RW_COUNT_UNSET) return RW_ERR_NOT_READY;
  if (app->n_unique < 3 || app->n_unique > app->n_input) return RW_ERR_DEGENERATE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = upload_counts(app, im, s)) return rc;
  RW_CUDA(rwt::launch_radix_tree(bufs_of(*app, im), scratch_of(im), plan_of(*app, im), false,
                                 s));
  if (geometric_delta(im))
    RW_CUDA(rwt::launch_prefix_shift(bufs_of(*app, im), scratch_of(im), plan_of(*app, im), s));
  return sync_status(im, s);
}

// ---- stage 5: edge count (cu_dispatcher.cu:654-666) ---------------------------
int rw_tree_run_stage5(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream) {
  if (int rc = check(app, im, kBrt | kEdge)) return rc;
  if (app->n_unique == RW_COUNT_UNSET) return RW_ERR_NOT_READY;
  if (app->n_unique < 3 || app->n_unique > app->n_input) return RW_ERR_DEGENERATE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = upload_counts(app, im, s)) return rc;
  RW_CUDA(rwt::launch_edge_count(bufs_of(*app, im), scratch_of(im), plan_of(*app, im), s));
  return sync_status(im, s);
}

// ---- stage 6: exclusive scan (cu_dispatcher.cu:672-686) -----------------------
int rw_tree_run_stage6(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream) {
  if (int rc = check(app, im, kEdge)) return rc;
  if (app->n_unique == RW_COUNT_UNSET) return RW_ERR_NOT_READY;
  if (app->n_unique < 3 || app->n_unique > app->n_input) return RW_ERR_DEGENERATE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = clear_all(im, s)) return rc;
  if (int rc = upload_counts(app, im, s)) return rc;
  RW_CUDA(rwt::launch_edge_scan(bufs_of(*app, im), scratch_of(im), plan_of(*app, im), s));
  if (int rc = sync_status(im, s)) return rc;
  app->n_octree_nodes = im->h_status->n_octree_nodes;
  return RW_OK;
}

// ---- stage 7: octree (cu_dispatcher.cu:692-752) -------------------------------
int rw_tree_run_stage7(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream) {
  if (int rc = check(app, im, kKeys | kBrt | kEdge | kOct)) return rc;
  if (app->n_unique == RW_COUNT_UNSET || app->n_octree_nodes == RW_COUNT_UNSET)
    return RW_ERR_NOT_READY;
  if (app->n_unique < 3 || app->n_unique > app->n_input) return RW_ERR_DEGENERATE;
  if (uint64_t(app->n_octree_nodes) + 1 > app->oct_capacity) return RW_ERR_CAPACITY;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = upload_counts(app, im, s)) return rc;
  RW_CUDA(rwt::launch_octree(bufs_of(*app, im), scratch_of(im), plan_of(*app, im), s));
  if (im->options & RW_TREE_OPT_LINK_LEAVES)
    RW_CUDA(rwt::launch_leaf_links(bufs_of(*app, im), scratch_of(im), plan_of(*app, im), s));
  return sync_status(im, s);
}

// ---- fused pipeline ----------------------------------------------------------
namespace {

// Enqueues the fused pipeline.  When `ev` is given, an event is recorded
// before the first launch and after every kernel launch (profiling only).
int enqueue_impl(rw_tree_app_data* app, rw_tree_im_storage* im, cudaStream_t s,
                 cudaEvent_t* ev, int* n_ev) {
  if (int rc = check(app, im, kPoints | kKeys | kAlt | kBrt | kEdge | kOct)) return rc;
  int k = 0;
  auto mark = [&]() -> cudaError_t {
    return ev ? cudaEventRecord(ev[k++], s) : cudaSuccess;
  };
  if (int rc = clear_all(im, s)) return rc;
  const auto b = bufs_of(*app, im);
  const auto sc = scratch_of(im);
  const auto pl = plan_of(*app, im);
  RW_CUDA(mark());
  if (im->learned) {
    // stage 1 without the digit histograms, then the learned-CDF sort (which
    // waits for its bucket plan once, and falls back to onesweep on `im`)
    RW_CUDA(rwt::launch_keys(b, sc, pl, true, false, s));
    RW_CUDA(mark());
    if (int rc = rwt::learned_sort_enqueue(im->learned, static_cast<const uint32_t*>(b.keys),
                                           static_cast<uint32_t*>(b.alt), app->n_input,
                                           im->learned_mode, im, false, s))
      return rc;
    RW_CUDA(mark());
  } else {
    RW_CUDA(rwt::launch_keys(b, sc, pl, true, true, s));
    RW_CUDA(mark());
    RW_CUDA(rwt::launch_sort_passes(b, sc, pl, s, ev ? ev + k : nullptr));
    if (ev) k += 1 + im->passes;
  }
  RW_CUDA(rwt::launch_unique(b, sc, pl, s));
  RW_CUDA(mark());
  if (geometric_delta(im)) {
    // the tree with the reference's delta, every prefix lowered by one, then
    // the edge counts from the lowered prefixes
    RW_CUDA(rwt::launch_radix_tree(b, sc, pl, false, s));
    RW_CUDA(rwt::launch_prefix_shift(b, sc, pl, s));
    RW_CUDA(rwt::launch_edge_count(b, sc, pl, s));
  } else {
    RW_CUDA(rwt::launch_radix_tree(b, sc, pl, true, s));
  }
  RW_CUDA(mark());
  RW_CUDA(rwt::launch_edge_sums(b, sc, pl, s));
  RW_CUDA(mark());
  RW_CUDA(rwt::launch_octree(b, sc, pl, s, ev ? ev + k : nullptr, true));
  if (ev) k += 2;
  if (im->options & RW_TREE_OPT_LINK_LEAVES) RW_CUDA(rwt::launch_leaf_links(b, sc, pl, s));
  RW_CUDA(cudaMemcpyAsync(im->h_status, im->d_status, sizeof(rwt::DevStatus),
                          cudaMemcpyDeviceToHost, s));
  if (n_ev) *n_ev = k;
  return RW_OK;
}

}  // namespace

int rw_tree_pipeline_enqueue(rw_tree_app_data* app, rw_tree_im_storage* im,
                             rw_stream_t stream) {
  return enqueue_impl(app, im, reinterpret_cast<cudaStream_t>(stream), nullptr, nullptr);
}

const char* rw_tree_pipeline_kernel_names(const rw_tree_im_storage* im) {
  static thread_local std::string names;
  if (im && im->learned) {
    names = "morton,learned_sort";
  } else {
    names = "morton_histogram,sort_init";
    for (int p = 0; p < (im ? im->passes : 0); ++p) names += ",sort_pass" + std::to_string(p);
  }
  names += ",unique,radix_tree_edges,edge_scan,octree,octree_far_links";
  return names.c_str();
}

int rw_tree_im_storage_set_learned(rw_tree_im_storage* im, rw_tree_learned* learned,
                                   int32_t mode) {
  if (!im || (mode != RW_LEARNED_MLP && mode != RW_LEARNED_SAMPLE_QUANTILES) ||
      (learned && im->key_bits != 32))
    return RW_ERR_ARG;
  im->learned = learned;
  im->learned_mode = mode;
  im->learned_stats = rw_tree_learned_stats{};
  return RW_OK;
}

int rw_tree_im_storage_learned_stats(const rw_tree_im_storage* im, rw_tree_learned_stats* out) {
  if (!im || !out) return RW_ERR_ARG;
  *out = im->learned_stats;
  return RW_OK;
}

int rw_tree_pipeline_profile(rw_tree_app_data* app, rw_tree_im_storage* im,
                             rw_stream_t stream, int32_t reps, float* kernel_ms,
                             int32_t max_kernels, int32_t* n_kernels) {
  if (!app || !im || !kernel_ms || reps < 1) return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int n_k = 7 + (im->learned ? 0 : im->passes);
  if (max_kernels < n_k) return RW_ERR_ARG;
  cudaEvent_t ev[64];
  for (int i = 0; i <= n_k; ++i) RW_CUDA(cudaEventCreate(&ev[i]));
  for (int i = 0; i < n_k; ++i) kernel_ms[i] = 0.0f;
  int rc = RW_OK;
  for (int r = 0; r < reps && rc == RW_OK; ++r) {
    int n_ev = 0;
    rc = enqueue_impl(app, im, s, ev, &n_ev);
    if (rc == RW_OK) rc = rw_tree_pipeline_finish(app, im, stream);
    for (int i = 0; rc == RW_OK && i + 1 < n_ev && i < n_k; ++i) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      kernel_ms[i] += ms / float(reps);
    }
  }
  for (int i = 0; i <= n_k; ++i) cudaEventDestroy(ev[i]);
  if (n_kernels) *n_kernels = n_k;
  return rc;
}

int rw_tree_pipeline_finish(rw_tree_app_data* app, rw_tree_im_storage* im,
                            rw_stream_t stream) {
  if (!app || !im) return RW_ERR_ARG;
  RW_CUDA(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)));
  if (im->learned) rwt::learned_last_stats(im->learned, &im->learned_stats);
  const rwt::DevStatus st = *im->h_status;
  app->n_unique = st.n_unique;
  app->n_brt_nodes = st.n_unique - 1;
  if (st.err != 0) {
    char buf[96];
    std::snprintf(buf, sizeof buf, "device error %d at site %u", st.err, st.err_site);
    g_last_error = buf;
    if (st.err != RW_ERR_DEGENERATE) app->n_octree_nodes = st.n_octree_nodes;
    return st.err;
  }
  app->n_octree_nodes = st.n_octree_nodes;
  return RW_OK;
}

int rw_tree_host_submit(rw_tree_app_data* app, rw_tree_im_storage* im, const float* h_points,
                        rw_stream_t stream) {
  if (!h_points) return RW_ERR_ARG;
  if (int rc = check(app, im, kPoints | kKeys | kAlt | kBrt | kEdge | kOct)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  RW_CUDA(cudaMemcpyAsync(app->u_input_points, h_points, size_t(16) * app->n_input,
                          cudaMemcpyHostToDevice, s));
  return rw_tree_pipeline_enqueue(app, im, stream);
}

int rw_tree_host_collect(rw_tree_app_data* app, rw_tree_im_storage* im,
                         rw_tree_host_out* h_out, rw_stream_t stream) {
  if (int rc = rw_tree_pipeline_finish(app, im, stream)) return rc;
  if (!h_out) return RW_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t ks = key_size(app->key_bits);
  const size_t n = app->n_input, u = app->n_unique, b = app->n_brt_nodes,
               m = app->n_octree_nodes;
  auto d2h = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    if (!dst || bytes == 0) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
  };
  RW_CUDA(d2h(h_out->sorted_keys, app->u_morton_keys_alt, ks * n));
  RW_CUDA(d2h(h_out->unique_keys, app->u_morton_keys, ks * u));
  RW_CUDA(d2h(h_out->prefix_n, app->brt_prefix_n, b));
  RW_CUDA(d2h(h_out->has_leaf_left, app->brt_has_leaf_left, b));
  RW_CUDA(d2h(h_out->has_leaf_right, app->brt_has_leaf_right, b));
  RW_CUDA(d2h(h_out->left_child, app->brt_left_child, 4 * b));
  RW_CUDA(d2h(h_out->parents, app->brt_parents, 4 * b));
  RW_CUDA(d2h(h_out->edge_count, app->u_edge_count, 4 * b));
  RW_CUDA(d2h(h_out->edge_offset, app->u_edge_offset, 4 * b));
  RW_CUDA(d2h(h_out->children, app->oct_children, 32 * m));
  RW_CUDA(d2h(h_out->corner, app->oct_corner, 16 * m));
  RW_CUDA(d2h(h_out->cell_size, app->oct_cell_size, 4 * m));
  RW_CUDA(d2h(h_out->child_node_mask, app->oct_child_node_mask, 4 * m));
  RW_CUDA(d2h(h_out->child_leaf_mask, app->oct_child_leaf_mask, 4 * m));
  return RW_OK;
}

int rw_tree_run_host(rw_tree_app_data* app, rw_tree_im_storage* im,
                     const float* h_points, rw_tree_host_out* h_out,
                     rw_stream_t stream) {
  if (int rc = rw_tree_host_submit(app, im, h_points, stream)) return rc;
  if (int rc = rw_tree_host_collect(app, im, h_out, stream)) return rc;
  RW_CUDA(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)));
  return RW_OK;
}

}  // extern "C"
