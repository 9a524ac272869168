/* rw_tree.h - C ABI of the B200 tree pipeline (point cloud -> octree).
 *
 * Drop-in for the CUDA path of ucsc-redwood/redwood-comp's tree app.  Every
 * entry point takes plain pointers and sizes.  The reference interfaces each
 * one replaces are cited beside it (paths inside the reference project).
 *
 * Buffers: `rw_tree_app_data` mirrors the reference's `AppData`
 * (apps/tree/app_data.hpp:15-158) field by field; the caller owns every buffer
 * (device or managed memory, as the reference's pmr memory resource decides,
 * redwood/cuda/cu_mem_resource.cu:9-27).  Scratch lives in an
 * `rw_tree_im_storage` (the reference's `cuda::ImStorage`,
 * apps/tree/cuda/im_storage.cuh:10-42), allocated by the library.
 *
 * Buffer contract (app_data.hpp:139-157): stage 2 leaves the sorted keys in
 * u_morton_keys_alt, stage 3 leaves the unique keys in u_morton_keys.
 * Every output is bit-exact with the reference's functions unless an option
 * of rw_tree_im_storage_set_options says otherwise.
 *
 * Errors: every call returns RW_OK (0) or an rw_status code; the C++ layer in
 * redwood_tree/ turns a non-zero code into std::runtime_error as the
 * reference's CUDA_CHECK does (redwood/cuda/helpers.cuh:12-20).
 */
#ifndef RW_TREE_H
#define RW_TREE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same type as cudaStream_t (CUstream_st*), declared here so that callers
 * need no CUDA headers.  NULL is the legacy default stream. */
typedef struct CUstream_st* rw_stream_t;

typedef enum rw_status {
  RW_OK = 0,
  RW_ERR_ARG = 1,        /* null pointer, n out of range, bad key width */
  RW_ERR_DEGENERATE = 2, /* fewer than 3 distinct keys: the reference's root
                            range [0, n_brt-1] (func_brt.hpp:80-83) is empty */
  RW_ERR_CAPACITY = 3,   /* n_octree_nodes + 1 exceeds the octree rows
                            (AppData allocates floor(0.6 n), app_data.hpp:28) */
  RW_ERR_CUDA = 4,       /* a CUDA runtime call failed (rw_tree_last_error) */
  RW_ERR_TIMEOUT = 5,    /* a device-side bounded wait gave up */
  RW_ERR_NOT_READY = 6,  /* a stage ran before the stage that sets its count */
  RW_ERR_NO_DEVICE = 7   /* no usable CUDA device / kernel image */
} rw_status;

#define RW_COUNT_UNSET 0xffffffffu
/* Largest point count: look-back descriptors carry 30-bit values. */
#define RW_MAX_POINTS ((uint32_t)1 << 30)

/* Mirror of AppData (app_data.hpp:15-96).  Counts start at RW_COUNT_UNSET
 * (the reference's numeric_limits<uint32_t>::max(), :49-51) and are set by
 * stages 3 and 6.  Keys are uint32_t (key_bits 32: 10 bits per axis, the
 * reference) or uint64_t (key_bits 64: 21 bits per axis, no reference
 * counterpart). */
typedef struct rw_tree_app_data {
  uint32_t n_input;
  uint32_t oct_capacity; /* rows of every oct_* buffer */
  int32_t key_bits;      /* 32 or 64 */
  float min_coord;       /* AppData::min_coord (0.0f) */
  float range;           /* AppData::range (1024.0f) */
  uint32_t n_unique;
  uint32_t n_brt_nodes;
  uint32_t n_octree_nodes;
  float* u_input_points;      /* [4 n] x y z w (glm::vec4) */
  void* u_morton_keys;        /* [n] */
  void* u_morton_keys_alt;    /* [n] */
  int32_t* u_edge_count;      /* [n] */
  int32_t* u_edge_offset;     /* [n] */
  uint8_t* brt_prefix_n;      /* [n] RadixTree (app_data.hpp:63-76) */
  uint8_t* brt_has_leaf_left; /* [n] */
  uint8_t* brt_has_leaf_right;/* [n] */
  int32_t* brt_left_child;    /* [n] */
  int32_t* brt_parents;       /* [n] */
  int32_t* oct_children;      /* [8 cap] Octree (app_data.hpp:78-96) */
  float* oct_corner;          /* [4 cap] */
  float* oct_cell_size;       /* [cap] */
  int32_t* oct_child_node_mask; /* [cap] */
  int32_t* oct_child_leaf_mask; /* [cap] stays 0: the reference never links
                                   leaves (cu_dispatcher.cu:738-749) */
} rw_tree_app_data;

/* Opaque scratch: sort histograms and look-back descriptors, the ping-pong
 * key buffer, device-side counts and the error word. */
typedef struct rw_tree_im_storage rw_tree_im_storage;

/* Opaque scratch of the learned-CDF sort (see its section below). */
typedef struct rw_tree_learned rw_tree_learned;

/* Octree rows for n points: floor(n * 0.6f) in float (app_data.hpp:13,28). */
uint32_t rw_tree_octree_capacity(uint32_t n_input);

/* Fills `app` for n points: counts unset, min 0, range 1024, buffers NULL. */
void rw_tree_app_data_init(rw_tree_app_data* app, uint32_t n_input,
                           int32_t key_bits);

/* ImStorage(int n) (im_storage.cuh:11, im_storage.cu:29-40): allocates the
 * scratch for up to n_input points on the current device. */
int rw_tree_im_storage_create(uint32_t n_input, int32_t key_bits,
                              rw_tree_im_storage** out);
/* Same, with the sort's digit width chosen: 8, 10 or 11 bits (0 = default 8).
 * The reference fixes 8-bit digits (cu_dispatcher.cu:25-27). */
int rw_tree_im_storage_create_ex(uint32_t n_input, int32_t key_bits,
                                 int32_t radix_bits, rw_tree_im_storage** out);
/* The onesweep sort comes in a menu of variants (threads per CTA, keys per
 * thread, warp ranking scheme: 0 ballot multi-split, 1 match.any,
 * 2 shared-memory atomic OR, 3 half-warp packed words, 4 atomic OR with the
 * top pass by ballots over its remaining bits) for each key and digit width; the autotuner
 * picks one per size class.  No reference counterpart (the reference fixes
 * 512 threads x 15 keys with ballots, cu_dispatcher.cu:44-49). */
int rw_tree_sort_variant_count(void);
int rw_tree_sort_variant_info(int32_t idx, int32_t* key_bits, int32_t* radix_bits,
                              int32_t* threads, int32_t* keys_per_thread,
                              int32_t* rank_mode);
/* Selects variant idx (its key and digit width must match the storage). */
int rw_tree_im_storage_set_sort_variant(rw_tree_im_storage* im, int32_t idx);
/* Options that change the reference's outputs on purpose, both off by
 * default (0 keeps every output bit-exact with the reference):
 *   RW_TREE_OPT_GEOMETRIC_DELTA - the radix tree's delta is clz(a ^ b) - 2
 *     for 32-bit keys, the true common-prefix length of 30-bit codes, so that
 *     octree levels and child links are geometrically exact.  The reference's
 *     delta_u32 is clz - 1 (func_brt.hpp:27-33), written for 31-bit codes.
 *     64-bit codes are 63 bits wide and their clz - 1 is already exact, so
 *     the option changes nothing for them.
 *   RW_TREE_OPT_LINK_LEAVES - after the octree, the reference's leaf linker
 *     process_link_leaf (func_octree.hpp:114-163; k_LinkLeafNodes,
 *     07_octree.cu:228-258, whose launch cu_dispatcher.cu:738-749 leaves
 *     commented out) for every radix-tree node, with the result of running
 *     them in ascending order: each leaf index goes into its slot of the
 *     bottom octree row of the nearest ancestor that owns rows, and the
 *     slot's child_leaf_mask bit is cleared (set_leaf, func_octree.hpp:18-25).
 *     The walk up the tree stops after 31 steps (the reference's CPU walk has
 *     no bound and never ends at a root without rows).
 * Applies to the stage calls and the fused pipeline of this scratch. */
#define RW_TREE_OPT_GEOMETRIC_DELTA 1
#define RW_TREE_OPT_LINK_LEAVES 2
int rw_tree_im_storage_set_options(rw_tree_im_storage* im, int32_t options);
/* ~ImStorage (im_storage.cu:42-52). */
int rw_tree_im_storage_destroy(rw_tree_im_storage* im);
/* ImStorage::clearSmem (im_storage.cu:53-60): zeroes histograms, descriptors
 * and the error word on `stream`.  The stage calls do this themselves. */
int rw_tree_im_storage_clear(rw_tree_im_storage* im, rw_stream_t stream);

/* cuda::run_stage1..7 (apps/tree/cuda/cu_dispatcher.cuh:8-19,
 * cu_dispatcher.cu:501-752).  Synchronous like the reference: each call ends
 * with a stream synchronisation and updates the counts in `app`.  The
 * reference passes ImStorage to stages 2 and 3 only; here every stage takes it
 * (the C++ layer supplies an internal one where the reference signature has
 * none).
 *   1: u_input_points -> u_morton_keys                         (01_morton.cu)
 *   2: u_morton_keys -> u_morton_keys_alt, ascending          (onesweep sort)
 *   3: u_morton_keys_alt -> u_morton_keys unique, n_unique    (03_unique.cu)
 *   4: unique keys -> brt_* for i in [0, n_brt)             (04_radix_tree.cu)
 *   5: brt -> u_edge_count                                 (05_edge_count.cu)
 *   6: u_edge_count -> u_edge_offset (exclusive), n_octree_nodes
 *                                                         (06_prefix_sum.cu)
 *   7: everything -> oct_* rows [0, n_octree_nodes)          (07_octree.cu) */
int rw_tree_run_stage1(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream);
int rw_tree_run_stage2(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream);
int rw_tree_run_stage3(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream);
int rw_tree_run_stage4(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream);
int rw_tree_run_stage5(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream);
int rw_tree_run_stage6(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream);
int rw_tree_run_stage7(rw_tree_app_data* app, rw_tree_im_storage* im,
                       rw_stream_t stream);

/* All seven stages as one asynchronous sequence on `stream` (the loop body of
 * pipe_main_baseline.cpp:55-92 without its per-stage host synchronisations):
 * fused kernels, counts kept on the device, no host round trip.  Capturable
 * into a CUDA graph.  Outputs are identical to stages 1..7 run one by one.
 * rw_tree_pipeline_finish waits for the stream, copies the counts into `app`
 * and reports any device-side error. */
int rw_tree_pipeline_enqueue(rw_tree_app_data* app, rw_tree_im_storage* im,
                             rw_stream_t stream);
int rw_tree_pipeline_finish(rw_tree_app_data* app, rw_tree_im_storage* im,
                            rw_stream_t stream);

/* Per-kernel device times of the fused pipeline, the role of the reference's
 * per-stage google-benchmark fixtures (apps/tree/bm_cuda.cpp:25-123): runs
 * the pipeline `reps` times with a CUDA event after every kernel and writes
 * the mean milliseconds of each kernel to kernel_ms (order and names as in
 * rw_tree_pipeline_kernel_names, comma separated). */
int rw_tree_pipeline_profile(rw_tree_app_data* app, rw_tree_im_storage* im,
                             rw_stream_t stream, int32_t reps, float* kernel_ms,
                             int32_t max_kernels, int32_t* n_kernels);
const char* rw_tree_pipeline_kernel_names(const rw_tree_im_storage* im);

/* Host-side result buffers for rw_tree_run_host; any pointer may be NULL. */
typedef struct rw_tree_host_out {
  void* sorted_keys;          /* [n] */
  void* unique_keys;          /* [n_unique] */
  uint8_t* prefix_n;          /* [n_brt] */
  uint8_t* has_leaf_left;
  uint8_t* has_leaf_right;
  int32_t* left_child;
  int32_t* parents;
  int32_t* edge_count;
  int32_t* edge_offset;
  int32_t* children;          /* [8 n_octree_nodes] */
  float* corner;              /* [4 n_octree_nodes] */
  float* cell_size;           /* [n_octree_nodes] */
  int32_t* child_node_mask;
  int32_t* child_leaf_mask;
} rw_tree_host_out;

/* End to end from host memory, the way the reference's callers use managed
 * AppData (apps/tree/main.cpp:48-88): copies h_points ([4 n] floats) into
 * app->u_input_points, runs the pipeline, reads the counts and copies the
 * requested outputs back.  Pinned host buffers give full PCIe bandwidth. */
int rw_tree_run_host(rw_tree_app_data* app, rw_tree_im_storage* im,
                     const float* h_points, rw_tree_host_out* h_out,
                     rw_stream_t stream);
/* rw_tree_run_host in two halves, for streaming many clouds: submit copies
 * h_points in and enqueues the pipeline, without waiting; collect waits for
 * that run's counts (rw_tree_pipeline_finish) and enqueues the copies of the
 * requested outputs, without waiting for them (h_out is complete once
 * `stream` has drained).  With two AppData/scratch pairs on two streams, a
 * caller alternating submit(k) and collect(k-1) overlaps one cloud's copies
 * back with the next cloud's copies in and its pipeline. */
int rw_tree_host_submit(rw_tree_app_data* app, rw_tree_im_storage* im, const float* h_points,
                        rw_stream_t stream);
int rw_tree_host_collect(rw_tree_app_data* app, rw_tree_im_storage* im,
                         rw_tree_host_out* h_out, rw_stream_t stream);

/* Seeded synthetic point clouds, generated on the host.
 *   RW_GEN_APPDATA: AppData's own generator (app_data.hpp:32-39):
 *     std::mt19937(seed), uniform_real_distribution<float>(min, min+range),
 *     w = 1.  The reference writes glm::vec4(dis(gen), dis(gen), dis(gen), 1)
 *     whose argument order C++ leaves unspecified; g++ builds of it draw z,
 *     then y, then x, and so does this generator.
 *   RW_GEN_UNIFORM: counter-based (splitmix64) uniform in [min, min+range).
 *   RW_GEN_GAUSSIAN_MIXTURE: counter-based isotropic Gaussian mixture with
 *     n_components centres uniform in the box, sigma uniform in
 *     [sigma_lo, sigma_hi], equal weights, clamped into the box. */
typedef enum rw_gen_kind {
  RW_GEN_APPDATA = 0,
  RW_GEN_UNIFORM = 1,
  RW_GEN_GAUSSIAN_MIXTURE = 2
} rw_gen_kind;

int rw_tree_generate_points(float* out, uint64_t n, int32_t kind,
                            uint64_t seed, float min_coord, float range,
                            int32_t n_components, float sigma_lo,
                            float sigma_hi);

/* ---- batched form: many clouds in one pass of launches --------------------
 * No reference counterpart (the reference builds one cloud per call,
 * pipe_main_baseline.cpp:55-92).  Clouds are stored back to back: cloud c's
 * points, keys, radix-tree and edge arrays occupy [point_offset[c],
 * point_offset[c+1]) of the concatenated buffers, its octree rows
 * [octree_offset[c], octree_offset[c+1]) with floor(0.6f * n_c) rows per cloud
 * as AppData allocates.  Every kernel runs once for the whole batch; each
 * cloud's outputs equal a plain run on that cloud alone. */
typedef struct rw_tree_batch rw_tree_batch;

typedef struct rw_tree_batch_buffers {
  float* points;             /* [4 n_total] */
  void* morton_keys;         /* [n_total] unique keys of each cloud after the run */
  void* morton_keys_alt;     /* [n_total] sorted keys of each cloud */
  int32_t* edge_count;       /* [n_total] */
  int32_t* edge_offset;      /* [n_total] */
  uint8_t* prefix_n;         /* [n_total] */
  uint8_t* has_leaf_left;
  uint8_t* has_leaf_right;
  int32_t* left_child;
  int32_t* parents;
  int32_t* children;         /* [8 octree_rows] */
  float* corner;             /* [4 octree_rows] */
  float* cell_size;          /* [octree_rows] */
  int32_t* child_node_mask;
  int32_t* child_leaf_mask;
} rw_tree_batch_buffers;

/* Plans a batch of n_clouds clouds of the given sizes (each >= 1) and
 * allocates its scratch on the current device.  Cloud c gets
 * floor(n_c * octree_ratio) octree rows (at least 1), computed in float as
 * AppData does with its 0.6f (app_data.hpp:13,28); octree_ratio <= 0 means
 * 0.6f.  Small uniform clouds can need more than 0.6 n rows: their status is
 * then RW_ERR_CAPACITY, exactly as a plain run with that capacity reports. */
int rw_tree_batch_create(const uint32_t* cloud_sizes, uint32_t n_clouds, int32_t key_bits,
                         int32_t radix_bits, float octree_ratio, rw_tree_batch** out);
int rw_tree_batch_destroy(rw_tree_batch* batch);
uint32_t rw_tree_batch_total_points(const rw_tree_batch* batch);
uint32_t rw_tree_batch_octree_rows(const rw_tree_batch* batch);
/* point_offsets and octree_offsets: [n_clouds + 1] each (either may be NULL). */
int rw_tree_batch_offsets(const rw_tree_batch* batch, uint32_t* point_offsets,
                          uint32_t* octree_offsets);
/* One onesweep variant for every cloud. */
int rw_tree_batch_set_sort_variant(rw_tree_batch* batch, int32_t idx);
/* Size classes of the sort (at most 4): a cloud of n points runs variant
 * variants[k] for the first k with n <= max_points[k] (the last class takes
 * every larger cloud).  The autotuner writes these tables. */
int rw_tree_batch_set_classes(rw_tree_batch* batch, uint32_t n_classes,
                              const uint32_t* max_points, const int32_t* variants);
/* Stage 2 of every cloud by the learned-CDF sort (32-bit keys), one sort per
 * cloud enqueued back to back (each decides its onesweep fallback on the
 * device, on `fallback_im`, so the batch stays capturable); the other stages
 * stay one launch for the whole batch.  `learned` must serve the largest
 * cloud, `fallback_im` hold storage for it, and both outlive their use here;
 * NULL restores the batched onesweep sort.  Outputs are identical either way. */
int rw_tree_batch_set_learned(rw_tree_batch* batch, rw_tree_learned* learned, int32_t mode,
                              rw_tree_im_storage* fallback_im);
/* All stages for every cloud, asynchronous on `stream` (capturable). */
int rw_tree_batch_enqueue(rw_tree_batch* batch, const rw_tree_batch_buffers* bufs,
                          rw_stream_t stream);
/* The same through a CUDA graph: captured on the first call for a buffer set
 * (and again when the buffers or the sort variant change), then replayed. */
int rw_tree_batch_graph_launch(rw_tree_batch* batch, const rw_tree_batch_buffers* bufs,
                               rw_stream_t stream);
/* Waits for the stream; per-cloud n_unique, n_octree_nodes and status
 * (rw_status: RW_ERR_DEGENERATE / RW_ERR_CAPACITY for that cloud), each
 * [n_clouds] (NULL to skip).  Returns RW_ERR_TIMEOUT if a device-side wait
 * gave up. */
int rw_tree_batch_finish(rw_tree_batch* batch, rw_stream_t stream, uint32_t* n_unique,
                         uint32_t* n_octree_nodes, int32_t* status);

/* Stage 2 alone, asynchronous on `stream` (no synchronisation, capturable):
 * sorts app->u_morton_keys[0, n) into app->u_morton_keys_alt with the onesweep
 * sort.  Only the two key buffers of `app` are used. */
int rw_tree_sort_enqueue(rw_tree_app_data* app, rw_tree_im_storage* im, rw_stream_t stream);
/* The same sort `reps` times with CUDA events between its kernels; mean
 * device milliseconds of the digit histogram, the pass set-up and each pass
 * (2 + passes entries, in that order) into kernel_ms.  Synchronous. */
int rw_tree_sort_profile(rw_tree_app_data* app, rw_tree_im_storage* im, rw_stream_t stream,
                         int32_t reps, float* kernel_ms, int32_t max_kernels,
                         int32_t* n_kernels);

/* Test hook of the sort's bounded wait.  The reference's look-back spins
 * without a bound (an unsigned `k >= 0` loop, cu_dispatcher.cu:376) and its
 * only error path is CUDA_CHECK (redwood/cuda/helpers.cuh:12-20); here every
 * wait gives up after a number of polls and reports RW_ERR_TIMEOUT.  This
 * call makes that happen on purpose, without any fault: it builds the digit
 * histograms of app->u_morton_keys, then runs the first onesweep pass into
 * app->u_morton_keys_alt with its first tile left out, so that every other
 * tile waits on a descriptor nothing publishes and gives up after spin_limit
 * polls.  Every write stays inside u_morton_keys_alt[0, n).  Needs at least
 * two tiles of keys; returns RW_ERR_TIMEOUT, and the scratch is fit for the
 * next normal run. */
int rw_tree_sort_lookback_probe(rw_tree_app_data* app, rw_tree_im_storage* im,
                                uint32_t spin_limit, rw_stream_t stream);

/* ---- learned-CDF bucketed sort (32-bit keys) -------------------------------
 * No reference counterpart.  A 64K-key stratified sample is sorted and 4,095
 * bucket boundaries are placed, one per 16 sample ranks: at the sample key of
 * rank 16(j+1) (plain sample quantiles, the method without the network), or
 * by the boundary MLP (16 -> 64 -> 64 -> 1, BF16 weights, FP32 accumulate),
 * which reads a context of 16*group sorted sample keys around that rank and
 * returns the boundary's offset from it in sample ranks; a prefix maximum
 * keeps the boundaries non-decreasing.  Keys are scattered into the 4,096
 * buckets in one pass, every bucket into a region of 4x the mean bucket size,
 * and each bucket is sorted exactly.  A bucket that overflows its region
 * sends the whole input to the onesweep sort.  The output is the sorted input
 * either way. */
#define RW_LEARNED_MLP 0
#define RW_LEARNED_SAMPLE_QUANTILES 1
#define RW_LEARNED_MLP_PARAMS 5313 /* 16*64 + 64 + 64*64 + 64 + 64 + 1 */
#define RW_LEARNED_MAX_GROUP 16    /* group: a power of two, 1..16 */

typedef struct rw_tree_learned_stats {
  uint32_t max_bucket;  /* keys in the fullest bucket */
  uint32_t big_buckets; /* buckets above one CTA's 32,768 keys (chunked path) */
  uint32_t fell_back;   /* 1 when a bucket overflowed and the onesweep sort ran */
  uint32_t mlp_timeout; /* 1 once a wait of the boundary network on the tensor cores
                           ran out (sticky for this scratch; the boundaries of that
                           tile stayed sample quantiles, the sort stays exact) */
} rw_tree_learned_stats;

/* Scratch for inputs of up to n_max (>= 65536) keys on the current device
 * (about 16 bytes per key of n_max, for the bucket regions). */
int rw_tree_learned_create(uint32_t n_max, rw_tree_learned** out);
int rw_tree_learned_destroy(rw_tree_learned* learned);
/* FP32 master parameters (RW_LEARNED_MLP_PARAMS floats, layout W1[64][16],
 * b1[64], W2[64][64], b2[64], W3[64], b3; used rounded to BF16) and the
 * context group size they were trained with. */
int rw_tree_learned_set_params(rw_tree_learned* learned, const float* params, int32_t count,
                               int32_t group);
/* Context group size alone (for rw_tree_learned_features); default 4. */
int rw_tree_learned_set_group(rw_tree_learned* learned, int32_t group);
/* Sorts d_keys[0, n) (16-byte aligned) into d_sorted.  With `fallback_im`
 * (storage for n keys) the call is asynchronous on `stream` and capturable in
 * a CUDA graph: the bucket sort and a onesweep sort on fallback_im are both
 * enqueued, and the plan's overflow word, on the device, lets exactly one of
 * them write d_sorted.  `stats` (may be NULL) is filled after one wait for
 * the stream.  Without fallback_im the call waits for the plan and returns
 * RW_ERR_CAPACITY on an overflow (and for n < 65,536) instead of sorting. */
int rw_tree_learned_sort(rw_tree_learned* learned, const uint32_t* d_keys, uint32_t* d_sorted,
                         uint32_t n, int32_t mode, rw_tree_im_storage* fallback_im,
                         rw_stream_t stream, rw_tree_learned_stats* stats);
/* Training data: the MLP inputs of the 4,095 boundaries for d_keys under the
 * current group size ([4095][16]; rows whose context does not fit inside the
 * sample are zero and such boundaries stay sample quantiles) and the sorted
 * sample ([65536]).  Host arrays, either may be NULL. */
int rw_tree_learned_features(rw_tree_learned* learned, const uint32_t* d_keys, uint32_t n,
                             float* features, uint32_t* sorted_sample, rw_stream_t stream);
/* Keys per bucket (host [4096]) under `mode`'s boundaries (d_keys 16-byte
 * aligned). */
int rw_tree_learned_bucket_counts(rw_tree_learned* learned, const uint32_t* d_keys, uint32_t n,
                                  int32_t mode, uint32_t* counts, rw_stream_t stream);

/* Stage 2 of this scratch's pipeline (rw_tree_run_stage2 and
 * rw_tree_pipeline_enqueue) sorts with `learned` in `mode` instead of the
 * onesweep sort; NULL restores onesweep.  32-bit keys only; `learned` must
 * serve n_input keys and outlive its use here.  The pipeline stays
 * asynchronous and capturable (the fallback is decided on the device), and
 * rw_tree_pipeline_profile reports "morton,learned_sort,..." (7 entries).
 * The output is bit-identical either way. */
int rw_tree_im_storage_set_learned(rw_tree_im_storage* im, rw_tree_learned* learned,
                                   int32_t mode);
/* The learned sort's statistics of the last run on this scratch. */
int rw_tree_im_storage_learned_stats(const rw_tree_im_storage* im,
                                     rw_tree_learned_stats* out);

/* Training kernels of the boundary MLP (device arrays).  x: [rows][16],
 * t: [rows]; mean squared error over `batch` examples (rows of this call may
 * be a part of the batch).  grad and loss_sum are accumulated into. */
int rw_tree_mlp_param_count(void);
int rw_tree_mlp_grad(const float* params, const float* x, const float* t, uint32_t rows,
                     uint32_t batch, float* grad, float* loss_sum, rw_stream_t stream);
/* Adam step (bias-corrected) on the FP32 master parameters; step >= 1. */
int rw_tree_mlp_adam(float* params, const float* grad, float* m, float* v, float lr,
                     float beta1, float beta2, float eps, int32_t step, rw_stream_t stream);
int rw_tree_mlp_forward(const float* params, const float* x, uint32_t rows, float* y,
                        rw_stream_t stream);

/* Stage 3 for callers that cannot allocate GPU memory (a host whose device
 * memory is all reserved by its own pool, a real-time loop that must not take
 * the driver's allocation locks, a plugin given only pointers and a stream).
 * No counterpart in the reference.  Same result as rw_tree_run_stage3: the
 * unique keys of sorted_keys[0, n) go to unique_keys and their count to
 * *n_unique (host memory); synchronous on `stream`.  Both key buffers must be
 * 16-byte aligned and must not overlap (RW_ERR_ARG otherwise: every tile
 * writes its output while other tiles still read the input).  Its scratch is a fixed
 * array inside the library (about 64 KiB on every GPU that loads it), so it
 * never allocates; n above RW_NOALLOC_MAX_KEYS is rejected with RW_ERR_ARG.
 * The first call on each device looks the array's address up (make that call
 * before any stream capture).  All calls share the array: calls that overlap
 * on the GPU race and must be serialised by the caller. */
#define RW_NOALLOC_MAX_KEYS ((uint32_t)1 << 26)
int rw_tree_unique_noalloc(const void* sorted_keys, void* unique_keys, uint32_t n,
                           int32_t key_bits, uint32_t* n_unique, rw_stream_t stream);

/* Text of the last CUDA error seen by this thread ("" if none). */
const char* rw_tree_last_error(void);
/* Library build tag (kernels compiled for sm_100a). */
const char* rw_tree_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RW_TREE_H */
