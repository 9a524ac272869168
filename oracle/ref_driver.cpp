// Test infrastructure: a project-written C-ABI driver around the reference's
// OWN CPU tree code, compiled from the reference sources in place (see
// oracle/Makefile).  Nothing in the product links this; only tests/ and the
// CPU-baseline leg of bench.py load it, as a checker or as the timed baseline.
//
// Three entry points:
//   ref_default_points  - AppData's seeded point generator (app_data.hpp:32-39)
//   ref_cpu_verbatim /  - the reference's cpu::run_stage1..7 exactly as
//   ref_cpu_time          pipe_main_baseline.cpp:15-45 drives them
//   ref_canonical       - the reference's per-element functions
//                         (func_morton.hpp, func_brt.hpp, func_edge.hpp,
//                         func_octree.hpp) wired with the buffer contract of
//                         app_data.hpp:139-157, a global exclusive scan for
//                         stage 6 and ascending-index order for stage 7.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory_resource>
#include <numeric>
#include <thread>
#include <vector>

#include "app_data.hpp"
#include "host/func_brt.hpp"
#include "host/func_edge.hpp"
#include "host/func_morton.hpp"
#include "host/func_octree.hpp"
#include "host/host_dispatchers.hpp"

namespace {

uint32_t octree_capacity(uint32_t n) {
  // AppData sizes its octree as n_input * k_memory_ratio (app_data.hpp:28).
  return static_cast<uint32_t>(static_cast<size_t>(n * k_memory_ratio));
}

void load_points(AppData& app, const float* pts) {
  std::memcpy(app.u_input_points.data(), pts,
              sizeof(float) * 4 * static_cast<size_t>(app.n_input));
}

}  // namespace

extern "C" {

struct ref_canonical_out {
  uint32_t* keys_after_stage1;  // [n]
  uint32_t* sorted_keys;        // [n]   u_morton_keys_alt after stage 2
  uint32_t* unique_keys;        // [n]   u_morton_keys after stage 3
  uint8_t* prefix_n;            // [n]
  uint8_t* has_leaf_left;       // [n]
  uint8_t* has_leaf_right;      // [n]
  int32_t* left_child;          // [n]
  int32_t* parents;             // [n]
  int32_t* edge_count;          // [n]
  int32_t* edge_offset;         // [n]
  int32_t* children;            // [8 * cap]
  float* corner;                // [4 * cap]
  float* cell_size;             // [cap]
  int32_t* child_node_mask;     // [cap]
  int32_t* child_leaf_mask;     // [cap]
  uint32_t n_unique;
  uint32_t n_brt_nodes;
  uint32_t n_octree_nodes;
  uint32_t capacity;
};

uint32_t ref_octree_capacity(uint32_t n) { return octree_capacity(n); }

int ref_default_points(float* out, uint32_t n) {
  AppData app(std::pmr::new_delete_resource(), n);
  std::memcpy(out, app.u_input_points.data(), sizeof(float) * 4 * size_t(n));
  return 0;
}

// Verbatim reference CPU pipeline.  Copies the stage-1 keys and the final
// counts (n_unique from stage 3, n_octree_nodes from stage 6).
int ref_cpu_verbatim(const float* pts, uint32_t n, int n_threads,
                     uint32_t* keys_after_stage1, uint32_t* counts_out) {
  if (n < 2 || n_threads < 1) return 1;
  AppData app(std::pmr::new_delete_resource(), n);
  load_points(app, pts);
  core::thread_pool pool(n_threads);
  const size_t t = static_cast<size_t>(n_threads);
  cpu::run_stage1(app, pool, t);
  if (keys_after_stage1)
    std::memcpy(keys_after_stage1, app.u_morton_keys.data(), 4 * size_t(n));
  cpu::run_stage2(app, pool, t);
  cpu::run_stage3(app, pool, t);
  cpu::run_stage4(app, pool, t);
  cpu::run_stage5(app, pool, t);
  cpu::run_stage6(app, pool, t);
  cpu::run_stage7(app, pool, t);
  if (counts_out) {
    counts_out[0] = app.get_n_unique();
    counts_out[1] = app.get_n_octree_nodes();
  }
  return 0;
}

// Times `iters` runs of the verbatim stages 1-7 on one AppData, the loop of
// pipe_main_baseline.cpp:21-44 (AppData construction and input generation
// excluded).  Writes each iteration's wall time in ms to per_iter_ms.
int ref_cpu_time(const float* pts, uint32_t n, int n_threads, int iters,
                 double* per_iter_ms) {
  if (n < 2 || n_threads < 1 || iters < 1) return 1;
  AppData app(std::pmr::new_delete_resource(), n);
  load_points(app, pts);
  core::thread_pool pool(n_threads);
  const size_t t = static_cast<size_t>(n_threads);
  for (int it = 0; it < iters; ++it) {
    const auto t0 = std::chrono::steady_clock::now();
    cpu::run_stage1(app, pool, t);
    cpu::run_stage2(app, pool, t);
    cpu::run_stage3(app, pool, t);
    cpu::run_stage4(app, pool, t);
    cpu::run_stage5(app, pool, t);
    cpu::run_stage6(app, pool, t);
    cpu::run_stage7(app, pool, t);
    const auto t1 = std::chrono::steady_clock::now();
    per_iter_ms[it] =
        std::chrono::duration<double, std::milli>(t1 - t0).count();
  }
  return 0;
}

// Canonical dataflow over the reference's own functions.  Returns 0 on
// success, 2 when fewer than 3 distinct keys exist (the reference's root range
// [0, n_brt-1] is empty below that), 3 when the octree overflows AppData's
// capacity.
static int canonical_impl(const float* pts, uint32_t n, int n_threads,
                          ref_canonical_out* out, bool link_leaves);

int ref_canonical(const float* pts, uint32_t n, int n_threads,
                  ref_canonical_out* out) {
  return canonical_impl(pts, n, n_threads, out, false);
}

// The same, then the reference's own leaf linker process_link_leaf
// (func_octree.hpp:114-163) for every radix-tree node in ascending order - the
// k_LinkLeafNodes launch the reference leaves commented out
// (cu_dispatcher.cu:738-749).  Its walk up the radix tree has no bound and
// never ends once it reaches the root without octree nodes (the root is its
// own parent); a cloud where some walk would get there returns 4 before any
// call, so that only clouds on which the reference's function is total are
// compared.
int ref_canonical_linked(const float* pts, uint32_t n, int n_threads,
                         ref_canonical_out* out) {
  return canonical_impl(pts, n, n_threads, out, true);
}

static int canonical_impl(const float* pts, uint32_t n, int n_threads,
                          ref_canonical_out* out, bool link_leaves) {
  if (n < 1 || n_threads < 1) return 1;
  AppData app(std::pmr::new_delete_resource(), n);
  load_points(app, pts);
  core::thread_pool pool(n_threads);
  const size_t t = static_cast<size_t>(n_threads);
  const uint32_t cap = octree_capacity(n);
  out->capacity = cap;

  // Stage 1 and the sorting passes of stage 2 are the reference's own
  // dispatchers.  Its 4 ping-pong passes leave the sorted keys in
  // u_morton_keys; the buffer contract (app_data.hpp:139-143) puts them in
  // u_morton_keys_alt, so they are copied there.
  cpu::run_stage1(app, pool, t);
  std::memcpy(out->keys_after_stage1, app.u_morton_keys.data(), 4 * size_t(n));
  if (n >= 2) {
    cpu::run_stage2(app, pool, t);
  }
  std::memcpy(app.u_morton_keys_alt.data(), app.u_morton_keys.data(),
              4 * size_t(n));
  std::memcpy(out->sorted_keys, app.u_morton_keys_alt.data(), 4 * size_t(n));

  // Stage 3: std::unique_copy (host_dispatchers.cpp:183-194) from the sorted
  // buffer into the unique buffer.
  const auto last = std::unique_copy(app.u_morton_keys_alt.data(),
                                     app.u_morton_keys_alt.data() + n,
                                     app.u_morton_keys.data());
  const auto n_unique =
      static_cast<uint32_t>(std::distance(app.u_morton_keys.data(), last));
  app.set_n_unique(n_unique);
  app.set_n_brt_nodes(n_unique - 1);
  out->n_unique = n_unique;
  out->n_brt_nodes = n_unique - 1;
  std::memcpy(out->unique_keys, app.u_morton_keys.data(), 4 * size_t(n));
  if (n_unique < 3) return 2;
  const int n_brt = static_cast<int>(n_unique - 1);

  // Stage 4: process_radix_tree_i for i in [0, n_brt), ascending.
  for (int i = 0; i < n_brt; ++i) {
    cpu::kernels::process_radix_tree_i(
        i, n_brt, app.get_unique_morton_keys(), app.brt.u_prefix_n.data(),
        app.brt.u_has_leaf_left.data(), app.brt.u_has_leaf_right.data(),
        app.brt.u_left_child.data(), app.brt.u_parents.data());
  }

  // Stage 5: process_edge_count_i for i in [0, n_brt).
  for (int i = 0; i < n_brt; ++i) {
    cpu::kernels::process_edge_count_i(i, app.brt.u_prefix_n.data(),
                                       app.brt.u_parents.data(),
                                       app.u_edge_count.data());
  }

  // Stage 6: global exclusive scan; the node count includes the last count.
  int32_t run = 0;
  for (int i = 0; i < n_brt; ++i) {
    app.u_edge_offset[i] = run;
    run += app.u_edge_count[i];
  }
  const uint32_t m = static_cast<uint32_t>(run);
  app.set_n_octree_nodes(m);
  out->n_octree_nodes = m;
  if (m >= cap) return 3;

  // Stage 7: the fresh AppData's octree buffers are zero (pmr vectors
  // value-initialise).  Root initialisation as cuda/07_octree.cu:188-198,
  // then process_oct_node for i = 1 .. n_brt-1 in ascending order.
  {
    const int root_level = app.brt.u_prefix_n[0] / 3;
    const uint32_t root_prefix =
        app.u_morton_keys[0] >> (cpu::kernels::morton_bits - 3 * root_level);
    cpu::kernels::morton32_to_xyz(
        &app.oct.u_corner[0],
        root_prefix << (cpu::kernels::morton_bits - 3 * root_level),
        app.min_coord, app.range);
    app.oct.u_cell_size[0] = app.range;
  }
  for (int i = 1; i < n_brt; ++i) {
    cpu::kernels::process_oct_node(
        i, reinterpret_cast<int(*)[8]>(app.oct.u_children.data()),
        app.oct.u_corner.data(), app.oct.u_cell_size.data(),
        app.oct.u_child_node_mask.data(), app.u_edge_offset.data(),
        app.u_edge_count.data(), app.get_unique_morton_keys(),
        app.brt.u_prefix_n.data(), app.brt.u_parents.data(), app.min_coord,
        app.range);
  }
  if (link_leaves) {
    for (int i = 0; i < n_brt; ++i) {
      if (!app.brt.u_has_leaf_left[i] && !app.brt.u_has_leaf_right[i]) continue;
      int rt = i, steps = 0;
      while (app.u_edge_count[rt] == 0 && steps <= 64) {
        rt = app.brt.u_parents[rt];
        ++steps;
      }
      if (app.u_edge_count[rt] == 0) return 4;
    }
    for (int i = 0; i < n_brt; ++i) {
      cpu::kernels::process_link_leaf(
          i, reinterpret_cast<int(*)[8]>(app.oct.u_children.data()),
          app.oct.u_child_leaf_mask.data(), app.u_edge_offset.data(),
          app.u_edge_count.data(), app.get_unique_morton_keys(),
          reinterpret_cast<const bool*>(app.brt.u_has_leaf_left.data()),
          reinterpret_cast<const bool*>(app.brt.u_has_leaf_right.data()),
          app.brt.u_prefix_n.data(), app.brt.u_parents.data(),
          app.brt.u_left_child.data());
    }
  }

  std::memcpy(out->prefix_n, app.brt.u_prefix_n.data(), size_t(n));
  std::memcpy(out->has_leaf_left, app.brt.u_has_leaf_left.data(), size_t(n));
  std::memcpy(out->has_leaf_right, app.brt.u_has_leaf_right.data(), size_t(n));
  std::memcpy(out->left_child, app.brt.u_left_child.data(), 4 * size_t(n));
  std::memcpy(out->parents, app.brt.u_parents.data(), 4 * size_t(n));
  std::memcpy(out->edge_count, app.u_edge_count.data(), 4 * size_t(n));
  std::memcpy(out->edge_offset, app.u_edge_offset.data(), 4 * size_t(n));
  std::memcpy(out->children, app.oct.u_children.data(), 32 * size_t(cap));
  std::memcpy(out->corner, app.oct.u_corner.data(), 16 * size_t(cap));
  std::memcpy(out->cell_size, app.oct.u_cell_size.data(), 4 * size_t(cap));
  std::memcpy(out->child_node_mask, app.oct.u_child_node_mask.data(),
              4 * size_t(cap));
  std::memcpy(out->child_leaf_mask, app.oct.u_child_leaf_mask.data(),
              4 * size_t(cap));
  return 0;
}

unsigned ref_hardware_threads() { return std::thread::hardware_concurrency(); }

}  // extern "C"
