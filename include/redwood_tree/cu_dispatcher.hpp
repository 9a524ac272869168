// cuda::run_stage1..7 and cuda::ImStorage with the reference's signatures
// (apps/tree/cuda/cu_dispatcher.cuh:8-19, im_storage.cuh:10-42), over the C
// ABI of rw_tree.h.  The stage functions are templates on the AppData type:
// they bind to the reference's own AppData (apps/tree/app_data.hpp) as well as
// to rwt::AppData (app_data.hpp here), through the member names only.
//
// Errors throw std::runtime_error, as the reference's CUDA_CHECK does
// (redwood/cuda/helpers.cuh:12-20).  Each stage is synchronous, as in the
// reference (cu_dispatcher.cu:521 and the other stream synchronisations); the
// one-argument overloads return a std::future (README.md:132-147).
#pragma once

#include <cuda_runtime.h>

#include <future>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "rw_tree.h"

namespace cuda {

inline void rw_check(int rc, const char* what) {
  if (rc != RW_OK)
    throw std::runtime_error(std::string(what) + ": rw_status " + std::to_string(rc) +
                             " (" + rw_tree_last_error() + ")");
}

// Scratch of the sort and unique stages (and, here, of every stage).
class ImStorage {
 public:
  explicit ImStorage(int n, int key_bits = 32, int radix_bits = 0) : n_(n) {
    rw_check(rw_tree_im_storage_create_ex(static_cast<uint32_t>(n), key_bits, radix_bits,
                                          &h_),
             "ImStorage");
  }
  ~ImStorage() { rw_tree_im_storage_destroy(h_); }
  ImStorage(const ImStorage&) = delete;
  ImStorage& operator=(const ImStorage&) = delete;

  // ImStorage::clearSmem (im_storage.cu:53-60); the stages clear what they use.
  void clearSmem(cudaStream_t stream = nullptr) {
    rw_check(rw_tree_im_storage_clear(h_, reinterpret_cast<rw_stream_t>(stream)),
             "clearSmem");
  }
  void set_sort_variant(int idx) {
    rw_check(rw_tree_im_storage_set_sort_variant(h_, idx), "set_sort_variant");
  }
  [[nodiscard]] rw_tree_im_storage* handle() const { return h_; }
  [[nodiscard]] int capacity() const { return n_; }

 private:
  rw_tree_im_storage* h_ = nullptr;
  int n_ = 0;
};

namespace detail {

template <typename A>
constexpr int32_t key_bits_of() {
  using K = std::remove_pointer_t<decltype(std::declval<A&>().u_morton_keys.data())>;
  return sizeof(K) == 4 ? 32 : 64;
}

// The C view of an AppData: the same buffers under the same names.
template <typename A>
rw_tree_app_data view(A& app) {
  rw_tree_app_data c;
  rw_tree_app_data_init(&c, static_cast<uint32_t>(app.n_input), key_bits_of<A>());
  c.min_coord = app.min_coord;
  c.range = app.range;
  c.n_unique = app.n_unique;
  c.n_brt_nodes = app.n_brt_nodes;
  c.n_octree_nodes = app.n_octree_nodes;
  c.u_input_points = reinterpret_cast<float*>(app.u_input_points.data());
  c.u_morton_keys = app.u_morton_keys.data();
  c.u_morton_keys_alt = app.u_morton_keys_alt.data();
  c.u_edge_count = app.u_edge_count.data();
  c.u_edge_offset = app.u_edge_offset.data();
  c.brt_prefix_n = app.brt.u_prefix_n.data();
  c.brt_has_leaf_left = app.brt.u_has_leaf_left.data();
  c.brt_has_leaf_right = app.brt.u_has_leaf_right.data();
  c.brt_left_child = app.brt.u_left_child.data();
  c.brt_parents = app.brt.u_parents.data();
  c.oct_children = app.oct.u_children.data();
  c.oct_corner = reinterpret_cast<float*>(app.oct.u_corner.data());
  c.oct_cell_size = app.oct.u_cell_size.data();
  c.oct_child_node_mask = app.oct.u_child_node_mask.data();
  c.oct_child_leaf_mask = app.oct.u_child_leaf_mask.data();
  c.oct_capacity = static_cast<uint32_t>(app.oct.u_cell_size.size());
  return c;
}

// Scratch for the stages whose reference signature takes no ImStorage: one per
// thread, grown to the largest cloud seen.
template <int KeyBits>
inline ImStorage& internal_storage(uint32_t n) {
  thread_local std::unique_ptr<ImStorage> im;
  if (!im || im->capacity() < static_cast<int>(n))
    im = std::make_unique<ImStorage>(static_cast<int>(n), KeyBits);
  return *im;
}

template <typename A>
ImStorage& storage_for(A& app) {
  return internal_storage<key_bits_of<A>()>(static_cast<uint32_t>(app.n_input));
}

}  // namespace detail

// input -> morton (cu_dispatcher.cu:501-522)
template <typename A>
void run_stage1(A& app, cudaStream_t stream) {
  auto c = detail::view(app);
  rw_check(rw_tree_run_stage1(&c, detail::storage_for(app).handle(),
                              reinterpret_cast<rw_stream_t>(stream)),
           "run_stage1");
}

// morton -> sorted morton in u_morton_keys_alt (cu_dispatcher.cu:528-591)
template <typename A>
void run_stage2(A& app, ImStorage& im, cudaStream_t stream) {
  auto c = detail::view(app);
  rw_check(rw_tree_run_stage2(&c, im.handle(), reinterpret_cast<rw_stream_t>(stream)),
           "run_stage2");
}

// sorted -> unique in u_morton_keys, sets n_unique (cu_dispatcher.cu:597-627)
template <typename A>
void run_stage3(A& app, ImStorage& im, cudaStream_t stream) {
  auto c = detail::view(app);
  rw_check(rw_tree_run_stage3(&c, im.handle(), reinterpret_cast<rw_stream_t>(stream)),
           "run_stage3");
  app.set_n_unique(c.n_unique);
  app.set_n_brt_nodes(c.n_unique - 1);
}

template <typename A>
void run_stage4(A& app, cudaStream_t stream) {
  auto c = detail::view(app);
  rw_check(rw_tree_run_stage4(&c, detail::storage_for(app).handle(),
                              reinterpret_cast<rw_stream_t>(stream)),
           "run_stage4");
}

template <typename A>
void run_stage5(A& app, cudaStream_t stream) {
  auto c = detail::view(app);
  rw_check(rw_tree_run_stage5(&c, detail::storage_for(app).handle(),
                              reinterpret_cast<rw_stream_t>(stream)),
           "run_stage5");
}

// edge count -> edge offset, sets n_octree_nodes (cu_dispatcher.cu:672-686)
template <typename A>
void run_stage6(A& app, cudaStream_t stream) {
  auto c = detail::view(app);
  rw_check(rw_tree_run_stage6(&c, detail::storage_for(app).handle(),
                              reinterpret_cast<rw_stream_t>(stream)),
           "run_stage6");
  app.set_n_octree_nodes(c.n_octree_nodes);
}

template <typename A>
void run_stage7(A& app, cudaStream_t stream) {
  auto c = detail::view(app);
  rw_check(rw_tree_run_stage7(&c, detail::storage_for(app).handle(),
                              reinterpret_cast<rw_stream_t>(stream)),
           "run_stage7");
}

// All seven stages fused, one synchronisation at the end.
template <typename A>
void run_pipeline(A& app, ImStorage& im, cudaStream_t stream) {
  auto c = detail::view(app);
  const auto s = reinterpret_cast<rw_stream_t>(stream);
  rw_check(rw_tree_pipeline_enqueue(&c, im.handle(), s), "pipeline_enqueue");
  rw_check(rw_tree_pipeline_finish(&c, im.handle(), s), "pipeline_finish");
  app.set_n_unique(c.n_unique);
  app.set_n_brt_nodes(c.n_unique - 1);
  app.set_n_octree_nodes(c.n_octree_nodes);
}

// Future-returning forms (README.md:132-147; hello_world/host/host_dispatchers.hpp:14):
// the stage runs on its own thread and default stream.
template <typename A>
std::future<void> run_stage1(A& app) {
  return std::async(std::launch::async, [&app] { run_stage1(app, cudaStream_t{}); });
}
template <typename A>
std::future<void> run_stage2(A& app) {
  return std::async(std::launch::async, [&app] {
    run_stage2(app, detail::storage_for(app), cudaStream_t{});
  });
}
template <typename A>
std::future<void> run_stage3(A& app) {
  return std::async(std::launch::async, [&app] {
    run_stage3(app, detail::storage_for(app), cudaStream_t{});
  });
}
template <typename A>
std::future<void> run_stage4(A& app) {
  return std::async(std::launch::async, [&app] { run_stage4(app, cudaStream_t{}); });
}
template <typename A>
std::future<void> run_stage5(A& app) {
  return std::async(std::launch::async, [&app] { run_stage5(app, cudaStream_t{}); });
}
template <typename A>
std::future<void> run_stage6(A& app) {
  return std::async(std::launch::async, [&app] { run_stage6(app, cudaStream_t{}); });
}
template <typename A>
std::future<void> run_stage7(A& app) {
  return std::async(std::launch::async, [&app] { run_stage7(app, cudaStream_t{}); });
}

}  // namespace cuda
