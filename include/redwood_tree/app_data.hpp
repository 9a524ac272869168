// AppData of the tree app with the reference's field names, types and sizes
// (apps/tree/app_data.hpp:15-158), for callers that do not bring their own.
// The dispatcher in cu_dispatcher.hpp also accepts the reference's own AppData
// type, since it only uses these member names.
#pragma once

#include <cstdint>
#include <limits>
#include <memory_resource>
#include <random>
#include <stdexcept>
#include <vector>

#if __has_include(<glm/glm.hpp>)
#include <glm/glm.hpp>
namespace rwt_glm = glm;
#else
namespace rwt_glm {
struct vec4 {
  float x = 0.0f, y = 0.0f, z = 0.0f, w = 0.0f;
  vec4() = default;
  vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  float& operator[](std::size_t i) { return (&x)[i]; }
  const float& operator[](std::size_t i) const { return (&x)[i]; }
};
}  // namespace rwt_glm
#endif

template <typename T>
using UsmVector = std::pmr::vector<T>;

namespace rwt {

// BaseAppData (redwood/base_appdata.hpp:15-21).
struct BaseAppData {
  explicit BaseAppData(std::pmr::memory_resource* mr) : mr_(mr) {}
  virtual ~BaseAppData() = default;
  std::pmr::memory_resource* mr_;
};

constexpr float k_memory_ratio = 0.6f;

struct AppData final : public BaseAppData {
  static constexpr float min_coord = 0.0f;
  static constexpr float range = 1024.0f;

  // Seeded like the reference (mt19937(114514), uniform [0, 1024)); the draw
  // order is that of a g++ build of the reference: z, then y, then x.
  AppData(std::pmr::memory_resource* mr, std::size_t n, unsigned seed = 114514)
      : BaseAppData(mr),
        n_input(static_cast<uint32_t>(n)),
        u_input_points(n, mr),
        u_morton_keys(n, mr),
        u_morton_keys_alt(n, mr),
        u_edge_count(n, mr),
        u_edge_offset(n, mr),
        brt(n, mr),
        oct(static_cast<std::size_t>(n * k_memory_ratio), mr) {
    std::mt19937 gen(seed);
    std::uniform_real_distribution<float> dis(min_coord, min_coord + range);
    for (auto& p : u_input_points) {
      const float z = dis(gen), y = dis(gen), x = dis(gen);
      p = rwt_glm::vec4(x, y, z, 1.0f);
    }
  }

  const uint32_t n_input;
  uint32_t n_unique = std::numeric_limits<uint32_t>::max();
  uint32_t n_brt_nodes = std::numeric_limits<uint32_t>::max();
  uint32_t n_octree_nodes = std::numeric_limits<uint32_t>::max();

  UsmVector<rwt_glm::vec4> u_input_points;
  UsmVector<uint32_t> u_morton_keys;
  UsmVector<uint32_t> u_morton_keys_alt;
  UsmVector<int32_t> u_edge_count;
  UsmVector<int32_t> u_edge_offset;

  struct RadixTree {
    RadixTree(std::size_t n, std::pmr::memory_resource* mr)
        : u_prefix_n(n, mr), u_has_leaf_left(n, mr), u_has_leaf_right(n, mr),
          u_left_child(n, mr), u_parents(n, mr) {}
    UsmVector<uint8_t> u_prefix_n;
    UsmVector<uint8_t> u_has_leaf_left;
    UsmVector<uint8_t> u_has_leaf_right;
    UsmVector<int32_t> u_left_child;
    UsmVector<int32_t> u_parents;
  } brt;

  struct Octree {
    Octree(std::size_t n, std::pmr::memory_resource* mr)
        : u_children(n * 8, mr), u_corner(n, mr), u_cell_size(n, mr),
          u_child_node_mask(n, mr), u_child_leaf_mask(n, mr) {}
    UsmVector<int32_t> u_children;
    UsmVector<rwt_glm::vec4> u_corner;
    UsmVector<float> u_cell_size;
    UsmVector<int32_t> u_child_node_mask;
    UsmVector<int32_t> u_child_leaf_mask;
  } oct;

  // getters and setters of app_data.hpp:108-137
  [[nodiscard]] uint32_t get_n_input() const { return n_input; }
  [[nodiscard]] uint32_t get_n_unique() const {
    if (n_unique == std::numeric_limits<uint32_t>::max())
      throw std::runtime_error("n_unique is not set");
    return n_unique;
  }
  void set_n_unique(uint32_t v) { n_unique = v; }
  void set_n_brt_nodes(uint32_t v) { n_brt_nodes = v; }
  [[nodiscard]] uint32_t get_n_brt_nodes() const { return get_n_unique() - 1; }
  [[nodiscard]] uint32_t get_n_octree_nodes() const {
    if (n_octree_nodes == std::numeric_limits<uint32_t>::max())
      throw std::runtime_error("n_octree_nodes is not set");
    return n_octree_nodes;
  }
  void set_n_octree_nodes(uint32_t v) { n_octree_nodes = v; }

  // buffer contract of app_data.hpp:139-157
  [[nodiscard]] uint32_t* get_sorted_morton_keys() { return u_morton_keys_alt.data(); }
  [[nodiscard]] uint32_t* get_unique_morton_keys() { return u_morton_keys.data(); }
};

// Moves every buffer of a managed-memory AppData to `device` ahead of the
// kernels (the reference lets page faults migrate them on first touch).
template <typename A>
inline void prefetch_to_device(A& app, int device, void* stream = nullptr) {
#ifdef __CUDA_RUNTIME_H__
  auto pf = [&](auto& v) {
    if (v.size())
      cudaMemPrefetchAsync(v.data(), v.size() * sizeof(*v.data()), device,
                           static_cast<cudaStream_t>(stream));
  };
  pf(app.u_input_points); pf(app.u_morton_keys); pf(app.u_morton_keys_alt);
  pf(app.u_edge_count); pf(app.u_edge_offset);
  pf(app.brt.u_prefix_n); pf(app.brt.u_has_leaf_left); pf(app.brt.u_has_leaf_right);
  pf(app.brt.u_left_child); pf(app.brt.u_parents);
  pf(app.oct.u_children); pf(app.oct.u_corner); pf(app.oct.u_cell_size);
  pf(app.oct.u_child_node_mask); pf(app.oct.u_child_leaf_mask);
#else
  (void)app; (void)device; (void)stream;
#endif
}

}  // namespace rwt
