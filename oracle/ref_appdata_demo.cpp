// Test infrastructure, not product code: the drop-in claim made concrete.
// The reference's OWN AppData (apps/tree/app_data.hpp, with its static
// constexpr min_coord / range, glm::vec4 corners, and its mt19937(114514)
// input generator), allocated on a managed-memory pmr resource, is handed to
// this project's cuda::run_stage1..7 (include/redwood_tree/cu_dispatcher.hpp)
// with the reference's call shapes: stages 2 and 3 take an ImStorage, the
// others only the AppData and a stream (apps/tree/cuda/cu_dispatcher.cuh:8-19),
// as in the reference's demo (apps/tree/main.cpp:48-88).  Then the same cloud
// through the future-returning stage calls and the fused pipeline.  Prints
// `key = value` lines (counts and FNV-1a digests of every output) that the
// GPU test compares with the committed fixture made from the reference's
// CPU functions.  Built by oracle/Makefile into _ref/ (it includes the
// reference's header, which only this machine has).
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "app_data.hpp"  // the reference's AppData
#include "redwood_tree/cu_dispatcher.hpp"
#include "redwood_tree/cu_mem_resource.hpp"

namespace {

uint64_t fnv1a64(const void* data, std::size_t bytes) {
  const auto* p = static_cast<const unsigned char*>(data);
  uint64_t h = 0xcbf29ce484222325ull;
  for (std::size_t i = 0; i < bytes; ++i) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

void print(const char* tag, const char* field, const void* data, std::size_t bytes) {
  std::printf("%s.fnv_%s = %#018llx\n", tag, field,
              static_cast<unsigned long long>(fnv1a64(data, bytes)));
}

void print_stats(const char* tag, const AppData& app) {
  const std::size_t n = app.get_n_input(), u = app.get_n_unique(), b = app.get_n_brt_nodes(),
                    m = app.get_n_octree_nodes();
  std::printf("%s.num_unique = %zu\n%s.num_brt = %zu\n%s.num_octree_nodes = %zu\n", tag, u, tag,
              b, tag, m);
  print(tag, "points", app.u_input_points.data(), 16 * n);
  print(tag, "sorted_keys", app.u_morton_keys_alt.data(), 4 * n);
  print(tag, "unique_keys", app.u_morton_keys.data(), 4 * u);
  print(tag, "prefix_n", app.brt.u_prefix_n.data(), b);
  print(tag, "has_leaf_left", app.brt.u_has_leaf_left.data(), b);
  print(tag, "has_leaf_right", app.brt.u_has_leaf_right.data(), b);
  print(tag, "left_child", app.brt.u_left_child.data(), 4 * b);
  print(tag, "parents", app.brt.u_parents.data(), 4 * b);
  print(tag, "edge_count", app.u_edge_count.data(), 4 * b);
  print(tag, "edge_offset", app.u_edge_offset.data(), 4 * b);
  print(tag, "children", app.oct.u_children.data(), 32 * m);
  print(tag, "corner", app.oct.u_corner.data(), 16 * m);
  print(tag, "cell_size", app.oct.u_cell_size.data(), 4 * m);
  print(tag, "child_node_mask", app.oct.u_child_node_mask.data(), 4 * m);
  print(tag, "child_leaf_mask", app.oct.u_child_leaf_mask.data(), 4 * m);
}

}  // namespace

int main(int argc, char** argv) {
  const std::size_t n = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 640 * 480;
  cudaStream_t stream;
  cuda::check_cuda(cudaStreamCreate(&stream), "cudaStreamCreate");
  cuda::CudaMemoryResource mr;
  {
    AppData app(&mr, n);  // fills its own input: mt19937(114514), uniform [0, 1024)
    cuda::ImStorage im(static_cast<int>(n));
    cuda::run_stage1(app, stream);
    cuda::run_stage2(app, im, stream);
    cuda::run_stage3(app, im, stream);
    cuda::run_stage4(app, stream);
    cuda::run_stage5(app, stream);
    cuda::run_stage6(app, stream);
    cuda::run_stage7(app, stream);
    print_stats("stagewise", app);

    AppData app2(&mr, n);
    cuda::run_stage1(app2).get();
    cuda::run_stage2(app2).get();
    cuda::run_stage3(app2).get();
    cuda::run_stage4(app2).get();
    cuda::run_stage5(app2).get();
    cuda::run_stage6(app2).get();
    cuda::run_stage7(app2).get();
    print_stats("futures", app2);

    AppData app3(&mr, n);
    cuda::run_pipeline(app3, im, stream);
    print_stats("fused", app3);
  }
  cuda::check_cuda(cudaStreamDestroy(stream), "cudaStreamDestroy");
  std::printf("done = 1\n");
  return 0;
}
