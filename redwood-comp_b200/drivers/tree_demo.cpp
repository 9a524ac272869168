// The reference's CUDA demo (apps/tree/main.cpp:48-88, print_stats :12-16)
// run unchanged in shape on the B200 path: AppData on a managed-memory
// resource, ImStorage, cuda::run_stage1..7, host-side checks and peeks.  Then
// the same cloud through the future-returning stage calls and the fused
// pipeline, and a typed_buffer from an Engine.  Prints `key = value` lines.
//
// usage: tree_demo [n_points]
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "redwood_tree/redwood_tree.hpp"

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

void print_stats(const char* tag, rwt::AppData& app) {
  const auto m = app.get_n_octree_nodes();
  const auto b = app.get_n_brt_nodes();
  std::printf("%s.num_unique = %u\n", tag, app.get_n_unique());
  std::printf("%s.num_brt = %u\n", tag, b);
  std::printf("%s.num_octree_nodes = %u\n", tag, m);
  std::printf("%s.fnv_prefix_n = %#018llx\n", tag,
              (unsigned long long)fnv1a64(app.brt.u_prefix_n.data(), b));
  std::printf("%s.fnv_parents = %#018llx\n", tag,
              (unsigned long long)fnv1a64(app.brt.u_parents.data(), 4ull * b));
  std::printf("%s.fnv_edge_offset = %#018llx\n", tag,
              (unsigned long long)fnv1a64(app.u_edge_offset.data(), 4ull * b));
  std::printf("%s.fnv_children = %#018llx\n", tag,
              (unsigned long long)fnv1a64(app.oct.u_children.data(), 32ull * m));
  std::printf("%s.fnv_corner = %#018llx\n", tag,
              (unsigned long long)fnv1a64(app.oct.u_corner.data(), 16ull * m));
  std::printf("%s.fnv_cell_size = %#018llx\n", tag,
              (unsigned long long)fnv1a64(app.oct.u_cell_size.data(), 4ull * m));
  std::printf("%s.fnv_child_node_mask = %#018llx\n", tag,
              (unsigned long long)fnv1a64(app.oct.u_child_node_mask.data(), 4ull * m));
}

}  // namespace

int main(int argc, char** argv) {
  const std::size_t n = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 640 * 480;
  cudaStream_t stream;
  cuda::check_cuda(cudaStreamCreate(&stream), "cudaStreamCreate");

  cuda::CudaMemoryResource mr;
  rwt::AppData app(&mr, n);
  cuda::ImStorage im(static_cast<int>(n));

  cuda::run_stage1(app, stream);
  cuda::run_stage2(app, im, stream);
  const bool sorted =
      std::is_sorted(app.u_morton_keys_alt.begin(), app.u_morton_keys_alt.end());
  std::printf("stagewise.sorted = %d\n", int(sorted));
  cuda::run_stage3(app, im, stream);
  cuda::run_stage4(app, stream);
  cuda::run_stage5(app, stream);
  for (int i = 0; i < 10; ++i) std::printf("edge_count[%d] = %d\n", i, app.u_edge_count[i]);
  cuda::run_stage6(app, stream);
  for (int i = 0; i < 10; ++i) std::printf("edge_offset[%d] = %d\n", i, app.u_edge_offset[i]);
  cuda::run_stage7(app, stream);
  print_stats("stagewise", app);

  // the README's future-returning form
  rwt::AppData app2(&mr, n);
  cuda::run_stage1(app2).get();
  cuda::run_stage2(app2).get();
  cuda::run_stage3(app2).get();
  cuda::run_stage4(app2).get();
  cuda::run_stage5(app2).get();
  cuda::run_stage6(app2).get();
  cuda::run_stage7(app2).get();
  print_stats("futures", app2);

  // all seven stages fused
  rwt::AppData app3(&mr, n);
  rwt::prefetch_to_device(app3, 0, stream);
  cuda::run_pipeline(app3, im, stream);
  print_stats("fused", app3);

  // Engine / typed_buffer (README.md:12-35)
  auto engine = Engine::create(EngineType::CUDA);
  auto buf = engine->typed_buffer<int>(1024);
  for (std::size_t i = 0; i < buf->size(); ++i) (*buf)[i] = static_cast<int>(i);
  std::printf("engine.buffer_sum = %d\n", [&] {
    int s = 0;
    for (std::size_t i = 0; i < buf->size(); ++i) s += (*buf)[i];
    return s;
  }());

  cuda::check_cuda(cudaStreamDestroy(stream), "cudaStreamDestroy");
  std::printf("done = 1\n");
  return 0;
}
