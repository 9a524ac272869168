// The reference's end-to-end loop (apps/tree/pipe_main_baseline.cpp:55-92):
// iterations of cuda::run_stage1..7, each stage synchronous, timed by wall
// clock.  Then the same iterations through the fused pipeline (one
// synchronisation per iteration) on device memory.
//
// usage: pipe_baseline [n_points] [iterations]
#include <chrono>
#include <cstdio>
#include <cstdlib>

#include "redwood_tree/redwood_tree.hpp"

int main(int argc, char** argv) {
  const std::size_t n = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 640 * 480;
  const int iters = argc > 2 ? std::atoi(argv[2]) : 1000;
  cudaStream_t stream;
  cuda::check_cuda(cudaStreamCreate(&stream), "cudaStreamCreate");

  cuda::CudaMemoryResource mr;
  rwt::AppData app(&mr, n);  // points generated on the host (managed memory)
  rwt::prefetch_to_device(app, 0, stream);
  cuda::ImStorage im(static_cast<int>(n));

  auto stagewise = [&] {
    cuda::run_stage1(app, stream);
    cuda::run_stage2(app, im, stream);
    cuda::run_stage3(app, im, stream);
    cuda::run_stage4(app, stream);
    cuda::run_stage5(app, stream);
    cuda::run_stage6(app, stream);
    cuda::run_stage7(app, stream);
  };
  auto fused = [&] { cuda::run_pipeline(app, im, stream); };

  auto time_loop = [&](const char* tag, auto&& body) {
    for (int i = 0; i < 3; ++i) body();
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < iters; ++i) body();
    const auto t1 = std::chrono::steady_clock::now();
    const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    std::printf("%s.total_ms = %.3f\n", tag, ms);
    std::printf("%s.ms_per_iteration = %.5f\n", tag, ms / iters);
    std::printf("%s.points_per_s = %.1f\n", tag, double(n) * iters / (ms / 1e3));
  };
  time_loop("stagewise", stagewise);
  time_loop("fused", fused);
  std::printf("num_unique = %u\nnum_octree_nodes = %u\n", app.get_n_unique(),
              app.get_n_octree_nodes());
  cuda::check_cuda(cudaStreamDestroy(stream), "cudaStreamDestroy");
  return 0;
}
