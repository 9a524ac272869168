// cuda::CudaMemoryResource: the std::pmr resource the reference's CUDA path
// builds AppData on (redwood/cuda/cu_mem_resource.cu:9-27).  Managed memory,
// so the host reads results directly, as the reference's callers do.
#pragma once

#include <cuda_runtime.h>

#include <memory_resource>
#include <stdexcept>
#include <string>

namespace cuda {

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("CUDA Error: ") + cudaGetErrorString(e) + " at " +
                             what);
}

class CudaMemoryResource final : public std::pmr::memory_resource {
 protected:
  void* do_allocate(std::size_t bytes, std::size_t) override {
    void* p = nullptr;
    check_cuda(cudaMallocManaged(&p, bytes == 0 ? 1 : bytes), "cudaMallocManaged");
    return p;
  }
  void do_deallocate(void* p, std::size_t, std::size_t) override { cudaFree(p); }
  bool do_is_equal(const memory_resource& other) const noexcept override {
    return dynamic_cast<const CudaMemoryResource*>(&other) != nullptr;
  }
};

// Device-only memory (no host access; the fastest choice when the host only
// reads counts and copies out what it needs).
class CudaDeviceMemoryResource final : public std::pmr::memory_resource {
 protected:
  void* do_allocate(std::size_t bytes, std::size_t) override {
    void* p = nullptr;
    check_cuda(cudaMalloc(&p, bytes == 0 ? 1 : bytes), "cudaMalloc");
    return p;
  }
  void do_deallocate(void* p, std::size_t, std::size_t) override { cudaFree(p); }
  bool do_is_equal(const memory_resource& other) const noexcept override {
    return dynamic_cast<const CudaDeviceMemoryResource*>(&other) != nullptr;
  }
};

}  // namespace cuda
