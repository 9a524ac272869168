// Engine / typed_buffer: the unified front end the reference's README
// describes (README.md:12-35) and its code never implements.  An Engine owns
// the device, a stream and the memory resource; typed_buffer<T>(n) returns a
// shared, host-visible device buffer.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
#include <stdexcept>

#include "cu_mem_resource.hpp"

enum class EngineType { CUDA };

namespace cuda {

template <typename T>
class TypedBuffer {
 public:
  TypedBuffer(std::pmr::memory_resource* mr, std::size_t n)
      : mr_(mr), n_(n), data_(static_cast<T*>(mr->allocate(sizeof(T) * (n ? n : 1), 256))) {
    for (std::size_t i = 0; i < n_; ++i) new (data_ + i) T();
  }
  ~TypedBuffer() { mr_->deallocate(data_, sizeof(T) * (n_ ? n_ : 1), 256); }
  TypedBuffer(const TypedBuffer&) = delete;
  TypedBuffer& operator=(const TypedBuffer&) = delete;

  [[nodiscard]] T* data() { return data_; }
  [[nodiscard]] const T* data() const { return data_; }
  [[nodiscard]] std::size_t size() const { return n_; }
  T& operator[](std::size_t i) { return data_[i]; }
  const T& operator[](std::size_t i) const { return data_[i]; }

 private:
  std::pmr::memory_resource* mr_;
  std::size_t n_;
  T* data_;
};

}  // namespace cuda

template <typename T>
using CudaBuffer = std::shared_ptr<cuda::TypedBuffer<T>>;

class Engine {
 public:
  static std::shared_ptr<Engine> create(EngineType type, int device = 0) {
    if (type != EngineType::CUDA) throw std::runtime_error("only EngineType::CUDA exists");
    return std::shared_ptr<Engine>(new Engine(device));
  }
  ~Engine() {
    if (stream_) cudaStreamDestroy(stream_);
  }

  template <typename T>
  CudaBuffer<T> typed_buffer(std::size_t n) {
    return std::make_shared<cuda::TypedBuffer<T>>(&mr_, n);
  }
  [[nodiscard]] std::pmr::memory_resource* get_mr() { return &mr_; }
  [[nodiscard]] cudaStream_t stream() const { return stream_; }
  [[nodiscard]] int device() const { return device_; }
  void sync() { cuda::check_cuda(cudaStreamSynchronize(stream_), "Engine::sync"); }

 private:
  explicit Engine(int device) : device_(device) {
    cuda::check_cuda(cudaSetDevice(device), "cudaSetDevice");
    cuda::check_cuda(cudaStreamCreate(&stream_), "cudaStreamCreate");
  }
  int device_;
  cudaStream_t stream_ = nullptr;
  cuda::CudaMemoryResource mr_;
};
