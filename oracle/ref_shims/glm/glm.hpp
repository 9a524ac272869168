// Project-written stand-in for the one glm type the reference's tree path
// uses: a four-float vector with x/y/z/w members and operator[].  glm is not
// installed here; the reference only stores and indexes vec4 (no glm math).
// Under nvcc the members are also device functions, since the reference's
// CUDA kernels index vec4 on the device (apps/tree/cuda/func_morton.cuh:54-76).
#pragma once

#include <cstddef>
#include <cstdint>  // real glm brings these in; the reference relies on it

#if defined(__CUDACC__)
#define RW_SHIM_HD __host__ __device__
#else
#define RW_SHIM_HD
#endif

namespace glm {

struct vec4 {
  float x = 0.0f, y = 0.0f, z = 0.0f, w = 0.0f;

  vec4() = default;
  RW_SHIM_HD vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}

  RW_SHIM_HD float& operator[](std::size_t i) { return (&x)[i]; }
  RW_SHIM_HD const float& operator[](std::size_t i) const { return (&x)[i]; }
};

static_assert(sizeof(vec4) == 16, "vec4 must be four packed floats");

}  // namespace glm
