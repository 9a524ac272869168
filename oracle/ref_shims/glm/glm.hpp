// Project-written stand-in for the one glm type the reference's CPU tree path
// uses: a four-float vector with x/y/z/w members and operator[].  glm is not
// installed here; the reference only stores and indexes vec4 (no glm math).
#pragma once

#include <cstddef>

namespace glm {

struct vec4 {
  float x = 0.0f, y = 0.0f, z = 0.0f, w = 0.0f;

  vec4() = default;
  vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}

  float& operator[](std::size_t i) { return (&x)[i]; }
  const float& operator[](std::size_t i) const { return (&x)[i]; }
};

static_assert(sizeof(vec4) == 16, "vec4 must be four packed floats");

}  // namespace glm
