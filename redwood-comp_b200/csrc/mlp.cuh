// Inference of the boundary MLP (16 -> 64 -> 64 -> 1, ReLU), shared by the
// training kernels and the learned sort.  Weights are passed already rounded
// to BF16 and widened to float (in shared memory); accumulation is FP32.
#pragma once

#include "internal.hpp"

namespace rwt {

__device__ __forceinline__ float mlp_eval(const float* __restrict__ x, const float* w1,
                                          const float* b1, const float* w2, const float* b2,
                                          const float* w3, float b3) {
  float h1[kMlpHidden];
#pragma unroll 8
  for (int u = 0; u < kMlpHidden; ++u) {
    float acc = b1[u];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) acc = fmaf(w1[u * kMlpIn + k], x[k], acc);
    h1[u] = fmaxf(acc, 0.0f);
  }
  float y = b3;
  for (int u = 0; u < kMlpHidden; ++u) {
    float acc = b2[u];
#pragma unroll 8
    for (int k = 0; k < kMlpHidden; ++k) acc = fmaf(w2[u * kMlpHidden + k], h1[k], acc);
    y = fmaf(w3[u], fmaxf(acc, 0.0f), y);
  }
  return y;
}

}  // namespace rwt
