// The boundary MLP of the learned-CDF sort: 16 -> 64 -> 64 -> 1, ReLU,
// BF16 weights with FP32 master copies, FP32 biases and FP32 accumulation.
// Training (forward + backward, FP32 activations) and Adam are hand-written
// for the CUDA cores: a block takes 32 rows and runs the layers as small
// matrix products in shared memory; weight gradients are reduced per block and
// added to the global gradient once.  Inference runs on the tensor cores
// (mlp.cuh).  No reference counterpart (the reference has no learned
// component).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "internal.hpp"
#include "mlp.cuh"

namespace rwt {

// parameter layout (FP32 master and gradients): W1 [64][16], b1 [64],
// W2 [64][64], b2 [64], W3 [64], b3 [1]
constexpr int kIn = kMlpIn, kH = kMlpHidden;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kIn, kOffW2 = kOffB1 + kH,
              kOffB2 = kOffW2 + kH * kH, kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH;
static_assert(kOffB3 + 1 == kMlpParams, "parameter layout");

__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// Rows per block and threads per block of the training kernel (4 threads per
// row, 16 hidden units each).
constexpr int kRows = 32, kMlpThreads = 128;

// Forward + backward over `rows` examples: grad += d(mean squared error)/d
// params for the batch, loss_sum += sum of squared errors.  Weights are used
// rounded to BF16 (the master copy stays FP32).
__global__ void __launch_bounds__(kMlpThreads)
    k_mlp_grad(const float* __restrict__ params, const float* __restrict__ x,
               const float* __restrict__ t, uint32_t rows, float inv_batch,
               float* __restrict__ grad, float* __restrict__ loss_sum) {
  __shared__ float s_w1[kH * kIn], s_w2[kH * kH], s_w3[kH], s_b1[kH], s_b2[kH];
  __shared__ float s_x[kRows * kIn];
  __shared__ float s_z1[kRows * kH], s_z2[kRows * kH];  // pre-activations
  __shared__ float s_d[kRows * kH];                      // dz2, then dz1
  __shared__ float s_dy[kRows];
  __shared__ float s_loss;
  const int tid = threadIdx.x;
  for (int i = tid; i < kH * kIn; i += kMlpThreads) s_w1[i] = bf16_round(params[kOffW1 + i]);
  for (int i = tid; i < kH * kH; i += kMlpThreads) s_w2[i] = bf16_round(params[kOffW2 + i]);
  for (int i = tid; i < kH; i += kMlpThreads) {
    s_w3[i] = bf16_round(params[kOffW3 + i]);
    s_b1[i] = params[kOffB1 + i];
    s_b2[i] = params[kOffB2 + i];
  }
  const float b3 = params[kOffB3];
  if (tid == 0) s_loss = 0.0f;
  const uint32_t r0 = blockIdx.x * kRows;
  const int nr = int(min(uint32_t(kRows), rows - r0));
  for (int i = tid; i < kRows * kIn; i += kMlpThreads) {
    const int r = i / kIn;
    s_x[i] = r < nr ? x[size_t(r0 + r) * kIn + (i % kIn)] : 0.0f;
  }
  __syncthreads();

  // z1 = W1 x + b1 ; z2 = W2 relu(z1) + b2   (thread: row r = tid / 4, 16 units)
  static_assert(kRows * 4 == kMlpThreads, "four threads per row");
  const int r = tid >> 2, u0 = (tid & 3) * 16;
  for (int u = u0; u < u0 + 16; ++u) {
    float acc = s_b1[u];
    for (int k = 0; k < kIn; ++k) acc = fmaf(s_w1[u * kIn + k], s_x[r * kIn + k], acc);
    s_z1[r * kH + u] = acc;
  }
  __syncthreads();
  for (int u = u0; u < u0 + 16; ++u) {
    float acc = s_b2[u];
    for (int k = 0; k < kH; ++k) acc = fmaf(s_w2[u * kH + k], fmaxf(s_z1[r * kH + k], 0.0f), acc);
    s_z2[r * kH + u] = acc;
  }
  __syncthreads();
  // y, dy (one thread per row)
  if (tid < kRows) {
    const int rr = tid;
    float y = b3;
    for (int k = 0; k < kH; ++k) y = fmaf(s_w3[k], fmaxf(s_z2[rr * kH + k], 0.0f), y);
    float dy = 0.0f;
    if (rr < nr) {
      const float e = y - t[r0 + rr];
      atomicAdd(&s_loss, e * e);
      dy = 2.0f * e * inv_batch;
    }
    s_dy[rr] = dy;
  }
  __syncthreads();
  // dz2 = dy * w3 * [z2 > 0]
  for (int i = tid; i < kRows * kH; i += kMlpThreads) {
    const int rr = i / kH, k = i % kH;
    s_d[i] = s_z2[i] > 0.0f ? s_dy[rr] * s_w3[k] : 0.0f;
  }
  __syncthreads();
  // gradients of layer 3 and 2: dW3[k] = sum dy h2 ; db3 ; dW2[u][k] = sum dz2[u] h1[k]
  for (int k = tid; k < kH; k += kMlpThreads) {
    float g3 = 0.0f, gb2 = 0.0f;
    for (int rr = 0; rr < kRows; ++rr) {
      g3 = fmaf(s_dy[rr], fmaxf(s_z2[rr * kH + k], 0.0f), g3);
      gb2 += s_d[rr * kH + k];
    }
    atomicAdd(&grad[kOffW3 + k], g3);
    atomicAdd(&grad[kOffB2 + k], gb2);
  }
  if (tid == 0) {
    float gb3 = 0.0f;
    for (int rr = 0; rr < kRows; ++rr) gb3 += s_dy[rr];
    atomicAdd(&grad[kOffB3], gb3);
  }
  for (int i = tid; i < kH * kH; i += kMlpThreads) {
    const int u = i / kH, k = i % kH;
    float g = 0.0f;
    for (int rr = 0; rr < kRows; ++rr) g = fmaf(s_d[rr * kH + u], fmaxf(s_z1[rr * kH + k], 0.0f), g);
    atomicAdd(&grad[kOffW2 + i], g);
  }
  __syncthreads();  // every read of z2 is done before it is overwritten
  // dh1 = W2^T dz2 ; dz1 = dh1 * [z1 > 0]   (written over s_z2, no longer needed)
  for (int k = u0; k < u0 + 16; ++k) {
    float acc = 0.0f;
    for (int u = 0; u < kH; ++u) acc = fmaf(s_w2[u * kH + k], s_d[r * kH + u], acc);
    s_z2[r * kH + k] = s_z1[r * kH + k] > 0.0f ? acc : 0.0f;
  }
  __syncthreads();
  // dW1[u][k] = sum dz1[u] x[k] ; db1[u] = sum dz1[u]
  for (int i = tid; i < kH * kIn; i += kMlpThreads) {
    const int u = i / kIn, k = i % kIn;
    float g = 0.0f;
    for (int rr = 0; rr < kRows; ++rr) g = fmaf(s_z2[rr * kH + u], s_x[rr * kIn + k], g);
    atomicAdd(&grad[kOffW1 + i], g);
  }
  for (int u = tid; u < kH; u += kMlpThreads) {
    float g = 0.0f;
    for (int rr = 0; rr < kRows; ++rr) g += s_z2[rr * kH + u];
    atomicAdd(&grad[kOffB1 + u], g);
  }
  __syncthreads();
  if (tid == 0 && loss_sum) atomicAdd(loss_sum, s_loss);
}

// Adam on the FP32 master parameters (Kingma & Ba 2015, bias-corrected).
__global__ void k_adam(float* __restrict__ params, const float* __restrict__ grad,
                       float* __restrict__ m, float* __restrict__ v, float lr, float beta1,
                       float beta2, float eps, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  const float g = grad[i];
  const float mi = beta1 * m[i] + (1.0f - beta1) * g;
  const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// Forward only (inference on `rows` feature rows) on the tensor cores, 128
// rows per CTA (mlp.cuh); a row whose tensor-core wait ran out gets NaN.
__global__ void __launch_bounds__(kMlpTcThreads)
    k_mlp_forward(const float* __restrict__ params, const float* __restrict__ x, uint32_t rows,
                  float* __restrict__ y) {
  const uint32_t r0 = blockIdx.x * uint32_t(kMlpTcRows);
  mlp_tile_tc(
      params,
      [&](int t, float (&v)[kMlpIn]) {
        const uint32_t row = r0 + uint32_t(t);
        if (row >= rows) return false;
        const float4* src = reinterpret_cast<const float4*>(x + size_t(row) * kMlpIn);
#pragma unroll
        for (int q = 0; q < kMlpIn / 4; ++q) {
          const float4 f = src[q];
          v[4 * q] = f.x;
          v[4 * q + 1] = f.y;
          v[4 * q + 2] = f.z;
          v[4 * q + 3] = f.w;
        }
        return true;
      },
      [&](int t, float out, bool ok) {
        const uint32_t row = r0 + uint32_t(t);
        if (row < rows) y[row] = ok ? out : __int_as_float(0x7fc00000);
      },
      nullptr);
}

}  // namespace rwt

extern "C" {

int rw_tree_mlp_param_count(void) { return rwt::kMlpParams; }

int rw_tree_mlp_grad(const float* d_params, const float* d_x, const float* d_t, uint32_t rows,
                     uint32_t batch, float* d_grad, float* d_loss_sum, rw_stream_t stream) {
  if (!d_params || !d_x || !d_t || !d_grad || rows < 1 || batch < 1) return RW_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const uint32_t blocks = (rows + rwt::kRows - 1) / rwt::kRows;
  rwt::k_mlp_grad<<<blocks, rwt::kMlpThreads, 0, s>>>(d_params, d_x, d_t, rows,
                                                     1.0f / float(batch), d_grad, d_loss_sum);
  return cudaGetLastError() == cudaSuccess ? RW_OK : RW_ERR_CUDA;
}

int rw_tree_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, float lr,
                     float beta1, float beta2, float eps, int32_t step, rw_stream_t stream) {
  if (!d_params || !d_grad || !d_m || !d_v || step < 1) return RW_ERR_ARG;
  const float bc1 = 1.0f - powf(beta1, float(step));
  const float bc2 = 1.0f - powf(beta2, float(step));
  rwt::k_adam<<<(rwt::kMlpParams + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      d_params, d_grad, d_m, d_v, lr, beta1, beta2, eps, bc1, bc2);
  return cudaGetLastError() == cudaSuccess ? RW_OK : RW_ERR_CUDA;
}

int rw_tree_mlp_forward(const float* d_params, const float* d_x, uint32_t rows, float* d_y,
                        rw_stream_t stream) {
  if (!d_params || !d_x || !d_y || rows < 1) return RW_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(d_x) & 15u) return RW_ERR_ARG;  // rows are read as float4
  rwt::k_mlp_forward<<<(rows + rwt::kMlpTcRows - 1) / rwt::kMlpTcRows, rwt::kMlpTcThreads, 0,
                       reinterpret_cast<cudaStream_t>(stream)>>>(d_params, d_x, rows, d_y);
  return cudaGetLastError() == cudaSuccess ? RW_OK : RW_ERR_CUDA;
}

}  // extern "C"
