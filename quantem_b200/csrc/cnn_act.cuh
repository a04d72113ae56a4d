// Activations of the CNN kernels (reference: core/ml/activation_functions.py:166-181 with
// torch's defaults: LeakyReLU slope 0.01, ELU alpha 1, Softplus beta 1 / threshold 20).
// The forward runs in the GEMM epilogue on the FP32 accumulator; the backward reads the
// stored activation output y and forms d act / dz from it (every one of these activations
// has its derivative as a function of its output).
#pragma once
#include <cuda_runtime.h>

namespace qb {

enum : int {
  ACT_NONE = 0,
  ACT_RELU = 1,
  ACT_LEAKY_RELU = 2,
  ACT_ELU = 3,
  ACT_TANH = 4,
  ACT_SIGMOID = 5,
  ACT_SOFTPLUS = 6,
  ACT_COUNT = 7
};

__device__ __forceinline__ float act_forward(int act, float v) {
  switch (act) {
    case ACT_RELU: return fmaxf(v, 0.0f);
    case ACT_LEAKY_RELU: return v > 0.0f ? v : 0.01f * v;
    case ACT_ELU: return v > 0.0f ? v : expm1f(v);
    case ACT_TANH: return tanhf(v);
    case ACT_SIGMOID: return 1.0f / (1.0f + expf(-v));
    case ACT_SOFTPLUS: return v > 20.0f ? v : log1pf(expf(v));
    default: return v;
  }
}

// d act / dz at the pre-activation z whose activation is y.  NaN y takes a zero derivative
// for ReLU (its mask), as the ReLU kernels always did.
__device__ __forceinline__ float act_grad_from_output(int act, float y) {
  switch (act) {
    case ACT_RELU: return y > 0.0f ? 1.0f : 0.0f;
    case ACT_LEAKY_RELU: return y > 0.0f ? 1.0f : 0.01f;
    case ACT_ELU: return y > 0.0f ? 1.0f : y + 1.0f;
    case ACT_TANH: return 1.0f - y * y;
    case ACT_SIGMOID: return y * (1.0f - y);
    case ACT_SOFTPLUS: return y > 20.0f ? 1.0f : -expm1f(-y);  // sigmoid(z) = 1 - exp(-softplus(z))
    default: return 1.0f;
  }
}

}  // namespace qb
