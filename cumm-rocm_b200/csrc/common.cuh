// common.cuh - element conversions and the epilogue shared by the conv and
// GEMM kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cstdint>

#include "sm100.cuh"

namespace scb {

template <typename T>
__device__ __forceinline__ float to_f32(T v);
template <>
__device__ __forceinline__ float to_f32<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 v) {
  return __bfloat162float(v);
}
template <>
__device__ __forceinline__ float to_f32<__half>(__half v) { return __half2float(v); }

template <typename T>
__device__ __forceinline__ T from_f32(float v);
template <>
__device__ __forceinline__ float from_f32<float>(float v) { return v; }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}
template <>
__device__ __forceinline__ __half from_f32<__half>(float v) { return __float2half_rn(v); }

// Activation of the reference's UnaryActivation (cumm/gemm/gemmmath/__init__.py:152-215):
// 0 none, 1 ReLU, 2 Sigmoid, 3 LeakyReLU(alpha).
__device__ __forceinline__ float apply_act(float x, int type, float a) {
  switch (type) {
    case 1:
      return fmaxf(x, 0.f);
    case 2:
      return 1.f / (1.f + expf(-x));
    case 3:
      return x >= 0.f ? x : x * a;
    default:
      return x;
  }
}

// Epilogue parameters.
//   mode 0 (LinearCombination, cumm/gemm/output_op/linear.py:16-183):
//       D = act(alpha * acc + beta * src)
//   mode 1 (scale/bias op, linear.py:185-392 without the int8 clamp):
//       D = act(scale[n] * acc + alpha * bias[n] + beta * src)
// src is `src` with row stride src_ld (elements); src_ld == 0 broadcasts one
// [n] row (bias used as the source, "d_is_bias").
struct EpiParams {
  float alpha, beta, act_alpha, act_beta;
  int act_type;
  int mode;
  const void *src;
  int64_t src_ld;
  const float *scale;
  const void *bias;
};

}  // namespace scb
