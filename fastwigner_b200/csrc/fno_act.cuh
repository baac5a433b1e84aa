// GELU and its derivative, shared by the FNO's element-wise kernels and the
// tensor-core GEMM epilogues so that fused and unfused paths round alike.
#pragma once
#include <math.h>

namespace fw {

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

}  // namespace fw
