// Kernels of the Fourier-neural-operator surrogate (forward, backward, Adam).
//
// The FNO is small (width 32, 16 x 16 retained modes); its dense contractions --
// truncated DFTs written as products with DFT matrices, the pointwise channel
// maps, the projection, the weight gradients -- run on the tensor-core GEMM
// (fno_umma.cu).  The per-mode complex channel mixing of the spectral
// convolution, bias + GELU, channel reductions, the relative-L2 loss and the
// Adam update have their own element-wise kernels here.  FP32 throughout, FP64
// accumulation in the reductions.
#include <cuda_runtime.h>
#include <math.h>
#include "fno_act.cuh"
#include "fw_internal.h"

namespace fw {

// Spectral mixing.  F: [B][Cin][2][K] (real block then imaginary block of the
// K retained modes), R: [Cin][Cout][2][K], O: [B][Cout][2][K].
// forward:   O[b][o][k] = sum_i F[b][i][k] R[i][o][k]
__global__ void mix_fwd_kernel(int Bn, int Ci, int Co, int K, const float* F, const float* R, float* O) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Bn * Co * K) return;
  const int k = idx % K;
  const int o = (idx / K) % Co;
  const int b = idx / ((long long)K * Co);
  float re = 0.f, im = 0.f;
  for (int i = 0; i < Ci; ++i) {
    const float fr = F[(((size_t)b * Ci + i) * 2) * K + k], fi = F[(((size_t)b * Ci + i) * 2 + 1) * K + k];
    const float rr = R[(((size_t)i * Co + o) * 2) * K + k], ri = R[(((size_t)i * Co + o) * 2 + 1) * K + k];
    re += fr * rr - fi * ri;
    im += fr * ri + fi * rr;
  }
  O[(((size_t)b * Co + o) * 2) * K + k] = re;
  O[(((size_t)b * Co + o) * 2 + 1) * K + k] = im;
}
// dF[b][i][k] = sum_o dO[b][o][k] conj(R[i][o][k])
__global__ void mix_bwd_in_kernel(int Bn, int Ci, int Co, int K, const float* dO, const float* R, float* dF) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Bn * Ci * K) return;
  const int k = idx % K;
  const int i = (idx / K) % Ci;
  const int b = idx / ((long long)K * Ci);
  float re = 0.f, im = 0.f;
  for (int o = 0; o < Co; ++o) {
    const float gr = dO[(((size_t)b * Co + o) * 2) * K + k], gi = dO[(((size_t)b * Co + o) * 2 + 1) * K + k];
    const float rr = R[(((size_t)i * Co + o) * 2) * K + k], ri = R[(((size_t)i * Co + o) * 2 + 1) * K + k];
    re += gr * rr + gi * ri;
    im += gi * rr - gr * ri;
  }
  dF[(((size_t)b * Ci + i) * 2) * K + k] = re;
  dF[(((size_t)b * Ci + i) * 2 + 1) * K + k] = im;
}
// dR[i][o][k] = sum_b conj(F[b][i][k]) dO[b][o][k]
__global__ void mix_bwd_w_kernel(int Bn, int Ci, int Co, int K, const float* F, const float* dO, float* dR) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Ci * Co * K) return;
  const int k = idx % K;
  const int o = (idx / K) % Co;
  const int i = idx / ((long long)K * Co);
  double re = 0.0, im = 0.0;
  for (int b = 0; b < Bn; ++b) {
    const float fr = F[(((size_t)b * Ci + i) * 2) * K + k], fi = F[(((size_t)b * Ci + i) * 2 + 1) * K + k];
    const float gr = dO[(((size_t)b * Co + o) * 2) * K + k], gi = dO[(((size_t)b * Co + o) * 2 + 1) * K + k];
    re += (double)fr * gr + (double)fi * gi;
    im += (double)fr * gi - (double)fi * gr;
  }
  dR[(((size_t)i * Co + o) * 2) * K + k] = (float)re;
  dR[(((size_t)i * Co + o) * 2 + 1) * K + k] = (float)im;
}

// pre = X + bias[c]; Y = act ? gelu(pre) : pre.  X, pre, Y: [B][C][L]
__global__ void bias_act_kernel(long long n, int C, long long L, const float* X, const float* bias, float* pre,
                                float* Y, int act) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (i / L) % C;
    const float p = X[i] + bias[c];
    if (pre) pre[i] = p;
    Y[i] = act ? gelu(p) : p;
  }
}
// dpre = act ? dY * gelu'(pre) : dY
__global__ void act_bwd_kernel(long long n, const float* dY, const float* pre, float* dpre, int act) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dpre[i] = act ? dY[i] * gelu_d(pre[i]) : dY[i];
}
// out[c] (+)= sum_{b, l} X[b][c][l]; one 1024-thread block per channel, FP64
// accumulation, float4 loads (four in flight per thread) when L % 4 == 0 and X
// is 16-byte aligned
constexpr int kCsumThreads = 1024;
__global__ void __launch_bounds__(kCsumThreads) channel_sum_kernel(int Bn, int C, long long L, const float* X,
                                                                   float* out, int accumulate, int vec) {
  const int c = blockIdx.x;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int b = 0; b < Bn; ++b) {
    const float* x = X + ((size_t)b * C + c) * L;
    if (vec) {
      const float4* x4 = reinterpret_cast<const float4*>(x);
      const long long n4 = L / 4;
      long long l = threadIdx.x;
      for (; l + 3 * kCsumThreads < n4; l += 4 * kCsumThreads) {
        const float4 a = __ldg(x4 + l), b1 = __ldg(x4 + l + kCsumThreads), c1 = __ldg(x4 + l + 2 * kCsumThreads),
                     d = __ldg(x4 + l + 3 * kCsumThreads);
        s0 += (double)a.x + a.y + (double)a.z + a.w;
        s1 += (double)b1.x + b1.y + (double)b1.z + b1.w;
        s2 += (double)c1.x + c1.y + (double)c1.z + c1.w;
        s3 += (double)d.x + d.y + (double)d.z + d.w;
      }
      for (; l < n4; l += kCsumThreads) {
        const float4 a = __ldg(x4 + l);
        s0 += (double)a.x + a.y + (double)a.z + a.w;
      }
    } else {
      for (long long l = threadIdx.x; l < L; l += kCsumThreads) s0 += x[l];
    }
  }
  double s = (s0 + s1) + (s2 + s3);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double red[kCsumThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = red[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) out[c] = (float)(t + (accumulate ? (double)out[c] : 0.0));
  }
}
// loss_b = ||Y_b - T_b||^2 / ||T_b||^2; dY = 2 (Y - T) / ||T_b||^2 / B.  One block per sample.
__global__ void rel_l2_kernel(long long L, const float* Y, const float* T, float* dY, double* loss, int Bn) {
  const int b = blockIdx.x;
  const float* y = Y + (size_t)b * L;
  const float* t = T + (size_t)b * L;
  double e = 0.0, n = 0.0;
  for (long long l = threadIdx.x; l < L; l += blockDim.x) {
    const double d = (double)y[l] - t[l];
    e += d * d;
    n += (double)t[l] * t[l];
  }
  __shared__ double r1[256], r2[256];
  r1[threadIdx.x] = e;
  r2[threadIdx.x] = n;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      r1[threadIdx.x] += r1[threadIdx.x + o];
      r2[threadIdx.x] += r2[threadIdx.x + o];
    }
    __syncthreads();
  }
  const double nn = r2[0] > 0 ? r2[0] : 1.0;
  if (threadIdx.x == 0) loss[b] = r1[0] / nn;
  if (dY) {
    const float s = (float)(2.0 / nn / Bn);
    for (long long l = threadIdx.x; l < L; l += blockDim.x) dY[(size_t)b * L + l] = s * (y[l] - t[l]);
  }
}
__global__ void adam_kernel(long long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                            float eps, float bc1, float bc2, float wd) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * p[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}
// lift input: feats[b][f][p][x], f = 0..(NP-1): sample parameters, NP, NP+1: x, p coordinates (normalised)
__global__ void features_kernel(int Bn, int NP, int G0, int G1, const float* params, const float* xs, const float* ps,
                                float* out) {
  const long long L = (long long)G0 * G1;
  const long long n = (long long)Bn * (NP + 2) * L;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long l = i % L;
    const int f = (i / L) % (NP + 2);
    const int b = i / (L * (NP + 2));
    float v;
    if (f < NP) v = params[(size_t)b * NP + f];
    else if (f == NP) v = xs[l % G1];
    else v = ps[l / G1];
    out[i] = v;
  }
}

}  // namespace fw

using namespace fw;

static int grid1(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b > 8192 ? 8192 : (b < 1 ? 1 : b));
}

extern "C" int fw_fno_mix(int mode, int Bn, int Ci, int Co, int K, const float* X, const float* Y, float* out,
                          void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (mode == 0) mix_fwd_kernel<<<grid1((long long)Bn * Co * K), 256, 0, st>>>(Bn, Ci, Co, K, X, Y, out);
  else if (mode == 1) mix_bwd_in_kernel<<<grid1((long long)Bn * Ci * K), 256, 0, st>>>(Bn, Ci, Co, K, X, Y, out);
  else if (mode == 2) mix_bwd_w_kernel<<<grid1((long long)Ci * Co * K), 256, 0, st>>>(Bn, Ci, Co, K, X, Y, out);
  else return fail(FW_EINVAL, "fw_fno_mix: mode must be 0 (forward), 1 (input grad) or 2 (weight grad)");
  count_launch(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_mix");
}

extern "C" int fw_fno_bias_act(long long n, int C, long long L, const float* X, const float* bias, float* pre, float* Y,
                               int act, void* stream) {
  bias_act_kernel<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, C, L, X, bias, pre, Y, act);
  count_launch(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_bias_act");
}

extern "C" int fw_fno_act_bwd(long long n, const float* dY, const float* pre, float* dpre, int act, void* stream) {
  act_bwd_kernel<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, dY, pre, dpre, act);
  count_launch(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_act_bwd");
}

extern "C" int fw_fno_channel_sum(int Bn, int C, long long L, const float* X, float* out, int accumulate,
                                  void* stream) {
  const int vec = (L % 4 == 0) && ((reinterpret_cast<uintptr_t>(X) & 15u) == 0);
  channel_sum_kernel<<<C, kCsumThreads, 0, static_cast<cudaStream_t>(stream)>>>(Bn, C, L, X, out, accumulate, vec);
  count_launch(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_channel_sum");
}

extern "C" int fw_fno_rel_l2(int Bn, long long L, const float* Y, const float* T, float* dY, double* loss,
                             void* stream) {
  rel_l2_kernel<<<Bn, 256, 0, static_cast<cudaStream_t>(stream)>>>(L, Y, T, dY, loss, Bn);
  count_launch(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_rel_l2");
}

extern "C" int fw_fno_adam(long long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                           float eps, int step, float weight_decay, void* stream) {
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, p, g, m, v, lr, b1, b2, eps, bc1, bc2,
                                                                        weight_decay);
  count_launch(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_adam");
}

extern "C" int fw_fno_features(int Bn, int NP, int G0, int G1, const float* params, const float* xs, const float* ps,
                               float* out, void* stream) {
  features_kernel<<<grid1((long long)Bn * (NP + 2) * G0 * G1), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      Bn, NP, G0, G1, params, xs, ps, out);
  count_launch(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_features");
}

extern "C" int fw_fno_status(int* status_out, int clear) {
  if (status_out == nullptr) return fail(FW_EINVAL, "fw_fno_status: NULL argument");
  return fno_status_read(status_out, clear);
}
