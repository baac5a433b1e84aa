// Fused half-step passes for real Wigner functions W(x, p) (Moyal, Bloch,
// random-collision).  A row pass (kinetic step) transforms along x, a column
// pass (potential step) along p.  Each CTA streams its tiles from HBM once,
// runs forward FFT -> spectral multiply -> inverse FFT out of registers and
// shared memory, and writes each tile back once.  Two real rows/columns are
// packed into one complex FFT.
#include "wigner_tiles.cuh"
#include "fw_internal.h"

namespace fw {
template <typename Rl, int N, int T, int G, int MINB>
__global__ void __launch_bounds__(G* T, MINB) row_pass_kernel(PassArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[34];
  row_tile<Rl, N, T, G, true>(a, blockIdx.y, blockIdx.x, smem_raw, red);
}

template <typename Rl, int N, int T, int CP, int MINB>
__global__ void __launch_bounds__(CP* T, MINB) col_pass_kernel(PassArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[34];
  __shared__ double ored[(CP * T) / 32][2 + 2 * MAXO];
  col_tile<Rl, N, T, CP>(a, blockIdx.y, blockIdx.x, gridDim.x, smem_raw, red, ored);
}

// Per-instance totals of a pass's partial-sum records: block b, warp m < M
// sums column m of instance b's records (lane l takes records l, l + 32, ...,
// then a fixed shuffle tree: deterministic) into tot[b*M + m], and into
// hist[b*M + m] when hist is set.
__global__ void totals_kernel(const double* part, int nparts, int M, double* tot, double* hist) {
  const int b = blockIdx.x, m = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (m >= M) return;  // whole warps
  const double* pp = part + (size_t)b * nparts * M + m;
  double s = 0.0;
  for (int c = lane; c < nparts; c += 32) s += __ldcg(pp + (size_t)c * M);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) {
    tot[(size_t)b * M + m] = s;
    if (hist != nullptr) hist[(size_t)b * M + m] = s;
  }
}

cudaError_t launch_totals(const double* part, int nparts, int M, int batch, double* tot, double* hist,
                          cudaStream_t st) {
  totals_kernel<<<batch, 32 * M, 0, st>>>(part, nparts, M, tot, hist);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// finalize: apply the last step's normalisation and reduce its partials.
// blockIdx.y = instance; 16-byte vectors when the instance is aligned to them.
template <typename Rl>
__global__ void finalize_kernel(PassArgs a, int vec) {
  __shared__ double red[34];
  const int b = blockIdx.y;
  const double sc = prev_scale(a, b, red, blockIdx.x == 0);
  Rl* W = reinterpret_cast<Rl*>(a.W) + (size_t)b * a.w_bs;
  const size_t n = (size_t)a.P * a.X;
  const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, di = (size_t)gridDim.x * blockDim.x;
  if (vec) {
    if constexpr (sizeof(Rl) == 4) {
      float4* W4 = reinterpret_cast<float4*>(W);
      for (size_t i = i0; i < n / 4; i += di) {
        float4 w = W4[i];
        w.x = (float)(w.x * sc);
        w.y = (float)(w.y * sc);
        w.z = (float)(w.z * sc);
        w.w = (float)(w.w * sc);
        W4[i] = w;
      }
    } else {
      double2* W2 = reinterpret_cast<double2*>(W);
      for (size_t i = i0; i < n / 2; i += di) {
        double2 w = W2[i];
        w.x *= sc;
        w.y *= sc;
        W2[i] = w;
      }
    }
  } else {
    for (size_t i = i0; i < n; i += di) W[i] = (Rl)(W[i] * sc);
  }
}

// ---------------------------------------------------------------------------
// Launch configuration per FFT length and precision (column passes above
// N = 1024 FP32 / 512 FP64 use 256-thread CTAs so that a thread may hold 255
// registers: the 32-value transforms spill badly at 128).
template <typename Rl, int N> struct RowCfg;
template <typename Rl, int N> struct ColCfg;
// float: T threads per transform, RV = N / T values per thread
template <> struct RowCfg<float, 128> { static constexpr int T = 16, G = 16, MINB = 1; };
template <> struct RowCfg<float, 256> { static constexpr int T = 32, G = 4, MINB = 2; };
template <> struct RowCfg<float, 512> { static constexpr int T = 32, G = 4, MINB = 2; };
template <> struct RowCfg<float, 1024> { static constexpr int T = 32, G = 4, MINB = 3; };
template <> struct RowCfg<float, 2048> { static constexpr int T = 64, G = 4, MINB = 1; };
template <> struct RowCfg<float, 4096> { static constexpr int T = 128, G = 2, MINB = 1; };
template <> struct RowCfg<double, 128> { static constexpr int T = 16, G = 16, MINB = 1; };
template <> struct RowCfg<double, 256> { static constexpr int T = 16, G = 8, MINB = 2; };
template <> struct RowCfg<double, 512> { static constexpr int T = 32, G = 8, MINB = 1; };
template <> struct RowCfg<double, 1024> { static constexpr int T = 64, G = 4, MINB = 1; };
template <> struct RowCfg<double, 2048> { static constexpr int T = 128, G = 2, MINB = 1; };
template <> struct RowCfg<double, 4096> { static constexpr int T = 256, G = 1, MINB = 1; };

template <> struct ColCfg<float, 128> { static constexpr int T = 16, CP = 32, MINB = 1; };
template <> struct ColCfg<float, 256> { static constexpr int T = 32, CP = 16, MINB = 1; };
template <> struct ColCfg<float, 512> { static constexpr int T = 32, CP = 16, MINB = 1; };
// 1024: the column tile of the persistent column pass (wigner_colp.cu), which
// writes the same partial-sum records
template <> struct ColCfg<float, 1024> { static constexpr int T = 64, CP = 8, MINB = 1; };
template <> struct ColCfg<float, 2048> { static constexpr int T = 64, CP = 4, MINB = 1; };
template <> struct ColCfg<float, 4096> { static constexpr int T = 128, CP = 2, MINB = 1; };
template <> struct ColCfg<double, 128> { static constexpr int T = 16, CP = 16, MINB = 1; };
template <> struct ColCfg<double, 256> { static constexpr int T = 16, CP = 8, MINB = 2; };
template <> struct ColCfg<double, 512> { static constexpr int T = 32, CP = 8, MINB = 1; };
template <> struct ColCfg<double, 1024> { static constexpr int T = 64, CP = 4, MINB = 1; };
template <> struct ColCfg<double, 2048> { static constexpr int T = 128, CP = 2, MINB = 1; };
template <> struct ColCfg<double, 4096> { static constexpr int T = 256, CP = 1, MINB = 1; };

// Shapes for batches whose column pass would leave SMs idle with the shapes
// above (the one-instance use of the drop-in classes): the same shapes unless
// a sweep found faster ones for one instance.
template <typename Rl, int N> struct RowCfgSmall : RowCfg<Rl, N> {};
template <typename Rl, int N> struct ColCfgSmall : ColCfg<Rl, N> {};
// FP64 256^2, one instance: 16.4 us per step vs 25.7 (at 512 instances the
// shapes above are faster: 6.09e10 vs 4.82e10 pt-steps/s)
template <> struct RowCfgSmall<double, 256> { static constexpr int T = 32, G = 4, MINB = 2; };
template <> struct ColCfgSmall<double, 256> { static constexpr int T = 32, CP = 4, MINB = 2; };
// FP32 2048-point rows of one 1024 x 2048 instance (strong field): 69.3 vs 72.3 us per step
template <> struct RowCfgSmall<float, 2048> { static constexpr int T = 64, G = 1, MINB = 2; };

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

template <typename Rl, int N, int T, int G, int MINB>
static cudaError_t launch_row_cfg(const PassArgs& a, cudaStream_t st) {
  const size_t smem = (size_t)G * 2 * (N + N / 32) * sizeof(Rl);
  auto kern = row_pass_kernel<Rl, N, T, G, MINB>;
  static PerDeviceOnce attr;  // per device: the attribute is set on the device current at the call
  cudaError_t e = set_smem_once(attr, kern, smem);
  if (e != cudaSuccess) return e;
  dim3 grid((a.P / 2 + G - 1) / G, a.batch);
  kern<<<grid, G * T, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename Rl, int N>
static cudaError_t launch_row_n(const PassArgs& a, cudaStream_t st) {
  if (a.small_shape) {
    using Cfg = RowCfgSmall<Rl, N>;
    return launch_row_cfg<Rl, N, Cfg::T, Cfg::G, Cfg::MINB>(a, st);
  }
  using Cfg = RowCfg<Rl, N>;
  return launch_row_cfg<Rl, N, Cfg::T, Cfg::G, Cfg::MINB>(a, st);
}

template <typename Rl, int N, int T, int CP, int MINB>
static cudaError_t launch_col_cfg(const PassArgs& a, cudaStream_t st, int* nparts) {
  const size_t smem = col_smem_bytes<Rl, N, T, CP>();
  auto kern = col_pass_kernel<Rl, N, T, CP, MINB>;
  static PerDeviceOnce attr;  // per device: the attribute is set on the device current at the call
  cudaError_t e = set_smem_once(attr, kern, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(a.X / (2 * CP), a.batch);
  if (nparts) *nparts = grid.x;
  kern<<<grid, CP * T, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename Rl, int N>
static cudaError_t launch_col_n(const PassArgs& a, cudaStream_t st, int* nparts) {
  if (a.small_shape) {
    using Cfg = ColCfgSmall<Rl, N>;
    return launch_col_cfg<Rl, N, Cfg::T, Cfg::CP, Cfg::MINB>(a, st, nparts);
  }
  using Cfg = ColCfg<Rl, N>;
  return launch_col_cfg<Rl, N, Cfg::T, Cfg::CP, Cfg::MINB>(a, st, nparts);
}

// Column passes of sizes the register-resident kernels do not take (P not a
// power of two in [128, 4096], or X not a multiple of their column tile) run
// the generic pass, one column pair per CTA.
static int col_cp(int dtype, int P, int small) {
  int cp = 0;
#define CPV(R, N) if (P == N) cp = small ? ColCfgSmall<R, N>::CP : ColCfg<R, N>::CP;
  if (dtype == FW_F32) { CPV(float, 128) CPV(float, 256) CPV(float, 512) CPV(float, 1024) CPV(float, 2048) CPV(float, 4096) }
  else { CPV(double, 128) CPV(double, 256) CPV(double, 512) CPV(double, 1024) CPV(double, 2048) CPV(double, 4096) }
#undef CPV
  return cp;
}

bool col_generic(int dtype, int P, int X) {
  const int cp = col_cp(dtype, P, 0);
  const int cps = col_cp(dtype, P, 1);
  return cp == 0 || X % (2 * cp) != 0 || X % (2 * cps) != 0;
}

// Partial-sum records per instance of a plan's column passes: X / (2 CP), or
// X / 2 for the generic pass.
int col_parts(int dtype, int P, int X, int small) {
  if (X < 2 || X % 2 != 0) return -1;
  if (col_generic(dtype, P, X)) return X / 2;
  int cp = 0;
#define CPV(R, N) if (P == N) cp = small ? ColCfgSmall<R, N>::CP : ColCfg<R, N>::CP;
  if (dtype == FW_F32) { CPV(float, 128) CPV(float, 256) CPV(float, 512) CPV(float, 1024) CPV(float, 2048) CPV(float, 4096) }
  else { CPV(double, 128) CPV(double, 256) CPV(double, 512) CPV(double, 1024) CPV(double, 2048) CPV(double, 4096) }
#undef CPV
  if (cp == 0 || X % (2 * cp) != 0) return -1;
  return X / (2 * cp);
}

// Values per thread of the row pass transform of length N (the radix plan
// its stage-layout twiddle table is built for).
int row_rv(int dtype, int N, int small) {
  if (!size_pow2_supported(N)) return 0;  // generic row pass: k-indexed twiddles
  int t = 0;
#define RT(R, N_) if (N == N_) t = small ? RowCfgSmall<R, N_>::T : RowCfg<R, N_>::T;
  if (dtype == FW_F32) { RT(float, 128) RT(float, 256) RT(float, 512) RT(float, 1024) RT(float, 2048) RT(float, 4096) }
  else { RT(double, 128) RT(double, 256) RT(double, 512) RT(double, 1024) RT(double, 2048) RT(double, 4096) }
#undef RT
  return t > 0 ? N / t : 0;
}
// Small-batch shapes when the column pass with the regular shapes would have
// fewer CTAs than the GPU has SMs.
int small_shapes(int dtype, int P, int X, int batch) {
  if (col_generic(dtype, P, X) || !size_pow2_supported(X)) return 0;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int np = col_parts(dtype, P, X, 0);
  return np > 0 && (long long)batch * np < sms ? 1 : 0;
}

bool size_pow2_supported(int n) { return n == 128 || n == 256 || n == 512 || n == 1024 || n == 2048 || n == 4096; }
bool size_supported(int n) { return n >= 4 && n <= 4096 && n % 2 == 0; }

cudaError_t launch_row(const PassArgs& a, int dtype, cudaStream_t st) {
  if (!size_pow2_supported(a.X)) return launch_generic_row(a, dtype, st);
  if (rowp_eligible(a, dtype)) return launch_row_persist(a, st);
#define ROWN(R, N) case N: return launch_row_n<R, N>(a, st);
  if (dtype == FW_F32) {
    switch (a.X) { ROWN(float, 128) ROWN(float, 256) ROWN(float, 512) ROWN(float, 1024) ROWN(float, 2048) ROWN(float, 4096) }
  } else {
    switch (a.X) { ROWN(double, 128) ROWN(double, 256) ROWN(double, 512) ROWN(double, 1024) ROWN(double, 2048) ROWN(double, 4096) }
  }
#undef ROWN
  return cudaErrorInvalidValue;
}

cudaError_t launch_col(const PassArgs& a, int dtype, cudaStream_t st, int* nparts) {
  if (col_generic(dtype, a.P, a.X)) return launch_generic_col(a, dtype, st, nparts);
  if (colp_eligible(a, dtype)) return launch_col_persist(a, st, nparts);
#define COLN(R, N) case N: return launch_col_n<R, N>(a, st, nparts);
  if (dtype == FW_F32) {
    switch (a.P) { COLN(float, 128) COLN(float, 256) COLN(float, 512) COLN(float, 1024) COLN(float, 2048) COLN(float, 4096) }
  } else {
    switch (a.P) { COLN(double, 128) COLN(double, 256) COLN(double, 512) COLN(double, 1024) COLN(double, 2048) COLN(double, 4096) }
  }
#undef COLN
  return cudaErrorInvalidValue;
}

cudaError_t launch_finalize(const PassArgs& a, int dtype, cudaStream_t st) {
  const size_t n = (size_t)a.P * a.X;
  const int per = dtype == FW_F32 ? 4 : 2;  // elements per 16-byte vector
  const int vec = (reinterpret_cast<uintptr_t>(a.W) & 15) == 0 && a.w_bs % per == 0 && n % per == 0;
  const size_t units = vec ? n / per : n;
  // about eight 256-thread blocks per SM over the whole batch
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long blocks = (8LL * sms + a.batch - 1) / a.batch;
  const long long need = (long long)((units + 255) / 256);
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  dim3 grid((unsigned)blocks, a.batch);
  if (dtype == FW_F32) finalize_kernel<float><<<grid, 256, 0, st>>>(a, vec);
  else finalize_kernel<double><<<grid, 256, 0, st>>>(a, vec);
  return cudaGetLastError();
}

// Forward DFT Wh[k] = sum_p w[p] exp(-2 pi i k p / P) of each p-observable
// weight vector, in FP64 (radix-2 Stockham through shared memory, one CTA per
// vector, twiddles from sincospi of an exact power-of-two ratio), rounded once
// to the state precision, stored bin-major out[b][k][q] (4 slots per bin).
// Block (q, b): vector q of instance b.
template <typename Rl>
__global__ void __launch_bounds__(256) pweight_dft_kernel(const double* wp, long long wp_bs, int P, void* out,
                                                          long long out_bs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* x = reinterpret_cast<double2*>(smem_raw);
  double2* y = x + P;
  const int q = blockIdx.x, b = blockIdx.y;
  const double* w = wp + (size_t)b * wp_bs + (size_t)q * P;
  for (int i = threadIdx.x; i < P; i += blockDim.x) x[i] = make_double2(w[i], 0.0);
  __syncthreads();
  const int h = P / 2;
  for (int ns = 1; ns < P; ns <<= 1) {
    for (int jj = threadIdx.x; jj < h; jj += blockDim.x) {
      const double2 v0 = x[jj], v1 = x[jj + h];
      const int k = jj & (ns - 1);
      double s, c;
      sincospi(-(double)k / (double)ns, &s, &c);
      const double tx = v1.x * c - v1.y * s, ty = v1.x * s + v1.y * c;
      const int d = 2 * (jj - k) + k;
      y[d] = make_double2(v0.x + tx, v0.y + ty);
      y[d + ns] = make_double2(v0.x - tx, v0.y - ty);
    }
    __syncthreads();
    double2* t = x;
    x = y;
    y = t;
  }
  cplx_t<Rl>* o = reinterpret_cast<cplx_t<Rl>*>(out) + (size_t)b * out_bs + q;  // [k][4] layout
  for (int i = threadIdx.x; i < P; i += blockDim.x) o[(size_t)i * 4] = mk<cplx_t<Rl>>((Rl)x[i].x, (Rl)x[i].y);
}

cudaError_t launch_pweight_dft(const double* wp, long long wp_bs, int Mp, int P, int nb, void* out, long long out_bs,
                               int dtype, cudaStream_t st) {
  const size_t smem = 2 * sizeof(double2) * (size_t)P;
  dim3 grid(Mp, nb);
  cudaError_t e;
  if (dtype == FW_F32) {
    e = cudaFuncSetAttribute(pweight_dft_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    pweight_dft_kernel<float><<<grid, 256, smem, st>>>(wp, wp_bs, P, out, out_bs);
  } else {
    e = cudaFuncSetAttribute(pweight_dft_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    pweight_dft_kernel<double><<<grid, 256, smem, st>>>(wp, wp_bs, P, out, out_bs);
  }
  return cudaGetLastError();
}

}  // namespace fw
