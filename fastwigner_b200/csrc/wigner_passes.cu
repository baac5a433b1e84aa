// Fused half-step passes for real Wigner functions W(x, p) (Moyal, Bloch,
// random-collision).  A row pass (kinetic step) transforms along x, a column
// pass (potential step) along p.  Each CTA streams its tile from HBM once,
// runs forward FFT -> spectral multiply -> inverse FFT (twice for a fused
// column pass) out of registers and shared memory, and writes the tile back
// once.  Two real rows/columns are packed into one complex FFT.
#include "passes.cuh"
#include "fw_internal.h"

namespace fw {

// ---------------------------------------------------------------------------
// spectral multiply between a forward and an inverse transform (shared by the
// row and column passes).  v holds the natural-order spectrum Z of a + i b.
// taba/tabb point at the half-spectrum factors of the two packed sequences;
// tab_stride is the distance between consecutive half-spectrum entries.
template <typename Rl, int N, int T, int RV, typename EX>
__device__ __forceinline__ void spectral_mul(cplx_t<Rl> (&v)[RV], const int j, EX& ex, const void* taba,
                                             const void* tabb, size_t tab_stride, int tab_real, const void* g,
                                             Rl f) {
  using C = cplx_t<Rl>;
#pragma unroll
  for (int m = 0; m < RV; ++m) ex.write(j + m * T, v[m]);
  ex.sync();
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int k = j + m * T;
    const int kk = (k <= N / 2) ? k : N - k;
    C ea = tab_load<Rl>(taba, tab_real, (size_t)kk * tab_stride);
    C eb = tab_load<Rl>(tabb, tab_real, (size_t)kk * tab_stride);
    if (g != nullptr) {
      const C gk = __ldg(reinterpret_cast<const C*>(g) + kk);
      ea = cmul(ea, gk);
      eb = cmul(eb, gk);
    }
    ea = herm(ea, k, N);
    eb = herm(eb, k, N);
    const C znk = ex.read((N - k) & (N - 1));
    v[m] = two_real_mul(v[m], znk, ea, eb, f);
  }
  ex.sync();
}

// ---------------------------------------------------------------------------
// Row pass: G groups of T threads, each group owns one pair of rows.
template <typename Rl, int N, int T, int G, int MINB>
__global__ void __launch_bounds__(G* T, MINB) row_pass_kernel(PassArgs a) {
  using C = cplx_t<Rl>;
  constexpr int RV = N / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[34];
  const int b = blockIdx.y;
  const double sc = prev_scale(a, b, red);
  const int g = threadIdx.x / T;
  const int j = threadIdx.x % T;
  const int rp = blockIdx.x * G + g;
  if (2 * rp >= a.P) return;  // group-scoped synchronisation only below
  constexpr int BUF = N + N / 32;
  Rl* base = reinterpret_cast<Rl*>(smem_raw) + (size_t)g * 2 * BUF;
  GroupEx<Rl, T> ex{base, base + BUF, 1 + g};
  Rl* W = reinterpret_cast<Rl*>(a.W) + (size_t)b * a.w_bs + (size_t)(2 * rp) * N;
  const C* tw = reinterpret_cast<const C*>(a.tw);
  C v[RV];
  const Rl s = (Rl)sc;
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int x = j + m * T;
    v[m] = mk<C>(W[x] * s, W[N + x] * s);
  }
  fft<N, T, RV, -1>(v, j, ex, tw);
  const size_t esz = a.tab_real ? sizeof(Rl) : sizeof(C);
  const size_t hs = N / 2 + 1;
  const char* tb = reinterpret_cast<const char*>(a.tab1) + ((size_t)b * a.tab_bs + (size_t)(2 * rp) * hs) * esz;
  const Rl f = (Rl)(a.out_scale / (double)N);
  spectral_mul<Rl, N, T, RV>(v, j, ex, tb, tb + hs * esz, 1, a.tab_real, a.g1, f);
  fft<N, T, RV, +1>(v, j, ex, tw);
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int x = j + m * T;
    W[x] = v[m].x;
    W[N + x] = v[m].y;
  }
}

// ---------------------------------------------------------------------------
// Column pass: CP column pairs per CTA, T threads per column pair.  Thread
// (c, j) = (tid % CP, tid / CP): a warp reads 32/CP consecutive rows of
// 2*CP consecutive reals (coalesced), the CP FFTs are interleaved in shared
// memory.
constexpr int MAXO = 4;  // max x- and p-observables per pass

template <typename Rl> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

template <typename Rl, int N, int T, int CP, int S, int MINB>
__global__ void __launch_bounds__(CP* T, MINB) col_pass_kernel(PassArgs a) {
  using C = cplx_t<Rl>;
  using V2 = typename Vec2<Rl>::type;
  constexpr int RV = N / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[34];
  __shared__ double ored[(CP * T) / 32][2 + 2 * MAXO];
  const int b = blockIdx.y;
  const double sc = prev_scale(a, b, red);
  const int c = threadIdx.x % CP;
  const int j = threadIdx.x / CP;
  const int X = a.X;
  const int xa = blockIdx.x * 2 * CP + 2 * c;
  Rl* re = reinterpret_cast<Rl*>(smem_raw);
  ColEx<Rl, CP, S> ex{re, re + (size_t)N * CP, c};
  Rl* W = reinterpret_cast<Rl*>(a.W) + (size_t)b * a.w_bs;
  const C* tw = reinterpret_cast<const C*>(a.tw);
  C v[RV];
  const Rl s = (Rl)sc;
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int p = j + m * T;
    const V2 w = *reinterpret_cast<const V2*>(W + (size_t)p * X + xa);
    v[m] = mk<C>(w.x * s, w.y * s);
  }
  if (a.blend_pre) {
    const Rl* S0 = reinterpret_cast<const Rl*>(a.s0) + (size_t)b * a.s0_bs;
    const Rl bc = (Rl)a.blend_c;
#pragma unroll
    for (int m = 0; m < RV; ++m) {
      const int p = j + m * T;
      const V2 w0 = __ldg(reinterpret_cast<const V2*>(S0 + (size_t)p * X + xa));
      v[m] = mk<C>(bc * v[m].x + w0.x, bc * v[m].y + w0.y);
    }
  }
  const size_t esz = a.tab_real ? sizeof(Rl) : sizeof(C);
  const Rl f = (Rl)(1.0 / (double)N);
  if (a.tab1 != nullptr) {
    fft<N, T, RV, -1>(v, j, ex, tw);
    const char* tb = reinterpret_cast<const char*>(a.tab1) + ((size_t)b * a.tab_bs + xa) * esz;
    spectral_mul<Rl, N, T, RV>(v, j, ex, tb, tb + esz, (size_t)X, a.tab_real, a.g1, f);
    fft<N, T, RV, +1>(v, j, ex, tw);
  }
  if (a.bxp != nullptr) {
    const Rl* B = reinterpret_cast<const Rl*>(a.bxp) + (size_t)b * a.bxp_bs;
#pragma unroll
    for (int m = 0; m < RV; ++m) {
      const int p = j + m * T;
      const V2 w = __ldg(reinterpret_cast<const V2*>(B + (size_t)p * X + xa));
      v[m] = mk<C>(v[m].x * w.x, v[m].y * w.y);
    }
  }
  if (a.blend_post) {
    const Rl* S0 = reinterpret_cast<const Rl*>(a.s0) + (size_t)b * a.s0_bs;
    const Rl bc = (Rl)a.blend_c;
#pragma unroll
    for (int m = 0; m < RV; ++m) {
      const int p = j + m * T;
      const V2 w0 = __ldg(reinterpret_cast<const V2*>(S0 + (size_t)p * X + xa));
      v[m] = mk<C>(bc * v[m].x + w0.x, bc * v[m].y + w0.y);
    }
  }
  if (a.part_out != nullptr) {
    double acc[2 + 2 * MAXO];
#pragma unroll
    for (int q = 0; q < 2 + 2 * MAXO; ++q) acc[q] = 0.0;
    double ca = 0.0, cb = 0.0;
    const double* wp = a.wp + (size_t)b * a.wp_bs;
    const int P = N;
#pragma unroll
    for (int m = 0; m < RV; ++m) {
      const double wa = (double)v[m].x, wb = (double)v[m].y;
      ca += wa;
      cb += wb;
      acc[1] += wa * wa + wb * wb;
      const int p = j + m * T;
#pragma unroll
      for (int q = 0; q < MAXO; ++q)
        if (q < a.Mp) acc[2 + MAXO + q] += (wa + wb) * __ldg(wp + (size_t)q * P + p);
    }
    acc[0] = ca + cb;
    const double* wx = a.wx + (size_t)b * a.wx_bs;
#pragma unroll
    for (int q = 0; q < MAXO; ++q)
      if (q < a.Mx) acc[2 + q] = ca * __ldg(wx + (size_t)q * X + xa) + cb * __ldg(wx + (size_t)q * X + xa + 1);
#pragma unroll
    for (int q = 0; q < 2 + 2 * MAXO; ++q)
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
      for (int q = 0; q < 2 + 2 * MAXO; ++q) ored[warp][q] = acc[q];
    }
    __syncthreads();
    if (threadIdx.x < a.M) {
      // output layout: [sum, sum sq, x-obs (Mx), p-obs (Mp)]
      const int mo = threadIdx.x;
      const int q = mo < 2 + a.Mx ? mo : 2 + MAXO + (mo - 2 - a.Mx);
      double t = 0.0;
      for (int w = 0; w < (CP * T) / 32; ++w) t += ored[w][q];
      a.part_out[((size_t)b * gridDim.x + blockIdx.x) * a.M + mo] = t;
    }
  }
  if (a.tab2 != nullptr) {
    fft<N, T, RV, -1>(v, j, ex, tw);
    const char* tb = reinterpret_cast<const char*>(a.tab2) + ((size_t)b * a.tab_bs + xa) * esz;
    spectral_mul<Rl, N, T, RV>(v, j, ex, tb, tb + esz, (size_t)X, a.tab_real, a.g2, f);
    fft<N, T, RV, +1>(v, j, ex, tw);
  }
  const Rl os = (Rl)a.out_scale;
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int p = j + m * T;
    V2 w;
    w.x = v[m].x * os;
    w.y = v[m].y * os;
    *reinterpret_cast<V2*>(W + (size_t)p * X + xa) = w;
  }
}

// ---------------------------------------------------------------------------
// finalize: apply the last step's normalisation and reduce its partials.
template <typename Rl>
__global__ void finalize_kernel(PassArgs a) {
  __shared__ double red[34];
  const int b = blockIdx.y;
  const double sc = prev_scale(a, b, red);
  Rl* W = reinterpret_cast<Rl*>(a.W) + (size_t)b * a.w_bs;
  const size_t n = (size_t)a.P * a.X;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    W[i] = (Rl)(W[i] * sc);
}

// ---------------------------------------------------------------------------
// Launch configuration per FFT length and precision.
template <typename Rl, int N> struct RowCfg;
template <typename Rl, int N> struct ColCfg;
// float: T threads per transform, RV = N / T values per thread
template <> struct RowCfg<float, 128> { static constexpr int T = 16, G = 16, MINB = 1; };
template <> struct RowCfg<float, 256> { static constexpr int T = 32, G = 4, MINB = 2; };
template <> struct RowCfg<float, 512> { static constexpr int T = 32, G = 4, MINB = 2; };
template <> struct RowCfg<float, 1024> { static constexpr int T = 32, G = 4, MINB = 2; };
template <> struct RowCfg<float, 2048> { static constexpr int T = 64, G = 4, MINB = 1; };
template <> struct RowCfg<float, 4096> { static constexpr int T = 128, G = 2, MINB = 1; };
template <> struct RowCfg<double, 128> { static constexpr int T = 16, G = 16, MINB = 1; };
template <> struct RowCfg<double, 256> { static constexpr int T = 16, G = 16, MINB = 1; };
template <> struct RowCfg<double, 512> { static constexpr int T = 32, G = 8, MINB = 1; };
template <> struct RowCfg<double, 1024> { static constexpr int T = 64, G = 4, MINB = 1; };
template <> struct RowCfg<double, 2048> { static constexpr int T = 128, G = 2, MINB = 1; };
template <> struct RowCfg<double, 4096> { static constexpr int T = 256, G = 1, MINB = 1; };

template <> struct ColCfg<float, 128> { static constexpr int T = 16, CP = 32, MINB = 1; };
template <> struct ColCfg<float, 256> { static constexpr int T = 32, CP = 16, MINB = 1; };
template <> struct ColCfg<float, 512> { static constexpr int T = 32, CP = 16, MINB = 1; };
template <> struct ColCfg<float, 1024> { static constexpr int T = 64, CP = 8, MINB = 1; };
template <> struct ColCfg<float, 2048> { static constexpr int T = 64, CP = 8, MINB = 1; };
template <> struct ColCfg<float, 4096> { static constexpr int T = 128, CP = 4, MINB = 1; };
template <> struct ColCfg<double, 128> { static constexpr int T = 16, CP = 16, MINB = 1; };
template <> struct ColCfg<double, 256> { static constexpr int T = 16, CP = 16, MINB = 1; };
template <> struct ColCfg<double, 512> { static constexpr int T = 32, CP = 8, MINB = 1; };
template <> struct ColCfg<double, 1024> { static constexpr int T = 64, CP = 8, MINB = 1; };
template <> struct ColCfg<double, 2048> { static constexpr int T = 128, CP = 4, MINB = 1; };
template <> struct ColCfg<double, 4096> { static constexpr int T = 256, CP = 2, MINB = 1; };

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

template <typename Rl, int N>
static cudaError_t launch_row_n(const PassArgs& a, cudaStream_t st) {
  using Cfg = RowCfg<Rl, N>;
  constexpr int T = Cfg::T, G = Cfg::G, MINB = Cfg::MINB;
  const size_t smem = (size_t)G * 2 * (N + N / 32) * sizeof(Rl);
  auto kern = row_pass_kernel<Rl, N, T, G, MINB>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid((a.P / 2 + G - 1) / G, a.batch);
  kern<<<grid, G * T, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename Rl, int N>
static cudaError_t launch_col_n(const PassArgs& a, cudaStream_t st, int* nparts) {
  using Cfg = ColCfg<Rl, N>;
  constexpr int T = Cfg::T, CP = Cfg::CP, MINB = Cfg::MINB;
  constexpr int S = ilog2(N / T > 32 ? 32 : N / T);
  const size_t smem = (size_t)2 * N * CP * sizeof(Rl);
  auto kern = col_pass_kernel<Rl, N, T, CP, S, MINB>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid(a.X / (2 * CP), a.batch);
  if (nparts) *nparts = grid.x;
  kern<<<grid, CP * T, smem, st>>>(a);
  return cudaGetLastError();
}

int col_parts(int dtype, int P, int X) {
  int cp = 0;
#define CPV(R, N) if (P == N) cp = ColCfg<R, N>::CP;
  if (dtype == FW_F32) { CPV(float, 128) CPV(float, 256) CPV(float, 512) CPV(float, 1024) CPV(float, 2048) CPV(float, 4096) }
  else { CPV(double, 128) CPV(double, 256) CPV(double, 512) CPV(double, 1024) CPV(double, 2048) CPV(double, 4096) }
#undef CPV
  if (cp == 0 || X % (2 * cp) != 0) return -1;
  return X / (2 * cp);
}

bool size_supported(int n) { return n == 128 || n == 256 || n == 512 || n == 1024 || n == 2048 || n == 4096; }

cudaError_t launch_row(const PassArgs& a, int dtype, cudaStream_t st) {
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
  int blocks = (int)((n + 255) / 256);
  if (blocks > 1184) blocks = 1184;
  dim3 grid(blocks, a.batch);
  if (dtype == FW_F32) finalize_kernel<float><<<grid, 256, 0, st>>>(a);
  else finalize_kernel<double><<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace fw
