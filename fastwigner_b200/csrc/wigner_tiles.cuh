// Device-side work items of the Wigner-function passes (row pass: pairs of
// rows; column pass: tiles of column pairs), shared by the per-pass kernels
// (wigner_passes.cu) and the persistent batched kernel (batch.cu).
#pragma once
#include "passes.cuh"

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
// One CTA-sized work item of a row pass: instance b, row pairs blk*G .. blk*G+G-1.
template <typename Rl, int N, int T, int G>
__device__ __forceinline__ void row_tile(const PassArgs& a, int b, int blk, unsigned char* smem_raw, double* red) {
  using C = cplx_t<Rl>;
  constexpr int RV = N / T;
  const double sc = prev_scale(a, b, red, blk == 0);
  const int g = threadIdx.x / T;
  const int j = threadIdx.x % T;
  const int rp = blk * G + g;
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
    v[m] = mk<C>(__ldcg(W + x) * s, __ldcg(W + N + x) * s);
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

// One work item of a column pass: instance b, column pairs tile*CP .. tile*CP+CP-1
// (ntiles = X / (2 CP) tiles per instance, the partial-sum records per instance).
template <typename Rl, int N, int T, int CP, int S>
__device__ __forceinline__ void col_tile(const PassArgs& a, int b, int tile, int ntiles, unsigned char* smem_raw,
                                         double* red, double (*ored)[2 + 2 * MAXO]) {
  using C = cplx_t<Rl>;
  using V2 = typename Vec2<Rl>::type;
  constexpr int RV = N / T;
  const double sc = prev_scale(a, b, red, tile == 0);
  const int c = threadIdx.x % CP;
  const int j = threadIdx.x / CP;
  const int X = a.X;
  const int xa = tile * 2 * CP + 2 * c;
  Rl* re = reinterpret_cast<Rl*>(smem_raw);
  ColEx<Rl, CP, S> ex{re, re + (size_t)N * CP, c};
  Rl* W = reinterpret_cast<Rl*>(a.W) + (size_t)b * a.w_bs;
  const C* tw = reinterpret_cast<const C*>(a.tw);
  C v[RV];
  const Rl s = (Rl)sc;
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int p = j + m * T;
    const V2 w = __ldcg(reinterpret_cast<const V2*>(W + (size_t)p * X + xa));
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
      a.part_out[((size_t)b * ntiles + tile) * a.M + mo] = t;
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

}  // namespace fw
