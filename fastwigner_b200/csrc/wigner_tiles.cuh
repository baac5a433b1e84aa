// Device-side work items of the Wigner-function passes (row pass: pairs of
// rows; column pass: tiles of column pairs), shared by the per-pass kernels
// (wigner_passes.cu) and the persistent batched kernel (batch.cu).
#pragma once
#include "passes.cuh"

namespace fw {

// ---------------------------------------------------------------------------
// Factors of the two packed sequences at full-spectrum index k: table entries
// kk = min(k, N-k) (taba/tabb, tab_stride apart), times g[kk] when g is given,
// Hermitian-extended.
template <typename Rl, int N>
__device__ __forceinline__ void factor_pair(const void* taba, const void* tabb, size_t tab_stride, int tab_real,
                                            const void* g, int k, cplx_t<Rl>& ea, cplx_t<Rl>& eb) {
  using C = cplx_t<Rl>;
  const int kk = (k <= N / 2) ? k : N - k;
  ea = tab_load<Rl>(taba, tab_real, (size_t)kk * tab_stride);
  eb = tab_load<Rl>(tabb, tab_real, (size_t)kk * tab_stride);
  if (g != nullptr) {
    const C gk = __ldg(reinterpret_cast<const C*>(g) + kk);
    ea = cmul(ea, gk);
    eb = cmul(eb, gk);
  }
  ea = herm(ea, k, N);
  eb = herm(eb, k, N);
}

// factor_pair for a column pair whose two entries are adjacent in a table
// that starts on 16 bytes (taba = entry of column xa, xa even): one vector
// load per bin.
template <typename Rl, int N>
__device__ __forceinline__ void factor_pair_vec(const void* taba, size_t tab_stride, int tab_real, const void* g,
                                                int k, cplx_t<Rl>& ea, cplx_t<Rl>& eb) {
  using C = cplx_t<Rl>;
  const int kk = (k <= N / 2) ? k : N - k;
  if constexpr (sizeof(Rl) == 4) {
    if (tab_real) {
      const float2 e = __ldg(reinterpret_cast<const float2*>(reinterpret_cast<const float*>(taba) + kk * tab_stride));
      ea = mk<C>(e.x, 0.f);
      eb = mk<C>(e.y, 0.f);
    } else {
      const float4 e = __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const float2*>(taba) + kk * tab_stride));
      ea = mk<C>(e.x, e.y);
      eb = mk<C>(e.z, e.w);
    }
  } else {
    if (tab_real) {
      const double2 e = __ldg(reinterpret_cast<const double2*>(reinterpret_cast<const double*>(taba) + kk * tab_stride));
      ea = mk<C>(e.x, 0.0);
      eb = mk<C>(e.y, 0.0);
    } else {
      ea = __ldg(reinterpret_cast<const C*>(taba) + kk * tab_stride);
      eb = __ldg(reinterpret_cast<const C*>(taba) + kk * tab_stride + 1);
    }
  }
  if (g != nullptr) {
    const C gk = __ldg(reinterpret_cast<const C*>(g) + kk);
    ea = cmul(ea, gk);
    eb = cmul(eb, gk);
  }
  ea = herm(ea, k, N);
  eb = herm(eb, k, N);
}

// The first n (<= MAXO) p-weight spectra at one bin ([k][q] layout, 4 entries,
// 16-byte aligned): FP32 as one or two 16-byte loads.
template <typename Rl>
__device__ __forceinline__ void load_bin_weights(const cplx_t<Rl>* gk, int n, cplx_t<Rl> (&g)[4]) {
  using C = cplx_t<Rl>;
  if constexpr (sizeof(Rl) == 4) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(gk));
    g[0] = mk<C>(a.x, a.y);
    g[1] = mk<C>(a.z, a.w);
    if (n > 2) {
      const float4 b = __ldg(reinterpret_cast<const float4*>(gk) + 1);
      g[2] = mk<C>(b.x, b.y);
      g[3] = mk<C>(b.z, b.w);
    } else {
      g[2] = g[3] = mk<C>(0.f, 0.f);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) g[q] = q < n ? __ldg(gk + q) : mk<C>(0.0, 0.0);
  }
}

// Spectral multiply between a forward and an inverse transform (shared by the
// row and column passes).  v holds the natural-order spectrum Z of a + i b.
// taba/tabb point at the half-spectrum factors of the two packed sequences;
// tab_stride is the distance between consecutive half-spectrum entries.
template <typename Rl, int N, int T, int RV, typename EX>
__device__ __forceinline__ void spectral_mul(cplx_t<Rl> (&v)[RV], const int j, EX& ex, const void* taba,
                                             const void* tabb, size_t tab_stride, int tab_real, const void* g,
                                             Rl f) {
  using C = cplx_t<Rl>;
  ex_write_natural<T, RV>(ex, j, v);
  ex.sync();
  // When T is a multiple of the exchange's padding period, the slot of N - k
  // (k = j + m T) is one per-thread base minus an immediate for every m
  // (slot of 0 for k = 0), as in the persistent passes (Bloch 512^2 FP32,
  // 16 instances: 0.0553 -> 0.0514 ms per step; the uneven batch 0.634 ->
  // 0.620 ms).
  constexpr bool kFoldMirror = EX::kFold && T % (1 << EX::kL) == 0;
  const int mbase = kFoldMirror ? ex.map(N - j) : 0;  // virtual slot of N for j = 0
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int k = j + m * T;
    C ea, eb;
    factor_pair<Rl, N>(taba, tabb, tab_stride, tab_real, g, k, ea, eb);
    C znk;
    if constexpr (kFoldMirror) {
      znk = ex.read_at(m == 0 ? (j == 0 ? ex.map(0) : mbase) : mbase - EX::delta(m * T));
    } else {
      znk = ex.read((N - k) & (N - 1));
    }
    v[m] = two_real_mul(v[m], znk, ea, eb, f);
  }
  ex.sync();
}

// ---------------------------------------------------------------------------
// Row pass: G groups of T threads, each group owns one pair of rows.
// One CTA-sized work item of a row pass: instance b, row pairs blk*G .. blk*G+G-1.
// STW: a.tw is the stage-layout twiddle table of (N, N/T) instead of exp(-2 pi i k/N).
template <typename Rl, int N, int T, int G, bool STW = false>
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
  using EXT = GroupEx<Rl, T>;
  Rl* W = reinterpret_cast<Rl*>(a.W) + (size_t)b * a.w_bs + (size_t)(2 * rp) * N;
  const C* tw = reinterpret_cast<const C*>(a.tw);
  C v[RV];
  const Rl s = (Rl)sc;
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int x = j + m * T;
    v[m] = mk<C>(__ldcg(W + x) * s, __ldcg(W + N + x) * s);
  }
  fft<N, T, RV, -1, C, EXT, STW>(v, j, ex, tw);
  const size_t esz = a.tab_real ? sizeof(Rl) : sizeof(C);
  const size_t hs = N / 2 + 1;
  const char* tb = reinterpret_cast<const char*>(a.tab1) + ((size_t)b * a.tab_bs + (size_t)(2 * rp) * hs) * esz;
  const Rl f = (Rl)(a.out_scale / (double)N);
  spectral_mul<Rl, N, T, RV>(v, j, ex, tb, tb + hs * esz, 1, a.tab_real, a.g1, f);
  fft<N, T, RV, +1, C, EXT, STW>(v, j, ex, tw);
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

// Reduce the per-thread observable accumulators over the CTA and write the
// tile's partial-sum record [sum, sum sq, x-obs (Mx), p-obs (Mp)].  Called by
// every thread of the CTA.
template <int NTHR>
__device__ __forceinline__ void obs_store(const PassArgs& a, int b, int tile, int ntiles, double (&acc)[2 + 2 * MAXO],
                                          double (*ored)[2 + 2 * MAXO]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)  // level-major: the accumulators reduce in parallel
#pragma unroll
    for (int q = 0; q < 2 + 2 * MAXO; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int q = 0; q < 2 + 2 * MAXO; ++q) ored[warp][q] = acc[q];
  }
  __syncthreads();
  if (threadIdx.x < a.M) {
    const int mo = threadIdx.x;
    const int q = mo < 2 + a.Mx ? mo : 2 + MAXO + (mo - 2 - a.Mx);
    double t = 0.0;
    for (int w = 0; w < NTHR / 32; ++w) t += ored[w][q];
    a.part_out[((size_t)b * ntiles + tile) * a.M + mo] = t;
  }
}

// Store a column pair (rows j, j+T, ...) times out_scale.
template <typename Rl, int N, int T, int RV>
__device__ __forceinline__ void col_store(const PassArgs& a, const cplx_t<Rl> (&v)[RV], Rl* W, int j, int xa) {
  using V2 = typename Vec2<Rl>::type;
  const Rl os = (Rl)a.out_scale;
  const int X = a.X;
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int p = j + m * T;
    V2 w;
    w.x = v[m].x * os;
    w.y = v[m].y * os;
    *reinterpret_cast<V2*>(W + (size_t)p * X + xa) = w;
  }
}

// Per-thread partial sums of a fused column pass, accumulated in FP64 whatever
// the state precision: sum |2A_k|^2 + |2B_k|^2 over the thread's bins (each
// bin's four squares summed in the state precision -- positive terms, so
// that short sum has no cancellation -- then added in FP64), sum
// Re(2(A_k+B_k) conj(Wh_k)) per p-weight, and (thread j == 0 only) the
// doubled DC bins of the pair.
template <typename Rl> struct MidSums {
  double s2, sq[MAXO], ca, cb;
};

// Mid-point of a fused column pass (a.fuse_mid): v holds the forward spectrum
// Z of the column pair a + i b (columns xa, xa+1).  Split Z into the two real
// spectra, apply the closing half-step factors (tab1, g1), take the partial
// sums from the mid-point spectra, apply the opening factors of the next step
// (tab2, g2) and repack, scaled for the unnormalised inverse transform.
//   sum_p a(p)        = A_0
//   sum_p a(p)^2      = sum_k |A_k|^2 / N
//   sum_p a(p) w(p)   = sum_k Re(A_k conj(Wh_k)) / N,  Wh = DFT(w)
template <typename Rl, int N, int T, int RV, int CP, typename EX>
__device__ __forceinline__ void fused_mid(const PassArgs& a, int b, cplx_t<Rl> (&v)[RV], const int j, EX& ex,
                                          int xa, int c, cplx_t<Rl>* psum, MidSums<Rl>& o) {
  using C = cplx_t<Rl>;
  const int X = a.X;
  const size_t esz = a.tab_real ? sizeof(Rl) : sizeof(C);
  const char* t1 = reinterpret_cast<const char*>(a.tab1) + ((size_t)b * a.tab_bs + xa) * esz;
  const char* t2 = reinterpret_cast<const char*>(a.tab2) + ((size_t)b * a.tab_bs + xa) * esz;
  const bool same = a.tab1 == a.tab2 && a.g1 == a.g2;  // time-independent factors: load once
  const C* G = reinterpret_cast<const C*>(a.wph) + (size_t)b * a.wph_bs;
  const bool obs = a.part_out != nullptr;
  const Rl h = (Rl)(0.5 / (double)N);
  ex_write_natural<T, RV>(ex, j, v);
  ex.sync();
  o.s2 = 0;
  o.ca = 0;
  o.cb = 0;
#pragma unroll
  for (int q = 0; q < MAXO; ++q) o.sq[q] = 0;
  // bins per block of the paired per-bin reduction (at most CP)
  constexpr int PB = CP >= 4 ? 4 : (CP >= 2 ? 2 : 1);
  static_assert(RV % PB == 0, "bin blocks must tile the thread's bins");
  C ub[PB];
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    const int k = j + m * T;
    C ea1, eb1, ea2, eb2;
    if (a.tab_vec) {
      factor_pair_vec<Rl, N>(t1, (size_t)X, a.tab_real, a.g1, k, ea1, eb1);
    } else {
      factor_pair<Rl, N>(t1, t1 + esz, (size_t)X, a.tab_real, a.g1, k, ea1, eb1);
    }
    if (same) {
      ea2 = ea1;
      eb2 = eb1;
    } else if (a.tab_vec) {
      factor_pair_vec<Rl, N>(t2, (size_t)X, a.tab_real, a.g2, k, ea2, eb2);
    } else {
      factor_pair<Rl, N>(t2, t2 + esz, (size_t)X, a.tab_real, a.g2, k, ea2, eb2);
    }
    const C zc = cconj(ex.read((N - k) & (N - 1)));
    const C A = cmul(cadd(v[m], zc), ea1);   // 2 x spectrum of column a at the mid-point
    const C Bi = cmul(csub(v[m], zc), eb1);  // 2i x spectrum of column b at the mid-point
    if (obs) {
      o.s2 += (double)(A.x * A.x + A.y * A.y + Bi.x * Bi.x + Bi.y * Bi.y);
      if (m == 0 && j == 0) {  // DC bin: the column sums
        o.ca = A.x;
        o.cb = Bi.y;
      }
      if (a.Mp > 0) {
        // 2 x (spectrum a + spectrum b), summed over the tile's CP column pairs
        // (lanes c of one row group are adjacent) for a block of PB bins at a
        // time: the first log2(PB) shuffle levels scatter the block (a lane
        // keeps half of its values and sends the other half), the rest sum one
        // value, and one lane per bin stores it (FP64 256^2, batch 512: 0.5266 ->
        // 0.5070 ms per step against a full butterfly per bin)
        ub[m % PB] = mk<C>(A.x + Bi.y, A.y - Bi.x);
        if (m % PB == PB - 1) {
          C kp = ub[0];
          int vi = 0;
          if constexpr (PB == 4) {
            const bool up = (c & (CP / 2)) != 0, up2 = (c & (CP / 4)) != 0;
            C k0 = up ? ub[2] : ub[0], k1 = up ? ub[3] : ub[1];
            const C s0 = up ? ub[0] : ub[2], s1 = up ? ub[1] : ub[3];
            k0 = cadd(k0, mk<C>(__shfl_xor_sync(0xffffffffu, s0.x, CP / 2), __shfl_xor_sync(0xffffffffu, s0.y, CP / 2)));
            k1 = cadd(k1, mk<C>(__shfl_xor_sync(0xffffffffu, s1.x, CP / 2), __shfl_xor_sync(0xffffffffu, s1.y, CP / 2)));
            kp = up2 ? k1 : k0;
            const C s = up2 ? k0 : k1;
            kp = cadd(kp, mk<C>(__shfl_xor_sync(0xffffffffu, s.x, CP / 4), __shfl_xor_sync(0xffffffffu, s.y, CP / 4)));
            vi = (up ? 2 : 0) + (up2 ? 1 : 0);
          } else if constexpr (PB == 2) {
            const bool up = (c & (CP / 2)) != 0;
            kp = up ? ub[1] : ub[0];
            const C s = up ? ub[0] : ub[1];
            kp = cadd(kp, mk<C>(__shfl_xor_sync(0xffffffffu, s.x, CP / 2), __shfl_xor_sync(0xffffffffu, s.y, CP / 2)));
            vi = up ? 1 : 0;
          }
#pragma unroll
          for (int off = CP / (2 * PB); off > 0; off >>= 1) {
            kp.x += __shfl_xor_sync(0xffffffffu, kp.x, off);
            kp.y += __shfl_xor_sync(0xffffffffu, kp.y, off);
          }
          if ((c & (CP / PB - 1)) == 0) psum[j + (m - (PB - 1) + vi) * T] = kp;
        }
      }
    }
    v[m] = cscale(cadd(cmul(A, ea2), cmul(Bi, eb2)), h);
  }
  ex.sync();
  if (obs && a.Mp > 0) {
    // the p-weight sums: each bin's tile sum against its weight spectra, the
    // weights loaded once per bin and CTA
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
      const C u = psum[k];
      C g[MAXO];
      load_bin_weights<Rl>(G + (size_t)k * MAXO, a.Mp, g);
#pragma unroll
      for (int q = 0; q < MAXO; ++q)
        if (q < a.Mp) o.sq[q] += (double)u.x * (double)g[q].x + (double)u.y * (double)g[q].y;
    }
  }
}

// Reduce MidSums over the CTA (column-interleaved layout: lane c of a row
// group is column pair c) and write the tile's partial-sum record.  The bin
// sums reduce in FP64 within each warp (shuffle tree) and across warps; the
// DC terms live in threads j == 0 (tid < CP, all in warp 0).
template <typename Rl, int N, int CP, int NTHR>
__device__ __forceinline__ void mid_store(const PassArgs& a, int b, int tile, int ntiles, MidSums<Rl>& o, int xa,
                                          double (*ored)[2 + 2 * MAXO]) {
  static_assert(CP <= 32, "DC lanes must sit in warp 0");
  static_assert(MAXO == 4, "the paired reduction below takes s2 and three bin sums");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {
    // s2 and the first three bin sums (zero beyond Mp) reduce together: at
    // each of the first two levels a lane keeps half of its values and sends
    // the other half, so the four cost 2 + 1 + 3 shuffles instead of 4 x 5.
    // Lane 8 v ends with the warp's total of value v (s2, sq0, sq1, sq2).
    // (Persistent column pass: 0.3047 -> 0.2888 ms per 64 x 1024^2 launch.)
    const bool h16 = (lane & 16) != 0, h8 = (lane & 8) != 0;
    double k0 = h16 ? o.sq[1] : o.s2, k1 = h16 ? o.sq[2] : o.sq[0];
    const double s0 = h16 ? o.s2 : o.sq[1], s1 = h16 ? o.sq[0] : o.sq[2];
    k0 += __shfl_xor_sync(0xffffffffu, s0, 16);
    k1 += __shfl_xor_sync(0xffffffffu, s1, 16);
    double k = h8 ? k1 : k0;
    k += __shfl_xor_sync(0xffffffffu, h8 ? k0 : k1, 8);
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) k += __shfl_xor_sync(0xffffffffu, k, off);
    if ((lane & 7) == 0) {
      const int v = lane >> 3;
      if (v == 0) ored[warp][1] = k * (0.25 / (double)N);
      else ored[warp][2 + MAXO + v - 1] = k * (0.5 / (double)N);
    }
    if (a.Mp > 3) {
      double k3 = o.sq[3];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) k3 += __shfl_xor_sync(0xffffffffu, k3, off);
      if (lane == 0) ored[warp][2 + MAXO + 3] = k3 * (0.5 / (double)N);
    }
  }
  if (warp == 0) {
    const double da = 0.5 * o.ca, db = 0.5 * o.cb;
    double d[1 + MAXO];
    d[0] = da + db;
    const double* wx = a.wx + (size_t)b * a.wx_bs;
#pragma unroll
    for (int q = 0; q < MAXO; ++q)
      d[1 + q] = (lane < CP && q < a.Mx) ? da * __ldg(wx + (size_t)q * a.X + xa) + db * __ldg(wx + (size_t)q * a.X + xa + 1)
                                         : 0.0;
#pragma unroll
    for (int off = CP / 2; off > 0; off >>= 1)
#pragma unroll
      for (int q = 0; q < 1 + MAXO; ++q) d[q] += __shfl_xor_sync(0xffffffffu, d[q], off);
    if (lane == 0) {
      ored[0][0] = d[0];
#pragma unroll
      for (int q = 0; q < MAXO; ++q) ored[0][2 + q] = d[1 + q];
    }
  }
  __syncthreads();
  if (threadIdx.x < a.M) {
    const int mo = threadIdx.x;
    const int q = mo < 2 + a.Mx ? mo : 2 + MAXO + (mo - 2 - a.Mx);
    double t;
    if (q == 0 || (q >= 2 && q < 2 + MAXO)) {
      t = ored[0][q];
    } else {
      t = 0.0;
      for (int w = 0; w < NTHR / 32; ++w) t += ored[w][q];
    }
    a.part_out[((size_t)b * ntiles + tile) * a.M + mo] = t;
  }
}

// One work item of a column pass: instance b, column pairs tile*CP .. tile*CP+CP-1
// (ntiles = X / (2 CP) tiles per instance, the partial-sum records per instance).
// Reals of shared memory a column tile's exchange buffer takes: CP
// interleaved transforms, two components, one pad slot per RV = N/T elements.
template <typename Rl, int N, int T, int CP> constexpr size_t col_ex_reals() { return (size_t)2 * (N + T) * CP; }
// Dynamic shared memory of a column tile: the exchange buffer, then N complex
// per-bin sums of the tile's column spectra (p-observables of the fused pass).
template <typename Rl, int N, int T, int CP> constexpr size_t col_smem_bytes() {
  return (col_ex_reals<Rl, N, T, CP>() + (size_t)2 * N) * sizeof(Rl);
}

template <typename Rl, int N, int T, int CP, bool STW = false>
__device__ __forceinline__ void col_tile(const PassArgs& a, int b, int tile, int ntiles, unsigned char* smem_raw,
                                         double* red, double (*ored)[2 + 2 * MAXO]) {
  using C = cplx_t<Rl>;
  using V2 = typename Vec2<Rl>::type;
  constexpr int RV = N / T;
  const double sc = prev_scale(a, b, red, tile == 0);
  const int c = threadIdx.x % CP;
  const int j = threadIdx.x / CP;
  // every launch of a column tile has exactly CP * T threads; telling the
  // compiler lets it resolve which half of the spectrum bin k = j + m T lies in
  __builtin_assume(j >= 0 && j < T);
  const int X = a.X;
  const int xa = tile * 2 * CP + 2 * c;
  Rl* re = reinterpret_cast<Rl*>(smem_raw);
  using EXT = ColPadEx<Rl, CP, ilog2_c(RV)>;
  EXT ex{re, re + (size_t)(N + T) * CP, c};
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
  if (a.fuse_mid) {
    fft<N, T, RV, -1, C, EXT, STW>(v, j, ex, tw);
    MidSums<Rl> o;
    C* psum = reinterpret_cast<C*>(re + col_ex_reals<Rl, N, T, CP>());
    fused_mid<Rl, N, T, RV, CP>(a, b, v, j, ex, xa, c, psum, o);
    if (a.part_out != nullptr) mid_store<Rl, N, CP, CP * T>(a, b, tile, ntiles, o, xa, ored);
    fft<N, T, RV, +1, C, EXT, STW>(v, j, ex, tw);
    col_store<Rl, N, T, RV>(a, v, W, j, xa);
    return;
  }
  const size_t esz = a.tab_real ? sizeof(Rl) : sizeof(C);
  const Rl f = (Rl)(1.0 / (double)N);
  if (a.tab1 != nullptr) {
    fft<N, T, RV, -1, C, EXT, STW>(v, j, ex, tw);
    const char* tb = reinterpret_cast<const char*>(a.tab1) + ((size_t)b * a.tab_bs + xa) * esz;
    spectral_mul<Rl, N, T, RV>(v, j, ex, tb, tb + esz, (size_t)X, a.tab_real, a.g1, f);
    fft<N, T, RV, +1, C, EXT, STW>(v, j, ex, tw);
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
    if constexpr (sizeof(Rl) == 4) {
      // FP32 state: the 2*CP columns of a row sit in CP adjacent lanes; reduce a
      // row's sums across them with shuffles (log2 CP additions), then one lane
      // per row accumulates the FP64 weighted sums; the per-thread column sums
      // over RV rows accumulate in FP64.
      double fa = 0.0, fb = 0.0;
      constexpr int CH = RV < 8 ? RV : 8;  // rows per batch of independent shuffles
#pragma unroll
      for (int m0 = 0; m0 < RV; m0 += CH) {
        float s[CH], s2[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          const float wa = v[m0 + u].x, wb = v[m0 + u].y;
          fa += wa;
          fb += wb;
          s[u] = wa + wb;
          s2[u] = wa * wa + wb * wb;
        }
#pragma unroll
        for (int o = CP / 2; o >= 1; o >>= 1)
#pragma unroll
          for (int u = 0; u < CH; ++u) {  // level-major: CH independent shuffles in flight
            s[u] += __shfl_xor_sync(0xffffffffu, s[u], o);
            s2[u] += __shfl_xor_sync(0xffffffffu, s2[u], o);
          }
        if (c == 0) {
#pragma unroll
          for (int u = 0; u < CH; ++u) {
            const int p = j + (m0 + u) * T;
            acc[0] += (double)s[u];
            acc[1] += (double)s2[u];
#pragma unroll
            for (int q = 0; q < MAXO; ++q)
              if (q < a.Mp) acc[2 + MAXO + q] += (double)s[u] * __ldg(wp + (size_t)q * P + p);
          }
        }
      }
      ca = fa;
      cb = fb;
    } else {
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
    }
    const double* wx = a.wx + (size_t)b * a.wx_bs;
#pragma unroll
    for (int q = 0; q < MAXO; ++q)
      if (q < a.Mx) acc[2 + q] = ca * __ldg(wx + (size_t)q * X + xa) + cb * __ldg(wx + (size_t)q * X + xa + 1);
    obs_store<CP * T>(a, b, tile, ntiles, acc, ored);
  }
  if (a.tab2 != nullptr) {
    fft<N, T, RV, -1, C, EXT, STW>(v, j, ex, tw);
    const char* tb = reinterpret_cast<const char*>(a.tab2) + ((size_t)b * a.tab_bs + xa) * esz;
    spectral_mul<Rl, N, T, RV>(v, j, ex, tb, tb + esz, (size_t)X, a.tab_real, a.g2, f);
    fft<N, T, RV, +1, C, EXT, STW>(v, j, ex, tw);
  }
  col_store<Rl, N, T, RV>(a, v, W, j, xa);
}

}  // namespace fw
