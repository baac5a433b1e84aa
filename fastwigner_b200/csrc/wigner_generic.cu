// Row and column passes for grid sizes that are not powers of two.
//
// The reference accepts any even grid size (wigner_moyal_fftw_1d.py:55, 62;
// wigner_moyal_cuda_1d.py:63, 70).  The register-resident passes of
// wigner_passes.cu cover the powers of two in [128, 4096]; every other even
// size up to 4096 runs here.  One CTA owns one row pair or one column pair of
// one instance and transforms it in shared memory with a mixed-radix Stockham
// FFT: radix-4, -2, -3 and -5 butterflies written out, any other prime
// factor p as a direct p-point DFT (O(p^2) per group of p elements, so every
// even N is covered).  Twiddles come from the plan's table exp(-2 pi i k/N),
// k < N.  The passes do what the regular ones do (scaling by the previous
// step's normalisation, the split blends, the x-p mask, FP64 partial sums of
// the observables in real space, the two half-steps of a column pass), but
// never fuse the two potential half-steps: the host runs the unfused column
// pass for these sizes.
#include "fw_internal.h"
#include "wigner_tiles.cuh"

namespace fw {

constexpr int kGenThreads = 256;
constexpr int kGenMaxFactors = 24;

struct GenFactors {
  int n;                       // number of factors
  int f[kGenMaxFactors];       // radices, in the order the stages use them
};

// Factor N into 4s, then 2, 3, 5, then the remaining primes.
GenFactors gen_factors(int N) {
  GenFactors g{};
  int m = N;
  while (m % 4 == 0 && g.n < kGenMaxFactors) { g.f[g.n++] = 4; m /= 4; }
  for (int p = 2; m > 1 && g.n < kGenMaxFactors; ++p)
    while (m % p == 0 && g.n < kGenMaxFactors) { g.f[g.n++] = p; m /= p; }
  return g;
}

// One Stockham stage of radix R (R may be any factor; 2, 3, 4, 5 hard-coded)
// from x to y: butterfly t (0 <= t < N/R) with k = t mod Ns reads
// x[t + r N/R], twiddles by exp(DIR 2 pi i k r / (Ns R)), and writes
// y[(t / Ns) Ns R + k + s Ns], s = 0..R-1.
template <typename C, int DIR>
__device__ void gen_stage(const C* x, C* y, int N, int R, int Ns, const C* tw) {
  using Rl = decltype(C::x);
  const int nb = N / R;
  const int tstep = N / (Ns * R);  // twiddle index step: exp(-2 pi i k r/(Ns R)) = tw[k r tstep]
  for (int t = threadIdx.x; t < nb; t += blockDim.x) {
    const int k = t % Ns;
    const int out0 = (t / Ns) * Ns * R + k;
    C in[5];
    if (R <= 5) {
      for (int r = 0; r < R; ++r) {
        C v = x[t + r * nb];
        if (r > 0 && k > 0) {
          C w = tw[(k * r * tstep) % N];
          if (DIR > 0) w = cconj(w);
          v = cmul(v, w);
        }
        in[r] = v;
      }
    }
    if (R == 2) {
      y[out0] = cadd(in[0], in[1]);
      y[out0 + Ns] = csub(in[0], in[1]);
    } else if (R == 4) {
      const C a0 = cadd(in[0], in[2]), a1 = csub(in[0], in[2]);
      const C b0 = cadd(in[1], in[3]), b1 = mul_i<DIR>(csub(in[1], in[3]));
      y[out0] = cadd(a0, b0);
      y[out0 + Ns] = cadd(a1, b1);
      y[out0 + 2 * Ns] = csub(a0, b0);
      y[out0 + 3 * Ns] = csub(a1, b1);
    } else if (R == 3) {
      // exp(DIR 2 pi i / 3) = -1/2 + DIR i sqrt(3)/2
      const Rl h = (Rl)0.8660254037844386;
      const C s = cadd(in[1], in[2]), d = csub(in[1], in[2]);
      const C m = mk<C>(in[0].x - (Rl)0.5 * s.x, in[0].y - (Rl)0.5 * s.y);
      const C rot = mul_i<DIR>(cscale(d, h));  // DIR i sqrt(3)/2 (in1 - in2)
      y[out0] = cadd(in[0], s);
      y[out0 + Ns] = cadd(m, rot);
      y[out0 + 2 * Ns] = csub(m, rot);
    } else if (R == 5) {
      // cos/sin of 2 pi/5 and 4 pi/5
      const Rl c1 = (Rl)0.30901699437494745, c2 = (Rl)-0.8090169943749475;
      const Rl s1 = (Rl)0.9510565162951535, s2 = (Rl)0.5877852522924731;
      const C t1 = cadd(in[1], in[4]), t2 = cadd(in[2], in[3]);
      const C t3 = csub(in[1], in[4]), t4 = csub(in[2], in[3]);
      const C a1 = mk<C>(in[0].x + c1 * t1.x + c2 * t2.x, in[0].y + c1 * t1.y + c2 * t2.y);
      const C a2 = mk<C>(in[0].x + c2 * t1.x + c1 * t2.x, in[0].y + c2 * t1.y + c1 * t2.y);
      // b1 = DIR i (s1 t3 + s2 t4), b2 = DIR i (s2 t3 - s1 t4)
      const C b1 = mul_i<DIR>(mk<C>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
      const C b2 = mul_i<DIR>(mk<C>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
      y[out0] = cadd(in[0], cadd(t1, t2));
      y[out0 + Ns] = cadd(a1, b1);
      y[out0 + 4 * Ns] = csub(a1, b1);
      y[out0 + 2 * Ns] = cadd(a2, b2);
      y[out0 + 3 * Ns] = csub(a2, b2);
    } else {
      // any other prime: direct R-point DFT, exp(DIR 2 pi i r s / R) = tw[(r s mod R) N/R] (conj for DIR > 0)
      const int rstep = N / R;
      for (int s = 0; s < R; ++s) {
        C acc = mk<C>((Rl)0, (Rl)0);
        for (int r = 0; r < R; ++r) {
          C v = x[t + r * nb];
          if (r > 0 && k > 0) {
            C w = tw[(k * r * tstep) % N];
            if (DIR > 0) w = cconj(w);
            v = cmul(v, w);
          }
          C e = tw[((r * s) % R) * rstep];
          if (DIR > 0) e = cconj(e);
          acc = cadd(acc, cmul(v, e));
        }
        y[out0 + s * Ns] = acc;
      }
    }
  }
}

// Full transform of z (N complex in shared memory, natural order) using
// scratch t of the same size; returns the buffer holding the result.
template <typename C, int DIR>
__device__ C* gen_fft(C* z, C* t, int N, const GenFactors& g, const C* tw) {
  C* x = z;
  C* y = t;
  int Ns = 1;
  for (int s = 0; s < g.n; ++s) {
    gen_stage<C, DIR>(x, y, N, g.f[s], Ns, tw);
    __syncthreads();
    Ns *= g.f[s];
    C* tmp = x;
    x = y;
    y = tmp;
  }
  return x;
}

// Spectral multiply of a packed pair (a + i b) in Z (natural order): the
// factor of row/column a is ea(kk), of b eb(kk), kk = min(k, N-k), loaded by
// fac(k, ea, eb); result scaled by f into O.
template <typename C, typename Fac>
__device__ void gen_pair_mul(const C* Z, C* O, int N, decltype(C::x) f, Fac fac) {
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    C ea, eb;
    fac(k, ea, eb);
    O[k] = two_real_mul(Z[k], Z[(N - k) % N], herm(ea, k, N), herm(eb, k, N), f);
  }
  __syncthreads();
}

// Forward transform, pair multiply, inverse transform of the pair held in
// buf0 (buf1 scratch); the result ends in buf0.
template <typename C, typename Fac>
__device__ void gen_half_step(C* buf0, C* buf1, int N, const GenFactors& g, const C* tw, decltype(C::x) f, Fac fac) {
  C* spec = gen_fft<C, -1>(buf0, buf1, N, g, tw);
  C* other = spec == buf0 ? buf1 : buf0;
  gen_pair_mul(spec, other, N, f, fac);
  C* res = gen_fft<C, +1>(other, spec, N, g, tw);
  if (res != buf0)
    for (int i = threadIdx.x; i < N; i += blockDim.x) buf0[i] = res[i];
  __syncthreads();
}

// Block-wide FP64 sums of `n` values per thread into out[0..n) (thread 0).
template <int NV>
__device__ void gen_block_sum(double (&v)[NV], double* red) {
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) red[q * 32 + w] = v[q];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int i = 0; i < nw; ++i) s += red[q * 32 + i];
      v[q] = s;
    }
  __syncthreads();
}

template <typename Rl>
__global__ void __launch_bounds__(kGenThreads) gen_row_kernel(PassArgs a, GenFactors g) {
  using C = cplx_t<Rl>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[34];
  const int N = a.X;
  C* z = reinterpret_cast<C*>(smem_raw);
  C* t = z + N;
  const int rp = blockIdx.x, b = blockIdx.y;
  const double sc = prev_scale(a, b, red, rp == 0);
  Rl* W = reinterpret_cast<Rl*>(a.W) + (size_t)b * a.w_bs + (size_t)(2 * rp) * N;
  const Rl s = (Rl)sc;
  for (int x = threadIdx.x; x < N; x += blockDim.x) z[x] = mk<C>(W[x] * s, W[N + x] * s);
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>(a.tw);
  const size_t esz = a.tab_real ? sizeof(Rl) : sizeof(C);
  const size_t hs = N / 2 + 1;
  const char* ta = reinterpret_cast<const char*>(a.tab1) + ((size_t)b * a.tab_bs + (size_t)(2 * rp) * hs) * esz;
  const char* tb = ta + hs * esz;
  gen_half_step(z, t, N, g, tw, (Rl)(a.out_scale / (double)N), [&](int k, C& ea, C& eb) {
    const int kk = k <= N / 2 ? k : N - k;
    ea = tab_load<Rl>(ta, a.tab_real, kk);
    eb = tab_load<Rl>(tb, a.tab_real, kk);
    if (a.g1 != nullptr) {
      const C gk = reinterpret_cast<const C*>(a.g1)[kk];
      ea = cmul(ea, gk);
      eb = cmul(eb, gk);
    }
  });
  for (int x = threadIdx.x; x < N; x += blockDim.x) {
    W[x] = z[x].x;
    W[N + x] = z[x].y;
  }
}

template <typename Rl>
__global__ void __launch_bounds__(kGenThreads) gen_col_kernel(PassArgs a, GenFactors g) {
  using C = cplx_t<Rl>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[12 * 32];  // prev_scale uses the first 34, gen_block_sum all
  const int N = a.P, X = a.X;
  C* z = reinterpret_cast<C*>(smem_raw);
  C* t = z + N;
  const int cp = blockIdx.x, b = blockIdx.y;
  const int xa = 2 * cp;
  const double sc = prev_scale(a, b, red, cp == 0);
  Rl* W = reinterpret_cast<Rl*>(a.W) + (size_t)b * a.w_bs;
  const Rl s = (Rl)sc;
  for (int p = threadIdx.x; p < N; p += blockDim.x) {
    C v = mk<C>(W[(size_t)p * X + xa] * s, W[(size_t)p * X + xa + 1] * s);
    if (a.blend_pre) {
      const Rl* S0 = reinterpret_cast<const Rl*>(a.s0) + (size_t)b * a.s0_bs;
      const Rl bc = (Rl)a.blend_c;
      v = mk<C>(bc * v.x + S0[(size_t)p * X + xa], bc * v.y + S0[(size_t)p * X + xa + 1]);
    }
    z[p] = v;
  }
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>(a.tw);
  const size_t esz = a.tab_real ? sizeof(Rl) : sizeof(C);
  const Rl f = (Rl)(1.0 / (double)N);
  auto half = [&](const void* tab, const void* gv) {
    const char* ta = reinterpret_cast<const char*>(tab) + ((size_t)b * a.tab_bs + xa) * esz;
    gen_half_step(z, t, N, g, tw, f, [&](int k, C& ea, C& eb) {
      const int kk = k <= N / 2 ? k : N - k;
      ea = tab_load<Rl>(ta, a.tab_real, (size_t)kk * X);
      eb = tab_load<Rl>(ta + esz, a.tab_real, (size_t)kk * X);
      if (gv != nullptr) {
        const C gk = reinterpret_cast<const C*>(gv)[kk];
        ea = cmul(ea, gk);
        eb = cmul(eb, gk);
      }
    });
  };
  if (a.tab1 != nullptr) half(a.tab1, a.g1);
  if (a.bxp != nullptr || a.blend_post) {
    const Rl* B = a.bxp ? reinterpret_cast<const Rl*>(a.bxp) + (size_t)b * a.bxp_bs : nullptr;
    const Rl* S0 = a.blend_post ? reinterpret_cast<const Rl*>(a.s0) + (size_t)b * a.s0_bs : nullptr;
    const Rl bc = (Rl)a.blend_c;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
      C v = z[p];
      if (B) v = mk<C>(v.x * B[(size_t)p * X + xa], v.y * B[(size_t)p * X + xa + 1]);
      if (S0) v = mk<C>(bc * v.x + S0[(size_t)p * X + xa], bc * v.y + S0[(size_t)p * X + xa + 1]);
      z[p] = v;
    }
    __syncthreads();
  }
  if (a.part_out != nullptr) {
    // [sum, sum sq, x-weights (Mx), p-weights (Mp)] of the pair, in FP64
    double acc[2 + 2 + 2 * MAXO];  // ca, cb, sum sq, p-obs (MAXO) -- x-obs follow from ca, cb
    for (int q = 0; q < 2 + 2 + 2 * MAXO; ++q) acc[q] = 0.0;
    const double* wp = a.wp + (size_t)b * a.wp_bs;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
      const double wa = (double)z[p].x, wb = (double)z[p].y;
      acc[0] += wa;
      acc[1] += wb;
      acc[2] += wa * wa + wb * wb;
      for (int q = 0; q < a.Mp && q < MAXO; ++q) acc[4 + q] += (wa + wb) * wp[(size_t)q * N + p];
    }
    gen_block_sum(acc, red);
    if (threadIdx.x == 0) {
      const double* wx = a.wx + (size_t)b * a.wx_bs;
      double* rec = a.part_out + ((size_t)b * gridDim.x + cp) * a.M;
      rec[0] = acc[0] + acc[1];
      rec[1] = acc[2];
      for (int q = 0; q < a.Mx; ++q) rec[2 + q] = acc[0] * wx[(size_t)q * X + xa] + acc[1] * wx[(size_t)q * X + xa + 1];
      for (int q = 0; q < a.Mp; ++q) rec[2 + a.Mx + q] = acc[4 + q];
    }
    __syncthreads();
  }
  if (a.tab2 != nullptr) half(a.tab2, a.g2);
  const Rl os = (Rl)a.out_scale;
  for (int p = threadIdx.x; p < N; p += blockDim.x) {
    W[(size_t)p * X + xa] = z[p].x * os;
    W[(size_t)p * X + xa + 1] = z[p].y * os;
  }
}

template <typename Rl>
static cudaError_t gen_launch(const PassArgs& a, bool row, cudaStream_t st, int* nparts) {
  const int N = row ? a.X : a.P;
  const size_t smem = (size_t)2 * N * sizeof(cplx_t<Rl>);
  // the attribute is the largest dynamic shared memory any launch of the
  // kernel may use (N up to 4096), not this launch's
  const size_t smem_max = (size_t)2 * 4096 * sizeof(cplx_t<Rl>);
  const GenFactors g = gen_factors(N);
  if (row) {
    static PerDeviceOnce attr;
    cudaError_t e = set_smem_once(attr, gen_row_kernel<Rl>, smem_max);
    if (e != cudaSuccess) return e;
    gen_row_kernel<Rl><<<dim3(a.P / 2, a.batch), kGenThreads, smem, st>>>(a, g);
  } else {
    static PerDeviceOnce attr;
    cudaError_t e = set_smem_once(attr, gen_col_kernel<Rl>, smem_max);
    if (e != cudaSuccess) return e;
    gen_col_kernel<Rl><<<dim3(a.X / 2, a.batch), kGenThreads, smem, st>>>(a, g);
    if (nparts) *nparts = a.X / 2;
  }
  return cudaGetLastError();
}

cudaError_t launch_generic_row(const PassArgs& a, int dtype, cudaStream_t st) {
  return dtype == FW_F32 ? gen_launch<float>(a, true, st, nullptr) : gen_launch<double>(a, true, st, nullptr);
}

cudaError_t launch_generic_col(const PassArgs& a, int dtype, cudaStream_t st, int* nparts) {
  return dtype == FW_F32 ? gen_launch<float>(a, false, st, nparts) : gen_launch<double>(a, false, st, nparts);
}

}  // namespace fw
