// Fused passes for complex density matrices rho[b][i][j] = <x'_i| rho |x_j>
// (N x N, j fastest) -- the von Neumann and Bloch density-matrix propagators
// and the tools around them (tuple observables, the shear-based Wigner
// transform).
//
// A pass handles whole rows (transform along j) or whole columns (transform
// along i) of every instance and applies, in order:
//   F0 -> T1 -> F1 -> [reductions] -> F2 -> T2 -> F3
// where T1/T2 are optional forward/inverse FFTs along the pass axis and each
// F is an optional element-wise factor
//   f(i, j) = s * u[j] * w[i] * tab[i][j] * exp(i c A(j) B(i)) * (-1)^(i*sign)
// (s complex scalar; u, w complex vectors; tab a real table; A, B a grid
// coordinate -- x: dX (k - N/2), p: dP ((k + N/2) % N - N/2)).
#include "fft.cuh"
#include "fw_internal.h"

namespace fw {

struct Factor {
  int on;
  double s_re, s_im;   // complex scalar
  const void* u;       // complex over j (Rl precision), may be null
  const void* w;       // complex over i, may be null
  const void* tab;     // real N x N, may be null
  long long tab_bs;    // table batch stride (elements)
  double shear_c;      // 0: no shear
  int shear_a, shear_b;  // coordinate kinds for j and i: 0 = x, 1 = p
  int sign;            // multiply by (-1)^i
};

struct RhoArgs {
  void* R;             // batch x N x N complex
  long long r_bs;      // complex elements between instances
  int N, batch;
  double dX, dP;
  Factor f0, f1, f2, f3;
  int t1, t2;          // 0 none, -1 forward, +1 inverse (unnormalised)
  // lazy normalisation from the previous pass's partials (complex trace)
  const double* prev_part;
  int prev_nparts;
  int M;               // doubles per partial record
  double* obs_hist;
  // reductions (row passes only): trace, sum |rho|^2, Mx diagonal weights, Mp Toeplitz kernels
  double* part_out;
  int Mx, Mp;
  const double* wx;    // Mx x N real (diagonal weights)
  const double* gp;    // Mp x N complex FP64 (G[(i - j) mod N])
  double* sum_out;     // if non-null: per-CTA complex sum of all elements after F3 (2 doubles)
  const void* tw;
};

template <typename Rl>
__device__ __forceinline__ double coord(int kind, int k, int N, double dX, double dP) {
  return kind == 0 ? dX * (k - 0.5 * N) : dP * (double)(((k + N / 2) & (N - 1)) - N / 2);
}

// factor at element (i, j); row-constant parts may be precomputed by the caller
// SH: the shear phase exp(i c coord_a(j) coord_b(i)) may be on (an FP64 sincos per
// element); passes without shear are compiled without that code.
template <typename Rl, bool SH>
__device__ __forceinline__ cplx_t<Rl> factor_sh(const Factor& f, int i, int j, int N, double dX, double dP,
                                             const Rl* tab) {
  using C = cplx_t<Rl>;
  C r = mk<C>((Rl)f.s_re, (Rl)f.s_im);
  if (f.u) r = cmul(r, __ldg(reinterpret_cast<const C*>(f.u) + j));
  if (f.w) r = cmul(r, __ldg(reinterpret_cast<const C*>(f.w) + i));
  if (tab) r = cscale(r, __ldg(tab + (size_t)i * N + j));
  if (SH && f.shear_c != 0.0) {
    const double ph = f.shear_c * coord<Rl>(f.shear_a, j, N, dX, dP) * coord<Rl>(f.shear_b, i, N, dX, dP);
    double sn, cs;
    sincos(ph, &sn, &cs);
    r = cmul(r, mk<C>((Rl)cs, (Rl)sn));
  }
  if (f.sign && (i & 1)) r = mk<C>(-r.x, -r.y);
  return r;
}

// complex previous-step scale 1 / (trace * dX)
__device__ __forceinline__ void rho_prev_scale(const RhoArgs& a, int b, double* red, double& sre, double& sim) {
  sre = 1.0;
  sim = 0.0;
  if (a.prev_part == nullptr) return;
  const double* pp = a.prev_part + (size_t)b * a.prev_nparts * a.M;
  // lane-strided sums over the records and a fixed shuffle tree (deterministic,
  // no serial chain through one thread); blockDim is a multiple of 32
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (warp == 0) {
    double tr = 0, ti = 0;
    for (int c = lane; c < a.prev_nparts; c += 32) {
      tr += pp[(size_t)c * a.M];
      ti += pp[(size_t)c * a.M + 1];
    }
    for (int o = 16; o > 0; o >>= 1) {
      tr += __shfl_xor_sync(0xffffffffu, tr, o);
      ti += __shfl_xor_sync(0xffffffffu, ti, o);
    }
    if (lane == 0) {
      red[0] = tr;
      red[1] = ti;
    }
  }
  if (a.obs_hist != nullptr && blockIdx.x == 0) {  // one warp per record column
    for (int m = warp; m < a.M; m += nw) {
      double acc = 0.0;
      for (int c = lane; c < a.prev_nparts; c += 32) acc += pp[(size_t)c * a.M + m];
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) a.obs_hist[(size_t)b * a.M + m] = acc;
    }
  }
  __syncthreads();
  const double tr = red[0] * a.dX, ti = red[1] * a.dX;
  const double d = tr * tr + ti * ti;
  sre = tr / d;
  sim = -ti / d;
  __syncthreads();
}

template <typename Rl, int N, int T, int RV, bool SH>
__device__ __forceinline__ void apply_factor_row(cplx_t<Rl> (&v)[RV], const Factor& f, int i, int j0, double dX,
                                                 double dP, int b) {
  if (!f.on) return;
  const Rl* tab = f.tab ? reinterpret_cast<const Rl*>(f.tab) + (size_t)b * f.tab_bs : nullptr;
#pragma unroll
  for (int m = 0; m < RV; ++m) v[m] = cmul(v[m], factor_sh<Rl, SH>(f, i, j0 + m * T, N, dX, dP, tab));
}

template <typename Rl, int N, int T, int RV, bool SH>
__device__ __forceinline__ void apply_factor_col(cplx_t<Rl> (&v)[RV], const Factor& f, int i0, int j, double dX,
                                                 double dP, int b) {
  if (!f.on) return;
  const Rl* tab = f.tab ? reinterpret_cast<const Rl*>(f.tab) + (size_t)b * f.tab_bs : nullptr;
#pragma unroll
  for (int m = 0; m < RV; ++m) v[m] = cmul(v[m], factor_sh<Rl, SH>(f, i0 + m * T, j, N, dX, dP, tab));
}

constexpr int RMAXO = 4;

// y if s else x, field by field (selects in registers; no copy of the kernel
// parameters to local memory).
__device__ __forceinline__ Factor pick_factor(bool s, const Factor& x, const Factor& y) {
  Factor f;
  f.on = s ? y.on : x.on;
  f.s_re = s ? y.s_re : x.s_re;
  f.s_im = s ? y.s_im : x.s_im;
  f.u = s ? y.u : x.u;
  f.w = s ? y.w : x.w;
  f.tab = s ? y.tab : x.tab;
  f.tab_bs = s ? y.tab_bs : x.tab_bs;
  f.shear_c = s ? y.shear_c : x.shear_c;
  f.shear_a = s ? y.shear_a : x.shear_a;
  f.shear_b = s ? y.shear_b : x.shear_b;
  f.sign = s ? y.sign : x.sign;
  return f;
}

// forward (dir < 0) or unnormalised inverse (dir > 0) transform; the inverse is
// conj(FFT(conj(x))) so each call site instantiates one transform.
template <typename Rl, int N, int T, int RV, typename EX>
__device__ __forceinline__ void transform(cplx_t<Rl> (&v)[RV], int dir, int j, EX& ex, const cplx_t<Rl>* tw) {
  if (dir == 0) return;
  if (dir > 0) {
#pragma unroll
    for (int m = 0; m < RV; ++m) v[m].y = -v[m].y;
  }
  fft<N, T, RV, -1>(v, j, ex, tw);
  if (dir > 0) {
#pragma unroll
    for (int m = 0; m < RV; ++m) v[m].y = -v[m].y;
  }
}

// Row pass: G groups of T threads; group g owns row i.
template <typename Rl, int N, int T, int G, int MINB, bool SH>
__global__ void __launch_bounds__(G* T, MINB) rho_row_kernel(RhoArgs a) {
  using C = cplx_t<Rl>;
  constexpr int RV = N / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[4];
  __shared__ double ored[G * T / 32][4 + 2 * (2 * RMAXO)];
  const int b = blockIdx.y;
  double sre, sim;
  rho_prev_scale(a, b, red, sre, sim);
  const int g = threadIdx.x / T;
  const int j = threadIdx.x % T;
  const int i = blockIdx.x * G + g;
  constexpr int BUF = N + N / 32;
  Rl* base = reinterpret_cast<Rl*>(smem_raw) + (size_t)g * 2 * BUF;
  GroupEx<Rl, T> ex{base, base + BUF, 1 + g};
  C* R = reinterpret_cast<C*>(a.R) + (size_t)b * a.r_bs + (size_t)i * N;
  const C* tw = reinterpret_cast<const C*>(a.tw);
  C v[RV];
  const C sc = mk<C>((Rl)sre, (Rl)sim);
#pragma unroll
  for (int m = 0; m < RV; ++m) v[m] = cmul(R[j + m * T], sc);
  // The two factor / transform / factor phases run as one loop body (not
  // unrolled): the second phase executes the instructions the first one just
  // fetched, which halves the straight-line code a one-wave launch streams
  // through the instruction cache.  The observables belong to the first phase.
#pragma unroll 1
  for (int it = 0; it < 2; ++it) {
    const bool second = it != 0;
    apply_factor_row<Rl, N, T, RV, SH>(v, pick_factor(second, a.f0, a.f2), i, j, a.dX, a.dP, b);
    transform<Rl, N, T, RV>(v, second ? a.t2 : a.t1, j, ex, tw);
    apply_factor_row<Rl, N, T, RV, SH>(v, pick_factor(second, a.f1, a.f3), i, j, a.dX, a.dP, b);
    if (!second && a.part_out != nullptr) {
      // [trace re, im, sum|rho|^2, 0, x-obs (re, im) x Mx, p-obs (re, im) x Mp]
      double acc[4 + 2 * (2 * RMAXO)];
#pragma unroll
      for (int q = 0; q < 4 + 4 * RMAXO; ++q) acc[q] = 0.0;
      // per-thread sums over the row's RV elements in the state precision (the
      // diagonal terms, one element per row, in FP64), then FP64 across threads
      Rl s2 = 0;
      Rl pr[RMAXO], pim[RMAXO];
#pragma unroll
      for (int q = 0; q < RMAXO; ++q) pr[q] = pim[q] = 0;
#pragma unroll
      for (int m = 0; m < RV; ++m) {
        const int jj = j + m * T;
        const Rl re = v[m].x, im = v[m].y;
        s2 += re * re + im * im;
        if (jj == i) {
          acc[0] += (double)re;
          acc[1] += (double)im;
#pragma unroll
          for (int q = 0; q < RMAXO; ++q)
            if (q < a.Mx) {
              const double wgt = __ldg(a.wx + (size_t)q * N + i);
              acc[4 + 2 * q] += (double)re * wgt;
              acc[5 + 2 * q] += (double)im * wgt;
            }
        }
#pragma unroll
        for (int q = 0; q < RMAXO; ++q)
          if (q < a.Mp) {
            const double2 gk = __ldg(reinterpret_cast<const double2*>(a.gp) + (size_t)q * N + ((i - jj) & (N - 1)));
            const Rl gx = (Rl)gk.x, gy = (Rl)gk.y;
            pr[q] += re * gx - im * gy;
            pim[q] += re * gy + im * gx;
          }
      }
      acc[2] = (double)s2;
#pragma unroll
      for (int q = 0; q < RMAXO; ++q) {
        acc[4 + 2 * RMAXO + 2 * q] = (double)pr[q];
        acc[5 + 2 * RMAXO + 2 * q] = (double)pim[q];
      }
      // level-major warp reduction of the accumulators in use (acc[3] stays 0)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < 4 + 4 * RMAXO; ++q) {
          const bool used = q < 3 || (q >= 4 && q < 4 + 2 * a.Mx) ||
                            (q >= 4 + 2 * RMAXO && q < 4 + 2 * RMAXO + 2 * a.Mp);
          if (used) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        }
      const int warp = threadIdx.x >> 5;
      if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int q = 0; q < 4 + 4 * RMAXO; ++q) ored[warp][q] = acc[q];
      }
      __syncthreads();
      if ((int)threadIdx.x < a.M) {
        const int mo = threadIdx.x;
        int q;
        if (mo < 4) q = mo;
        else if (mo < 4 + 2 * a.Mx) q = mo;
        else q = 4 + 2 * RMAXO + (mo - 4 - 2 * a.Mx);
        double t = 0.0;
        for (int w = 0; w < G * T / 32; ++w) t += ored[w][q];
        a.part_out[((size_t)b * gridDim.x + blockIdx.x) * a.M + mo] = t;
      }
    }
  }
#pragma unroll
  for (int m = 0; m < RV; ++m) R[j + m * T] = v[m];
  if (a.sum_out != nullptr) {
    double sr = 0, si = 0;
#pragma unroll
    for (int m = 0; m < RV; ++m) { sr += (double)v[m].x; si += (double)v[m].y; }
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { ored[warp][0] = sr; ored[warp][1] = si; }
    __syncthreads();
    if (threadIdx.x < 2) {
      double t = 0;
      for (int w = 0; w < G * T / 32; ++w) t += ored[w][threadIdx.x];
      a.sum_out[((size_t)b * gridDim.x + blockIdx.x) * 2 + threadIdx.x] = t;
    }
  }
}

// Column pass: CP columns per CTA, T threads per column (interleaved exchange).
template <typename Rl, int N, int T, int CP, int S, int MINB, bool SH>
__global__ void __launch_bounds__(CP* T, MINB) rho_col_kernel(RhoArgs a) {
  using C = cplx_t<Rl>;
  constexpr int RV = N / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[4];
  const int b = blockIdx.y;
  double sre, sim;
  rho_prev_scale(a, b, red, sre, sim);
  const int c = threadIdx.x % CP;
  const int jt = threadIdx.x / CP;
  __builtin_assume(jt >= 0 && jt < T);  // launched with exactly CP * T threads
  const int col = blockIdx.x * CP + c;
  Rl* re = reinterpret_cast<Rl*>(smem_raw);
  ColEx<Rl, CP, S> ex{re, re + (size_t)N * CP, c};
  C* R = reinterpret_cast<C*>(a.R) + (size_t)b * a.r_bs;
  const C* tw = reinterpret_cast<const C*>(a.tw);
  C v[RV];
  const C sc = mk<C>((Rl)sre, (Rl)sim);
#pragma unroll
  for (int m = 0; m < RV; ++m) v[m] = cmul(R[(size_t)(jt + m * T) * N + col], sc);
  apply_factor_col<Rl, N, T, RV, SH>(v, a.f0, jt, col, a.dX, a.dP, b);
  transform<Rl, N, T, RV>(v, a.t1, jt, ex, tw);
  apply_factor_col<Rl, N, T, RV, SH>(v, a.f1, jt, col, a.dX, a.dP, b);
  apply_factor_col<Rl, N, T, RV, SH>(v, a.f2, jt, col, a.dX, a.dP, b);
  transform<Rl, N, T, RV>(v, a.t2, jt, ex, tw);
  apply_factor_col<Rl, N, T, RV, SH>(v, a.f3, jt, col, a.dX, a.dP, b);
#pragma unroll
  for (int m = 0; m < RV; ++m) R[(size_t)(jt + m * T) * N + col] = v[m];
}

// ---------------------------------------------------------------------------
template <typename Rl, int N> struct RhoRowCfg;
template <typename Rl, int N> struct RhoColCfg;
#define RCFG(R, N_, T_, G_, MB_) template <> struct RhoRowCfg<R, N_> { static constexpr int T = T_, G = G_, MINB = MB_; };
#define CCFG(R, N_, T_, CP_, MB_) template <> struct RhoColCfg<R, N_> { static constexpr int T = T_, CP = CP_, MINB = MB_; };
RCFG(float, 128, 16, 8, 1) RCFG(float, 256, 32, 4, 2) RCFG(float, 512, 32, 4, 2) RCFG(float, 1024, 32, 4, 2)
RCFG(float, 2048, 64, 4, 1) RCFG(float, 4096, 128, 2, 1)
RCFG(double, 128, 16, 8, 1) RCFG(double, 256, 16, 8, 1) RCFG(double, 512, 32, 4, 1) RCFG(double, 1024, 64, 2, 1)
RCFG(double, 2048, 128, 2, 1) RCFG(double, 4096, 256, 1, 1)
CCFG(float, 128, 16, 16, 1) CCFG(float, 256, 32, 16, 1) CCFG(float, 512, 32, 16, 1) CCFG(float, 1024, 64, 8, 1)
CCFG(float, 2048, 64, 8, 1) CCFG(float, 4096, 128, 4, 1)
CCFG(double, 128, 16, 8, 1) CCFG(double, 256, 16, 8, 1) CCFG(double, 512, 32, 8, 1) CCFG(double, 1024, 64, 4, 1)
CCFG(double, 2048, 128, 2, 1) CCFG(double, 4096, 256, 2, 1)
#undef RCFG
#undef CCFG

static bool any_shear(const RhoArgs& a) {
  return a.f0.shear_c != 0.0 || a.f1.shear_c != 0.0 || a.f2.shear_c != 0.0 || a.f3.shear_c != 0.0;
}

template <typename Rl, int N, bool SH>
static cudaError_t rho_row_sh(const RhoArgs& a, cudaStream_t st, int* nparts) {
  using Cfg = RhoRowCfg<Rl, N>;
  constexpr int T = Cfg::T, G = Cfg::G, MINB = Cfg::MINB;
  const size_t smem = (size_t)G * 2 * (N + N / 32) * sizeof(Rl);
  auto kern = rho_row_kernel<Rl, N, T, G, MINB, SH>;
  static PerDeviceOnce attr;  // per device: the attribute is set on the device current at the call
  cudaError_t e = set_smem_once(attr, kern, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(N / G, a.batch);
  if (nparts) *nparts = grid.x;
  kern<<<grid, G * T, smem, st>>>(a);
  return cudaGetLastError();
}

// Passes whose factors shear (the rho -> W transform) use the instantiation
// with the per-element sincos; propagation passes carry none of that code.
template <typename Rl, int N>
static cudaError_t rho_row_n(const RhoArgs& a, cudaStream_t st, int* nparts) {
  return any_shear(a) ? rho_row_sh<Rl, N, true>(a, st, nparts) : rho_row_sh<Rl, N, false>(a, st, nparts);
}

template <typename Rl, int N, bool SH>
static cudaError_t rho_col_sh(const RhoArgs& a, cudaStream_t st) {
  using Cfg = RhoColCfg<Rl, N>;
  constexpr int T = Cfg::T, CP = Cfg::CP, MINB = Cfg::MINB;
  constexpr int S = ilog2_c(N / T > 32 ? 32 : N / T);
  const size_t smem = (size_t)2 * N * CP * sizeof(Rl);
  auto kern = rho_col_kernel<Rl, N, T, CP, S, MINB, SH>;
  static PerDeviceOnce attr;  // per device: the attribute is set on the device current at the call
  cudaError_t e = set_smem_once(attr, kern, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(N / CP, a.batch);
  kern<<<grid, CP * T, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename Rl, int N>
static cudaError_t rho_col_n(const RhoArgs& a, cudaStream_t st) {
  return any_shear(a) ? rho_col_sh<Rl, N, true>(a, st) : rho_col_sh<Rl, N, false>(a, st);
}

int rho_row_parts(int dtype, int N) {
  int g = 0;
#define RP(R, N_) if (N == N_) g = RhoRowCfg<R, N_>::G;
  if (dtype == FW_F32) { RP(float, 128) RP(float, 256) RP(float, 512) RP(float, 1024) RP(float, 2048) RP(float, 4096) }
  else { RP(double, 128) RP(double, 256) RP(double, 512) RP(double, 1024) RP(double, 2048) RP(double, 4096) }
#undef RP
  return g == 0 ? -1 : N / g;
}

cudaError_t launch_rho_row(const RhoArgs& a, int dtype, cudaStream_t st, int* nparts) {
#define RN(R, N_) case N_: return rho_row_n<R, N_>(a, st, nparts);
  if (dtype == FW_F32) { switch (a.N) { RN(float, 128) RN(float, 256) RN(float, 512) RN(float, 1024) RN(float, 2048) RN(float, 4096) } }
  else { switch (a.N) { RN(double, 128) RN(double, 256) RN(double, 512) RN(double, 1024) RN(double, 2048) RN(double, 4096) } }
#undef RN
  return cudaErrorInvalidValue;
}

cudaError_t launch_rho_col(const RhoArgs& a, int dtype, cudaStream_t st) {
#define CN(R, N_) case N_: return rho_col_n<R, N_>(a, st);
  if (dtype == FW_F32) { switch (a.N) { CN(float, 128) CN(float, 256) CN(float, 512) CN(float, 1024) CN(float, 2048) CN(float, 4096) } }
  else { switch (a.N) { CN(double, 128) CN(double, 256) CN(double, 512) CN(double, 1024) CN(double, 2048) CN(double, 4096) } }
#undef CN
  return cudaErrorInvalidValue;
}

}  // namespace fw
