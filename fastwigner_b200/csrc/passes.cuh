// Argument blocks and shared device helpers for the fused half-step passes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "fft.cuh"

namespace fw {

// One fused pass over a batch of real Wigner functions W[b][p][x] (P x X,
// x fastest).  Column passes transform along p (the theta <-> p axis, the
// potential half-steps); row passes transform along x (lambda <-> x, the
// kinetic step).  Everything a pass may do, in order:
//
//   load:  W *= scale_in                     (lazy normalisation of the previous step)
//          W  = blend_c*W + s0               (blend_pre: collision blend at step start)
//   tab1:  W  = irfft( rfft(W) * tab1 * g1 ) (the half-step; skipped if tab1 == null)
//   mid:   W *= bxp                          (abs_boundary_x_p, col pass only)
//          W  = blend_c*W + s0               (blend_post)
//          partial sums of W, W^2, W*wx(x), W*wp(p) -> part_out (col pass only)
//   tab2:  W  = irfft( rfft(W) * tab2 * g2 ) (second fused half-step; col pass only)
//   store: W *= out_scale
//
// fuse_mid (col pass with tab1 and tab2, no bxp, no blends): the two half-steps
// share one transform pair, W = irfft( rfft(W) * tab1*g1 * tab2*g2 ), and the
// partial sums come from the mid-point spectrum (Parseval): sum = DC bin,
// sum W^2 = |spectrum|^2 / N, sum W wp = Re(spectrum . conj(wph)) / N with
// wph[k][q] the forward DFT of wp[q] at bin k (wph_bs complex entries between
// instances).
//
// scale_in = scale_const if prev_part == null, else 1/(sum_c prev_part[b][c][0] * dxdp).
// When obs_hist != null, block 0 of every instance also writes the reduced
// previous partials (M doubles) to obs_hist[b*M ...].
struct PassArgs {
  void* W;
  long long w_bs;
  int P, X, batch;
  const void* tab1;
  const void* tab2;
  long long tab_bs;
  int tab_real;
  const void* g1;
  const void* g2;
  const double* prev_part;
  int prev_nparts;
  double dxdp;
  double scale_const;
  double* obs_hist;
  const void* bxp;
  long long bxp_bs;
  const void* s0;
  long long s0_bs;
  double blend_c;
  int blend_pre;
  int blend_post;
  double* part_out;
  int M;
  int Mx;
  int Mp;
  const double* wx;
  long long wx_bs;
  const double* wp;
  long long wp_bs;
  const void* tw;
  double out_scale;
  int* status;  // device status word (error flags); may be null
  int fuse_mid;
  const void* wph;  // complex, same precision as W, [b][k][4] (bin-major, 4 weights per bin)
  long long wph_bs;
  int tab_vec;      // tab1/tab2 start on 16 bytes: a column pair's two entries load as one vector
  // Per-instance totals of the previous pass's partial sums (reduced by
  // totals_kernel, M doubles per instance): the input scale is read from
  // prev_tot[b*M] instead of reducing prev_part in every CTA.
  const double* prev_tot;
  // launch shapes for small batches (RowCfgSmall / ColCfgSmall); decided once
  // per plan, since the row twiddle table and the column record count follow it
  int small_shape;
};

// Reduce previous-pass partial sums (per instance) into the input scale.
// Called by every thread; uses `red` (>= 33 doubles of shared memory).
__device__ __forceinline__ double prev_scale(const PassArgs& a, int b, double* red, bool first_tile) {
  if (a.prev_tot != nullptr) return 1.0 / (__ldcg(a.prev_tot + (size_t)b * a.M) * a.dxdp);
  if (a.prev_part == nullptr) return a.scale_const;
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  const double* pp = a.prev_part + (size_t)b * a.prev_nparts * a.M;
  // deterministic: thread t sums parts t, t+nth, ...; then a fixed tree.
  double s = 0.0;
  for (int c = tid; c < a.prev_nparts; c += nth) s += __ldcg(pp + (size_t)c * a.M);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = s;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < (nth + 31) / 32; ++w) t += red[w];
    red[32] = t;
  }
  __syncthreads();
  const double tot = red[32];
  if (a.obs_hist != nullptr && first_tile) {
    // one warp per column m: lanes sum records lane, lane+32, ...; fixed tree
    double* oh = a.obs_hist + (size_t)b * a.M;
    const int lane = tid & 31;
    for (int m = tid >> 5; m < a.M; m += (nth + 31) >> 5) {
      double acc = 0.0;
      for (int c = lane; c < a.prev_nparts; c += 32) acc += __ldcg(pp + (size_t)c * a.M + m);
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) oh[m] = acc;
    }
  }
  return 1.0 / (tot * a.dxdp);
}

template <typename Rl> struct TabVal;
// Load table entry k (0 <= k <= N/2) of a complex or real phase table.
template <typename Rl>
__device__ __forceinline__ cplx_t<Rl> tab_load(const void* tab, int real, size_t idx) {
  using C = cplx_t<Rl>;
  if (real) return mk<C>(__ldg(reinterpret_cast<const Rl*>(tab) + idx), (Rl)0);
  return __ldg(reinterpret_cast<const C*>(tab) + idx);
}

// Hermitian-extended spectral factor at full-spectrum index k (0..N-1) from
// a half-spectrum factor e(kk), kk = min(k, N-k): e(k) for k < N/2,
// conj(e(N-k)) for k > N/2, Re e(k) at k = 0 and k = N/2 (the imaginary parts
// of the DC and Nyquist bins are dropped by a complex-to-real transform).
template <typename C> __device__ __forceinline__ C herm(C e, int k, int N) {
  const int h = N >> 1;
  if (k == 0 || k == h) { e.y = 0; }
  else if (k > h) { e.y = -e.y; }
  return e;
}

// Two real sequences a, b packed as z = a + i b with spectrum Z.  Given Z_k
// and Z_{N-k}, return the spectrum of a' + i b' where a' = irfft(rfft(a)*ea),
// b' = irfft(rfft(b)*eb) (ea, eb already Hermitian-extended at k), times f.
template <typename C>
__device__ __forceinline__ C two_real_mul(C zk, C znk, C ea, C eb, decltype(C::x) f) {
  const C zc = cconj(znk);
  const C A = cadd(zk, zc);                  // 2 A_k
  const C Bi = csub(zk, zc);                 // 2 i B_k
  // Z' = A ea + i B eb = 0.5*(2A) ea + 0.5*(2iB) eb
  const C t = cadd(cmul(A, ea), cmul(Bi, eb));
  return cscale(t, f * (decltype(C::x))0.5);
}

}  // namespace fw
