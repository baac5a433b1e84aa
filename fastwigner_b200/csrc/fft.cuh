// Register/shared-memory FFT building blocks for the split-operator passes.
//
// Every hot pass of the propagators is "transform one axis, multiply by a
// phase, transform back".  The transforms here are radix-R Stockham FFTs
// (Govindaraju et al., SC'08 formulation) in which each thread holds RV
// complex values in registers, performs complete radix-R butterflies in
// registers, and exchanges data with the other T-1 threads of its FFT group
// through shared memory between stages.  N = RV * T; the radix list is
// RV, RV, ..., rem (rem < RV) so a 1024-point transform with 32 threads is two
// radix-32 stages and a single shared-memory exchange.
//
// Register order convention ("natural"): thread j of a group holds element
// n = j + m*T in v[m], m = 0..RV-1.  A transform reads natural order and
// leaves natural order, so a forward transform, a point-wise spectral
// multiply and an inverse transform chain with no extra reordering, and the
// first and last stage read/write global memory in coalesced order.
//
// Twiddles between stages come from a table tw[k] = exp(-2*pi*i*k/N)
// (computed in FP64 on the host, rounded once to the working precision).
// The in-register DFT_R uses compile-time constants.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fw {

template <typename R> struct cplx;
template <> struct cplx<float> { using type = float2; };
template <> struct cplx<double> { using type = double2; };
template <typename R> using cplx_t = typename cplx<R>::type;

template <typename C> __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) { C c; c.x = a; c.y = b; return c; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mk<C>(a.x * s, a.y * s); }
// multiply by -i (DIR=-1) or +i (DIR=+1)
template <int DIR, typename C> __device__ __forceinline__ C mul_i(C a) {
  return DIR < 0 ? mk<C>(a.y, -a.x) : mk<C>(-a.y, a.x);
}

// cos(2*pi*k/64), k = 0..16; the remaining 64th roots follow by symmetry.
__host__ __device__ constexpr double cos64_q(int k) {
  return k == 0 ? 1.0 : k == 1 ? 0.9951847266721969 : k == 2 ? 0.9807852804032304
       : k == 3 ? 0.9569403357322088 : k == 4 ? 0.9238795325112867 : k == 5 ? 0.881921264348355
       : k == 6 ? 0.8314696123025452 : k == 7 ? 0.773010453362737 : k == 8 ? 0.7071067811865476
       : k == 9 ? 0.6343932841636455 : k == 10 ? 0.5555702330196023 : k == 11 ? 0.4713967368259978
       : k == 12 ? 0.38268343236508984 : k == 13 ? 0.29028467725446233 : k == 14 ? 0.19509032201612833
       : k == 15 ? 0.09801714032956077 : 0.0;
}
// cos(2*pi*m/64) for any integer m
__host__ __device__ constexpr double cos64(int m) {
  return (m = ((m % 64) + 64) % 64, m <= 16) ? cos64_q(m)
       : m <= 32 ? -cos64_q(32 - m)
       : m <= 48 ? -cos64_q(m - 32)
       : cos64_q(64 - m);
}
__host__ __device__ constexpr double sin64(int m) { return cos64(16 - m); }

// In-register DFT of length R (R | 64), natural order in and out.
// DIR = -1: forward exp(-2 pi i n k / R); DIR = +1: inverse (unnormalised).
template <int R, int DIR, typename C> struct DFT {
  static __device__ __forceinline__ void run(C* v) {
    constexpr int H = R / 2;
    C e[H], o[H];
#pragma unroll
    for (int i = 0; i < H; ++i) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
    DFT<H, DIR, C>::run(e);
    DFT<H, DIR, C>::run(o);
#pragma unroll
    for (int k = 0; k < H; ++k) {
      C t;
      if (k == 0) {
        t = o[k];
      } else if (4 * k == R) {
        t = mul_i<DIR>(o[k]);
      } else {
        using Rl = decltype(C::x);
        constexpr int S = 64 / R;
        const Rl c = (Rl)cos64(k * S);
        const Rl s = (Rl)(DIR * sin64(k * S));
        t = cmul(o[k], mk<C>(c, s));
      }
      v[k] = cadd(e[k], t);
      v[k + H] = csub(e[k], t);
    }
  }
};
template <int DIR, typename C> struct DFT<1, DIR, C> {
  static __device__ __forceinline__ void run(C*) {}
};

constexpr int ilog2_c(int n) { return n <= 1 ? 0 : 1 + ilog2_c(n / 2); }

// Stage-layout twiddle table of an N-point transform with RV values per
// thread: for every stage with stride NS > 1 (radix R = min(RV, N/NS)) the
// entries w^(bm r N/(NS R)), r = 1..R-1, bm = 0..NS-1, stored [r-1][bm] so a
// warp's consecutive bm read consecutive entries.  stage_off(NS) is the
// offset of that stage; stage_off(N) the table length.
__host__ __device__ constexpr int stage_off(int N, int RV, int NS) {
  int off = 0;
  for (int ns = RV; ns < NS; ns *= RV) off += ((N / ns >= RV ? RV : N / ns) - 1) * ns;
  return off;
}

// Stockham radix-R stage chain.  EX is the exchange object (shared memory
// layout + synchronisation scope of the group).  tw: table of exp(-2 pi i k/N),
// k < N, readable by every thread (shared or global memory).
template <int N, int T, int RV, int NS, int DIR, typename C, typename EX, bool STW = false>
__device__ __forceinline__ void stockham(C (&v)[RV], const int j, EX& ex, const C* __restrict__ tw) {
  static_assert(N == RV * T, "N must equal RV*T");
  constexpr int REM = N / NS;
  constexpr int R = (REM >= RV) ? RV : REM;
  constexpr int Q = RV / R;
  constexpr bool FIRST = (NS == 1);
  constexpr bool LAST = (NS * R == N);
  // Address folding: with a layout padded once per 2^L elements (L = log2 RV)
  // and T >= RV, every in-stage offset (q*T + r*N/R on reads, r*NS on writes)
  // is a multiple of 2^L, or a write offset r < RV from an RV-aligned base, so
  // map(base + d) = map(base) + delta(d) and the per-access address is one
  // per-thread register plus an immediate.
  constexpr bool FOLD = EX::kFold && EX::kL == ilog2_c(RV) && T >= RV;
  static_assert(R >= 2 && (RV % R) == 0, "bad radix plan");
  C u[RV];
  if constexpr (FIRST) {
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r) u[q * R + r] = v[q + r * Q];
  } else {
    const int aj = ex.map(j);  // per-thread part of every read address of this stage
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int d = q * T + r * (N / R);
        u[q * R + r] = ex.read_at(FOLD ? aj + ex.delta(d) : ex.map(j + d));
      }
    ex.sync();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int bm = (j + q * T) & (NS - 1);
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = STW ? tw[stage_off(N, RV, NS) + (r - 1) * NS + bm] : tw[bm * r * (N / (NS * R))];
        if (DIR > 0) w = cconj(w);
        u[q * R + r] = cmul(u[q * R + r], w);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) DFT<R, DIR, C>::run(&u[q * R]);
  if constexpr (LAST) {
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r) v[q + r * Q] = u[q * R + r];
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int b = j + q * T;
      const int base = (b / NS) * NS * R + (b & (NS - 1));
      const int ab = ex.map(base);
#pragma unroll
      for (int r = 0; r < R; ++r) ex.write_at(FOLD ? ab + ex.delta(r * NS) : ex.map(base + r * NS), u[q * R + r]);
    }
    ex.sync();
    stockham<N, T, RV, NS * R, DIR, C, EX, STW>(v, j, ex, tw);
  }
}

// tw: the table exp(-2 pi i k/N), k < N (STW = false) or the stage-layout
// table of (N, RV) (STW = true).
template <int N, int T, int RV, int DIR, typename C, typename EX, bool STW = false>
__device__ __forceinline__ void fft(C (&v)[RV], const int j, EX& ex, const C* __restrict__ tw) {
  stockham<N, T, RV, 1, DIR, C, EX, STW>(v, j, ex, tw);
}

// Write v[m] (natural order: element j + m*T) into the exchange buffer,
// folding the addresses when the layout allows it (see stockham).
template <int T, int RV, typename EX, typename C>
__device__ __forceinline__ void ex_write_natural(const EX& ex, const int j, const C (&v)[RV]) {
  constexpr bool FOLD = EX::kFold && EX::kL == ilog2_c(RV) && T >= RV;
  const int aj = ex.map(j);
#pragma unroll
  for (int m = 0; m < RV; ++m) ex.write_at(FOLD ? aj + ex.delta(m * T) : ex.map(j + m * T), v[m]);
}

// Named barrier over `nthreads` threads (multiple of 32) with id 1..15.
__device__ __forceinline__ void named_barrier(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Exchange for a group of T threads that owns a private SoA buffer of
// N + N/32 reals per component (one pad slot per 32 breaks the power-of-two
// bank strides of the Stockham write pattern).
template <typename Rl, int T> struct GroupEx {
  Rl* re;
  Rl* im;
  int bar_id;  // used only when T > 32
  using C = cplx_t<Rl>;
  static constexpr int kL = 5;
  static constexpr bool kFold = true;
  __device__ __forceinline__ static int pad(int i) { return i + (i >> 5); }
  __device__ __forceinline__ static int map(int i) { return pad(i); }
  __device__ __forceinline__ static constexpr int delta(int d) { return d + (d >> 5); }
  __device__ __forceinline__ C read_at(int a) const { return mk<C>(re[a], im[a]); }
  __device__ __forceinline__ void write_at(int a, C v) const { re[a] = v.x; im[a] = v.y; }
  __device__ __forceinline__ C read(int i) const { return read_at(pad(i)); }
  __device__ __forceinline__ void write(int i, C v) const { write_at(pad(i), v); }
  __device__ __forceinline__ void sync() const {
    if constexpr (T <= 32) __syncwarp();
    else named_barrier(bar_id, T);
  }
};

// Exchange for the column passes: CP independent FFTs (one per column pair)
// interleaved element-wise in one CTA-wide SoA buffer: element i of FFT c at
// row-slot (i ^ ((i >> S) & 1)) * CP + c.  The xor of bit 0 with bit S puts the
// two FFT indices that share a warp in different bank halves for both the
// Stockham write and read patterns.  Synchronisation is CTA-wide.
template <typename Rl, int CP, int S> struct ColEx {
  Rl* re;
  Rl* im;
  int c;
  using C = cplx_t<Rl>;
  static constexpr int kL = 0;
  static constexpr bool kFold = false;
  __device__ __forceinline__ int map(int i) const { return (i ^ ((i >> S) & 1)) * CP + c; }
  __device__ __forceinline__ static constexpr int delta(int) { return 0; }
  __device__ __forceinline__ C read_at(int a) const { return mk<C>(re[a], im[a]); }
  __device__ __forceinline__ void write_at(int a, C v) const { re[a] = v.x; im[a] = v.y; }
  __device__ __forceinline__ C read(int i) const { return read_at(map(i)); }
  __device__ __forceinline__ void write(int i, C v) const { write_at(map(i), v); }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// Exchange for the column passes with a padded instead of a swizzled layout:
// element i of FFT c at slot (i + (i >> L)) * CP + c, one pad slot per 2^L
// elements (L = log2 RV).  With 32/CP consecutive transform threads per warp
// the Stockham reads and writes, and the natural-order mid-point accesses,
// fall in distinct banks, and every in-stage address folds into a
// per-thread base plus an immediate.  Each component array holds
// (N + N/2^L) * CP reals.  Synchronisation is CTA-wide.
template <typename Rl, int CP, int L> struct ColPadEx {
  Rl* re;
  Rl* im;
  int c;
  using C = cplx_t<Rl>;
  static constexpr int kL = L;
  static constexpr bool kFold = true;
  __device__ __forceinline__ int map(int i) const { return (i + (i >> L)) * CP + c; }
  __device__ __forceinline__ static constexpr int delta(int d) { return (d + (d >> L)) * CP; }
  __device__ __forceinline__ C read_at(int a) const { return mk<C>(re[a], im[a]); }
  __device__ __forceinline__ void write_at(int a, C v) const { re[a] = v.x; im[a] = v.y; }
  __device__ __forceinline__ C read(int i) const { return read_at(map(i)); }
  __device__ __forceinline__ void write(int i, C v) const { write_at(map(i), v); }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// Exchange for the column passes with complex slots (one 8- or 16-byte access
// per element instead of one per component): element i of FFT c at slot
// (i + (i >> L)) * CP + c of one interleaved complex array, one pad slot per
// 2^L elements (L = log2 RV), which keeps the Stockham and mid-point accesses
// of 32/CP consecutive transform threads in distinct bank pairs and lets every
// in-stage address fold into a per-thread base plus an immediate.  The array
// holds (N + N/2^L) * CP complex values.  Synchronisation is CTA-wide.
template <typename Rl, int CP, int L> struct ColPadExC {
  cplx_t<Rl>* z;
  int c;
  using C = cplx_t<Rl>;
  static constexpr int kL = L;
  static constexpr bool kFold = true;
  __device__ __forceinline__ int map(int i) const { return (i + (i >> L)) * CP + c; }
  __device__ __forceinline__ static constexpr int delta(int d) { return (d + (d >> L)) * CP; }
  __device__ __forceinline__ C read_at(int a) const { return z[a]; }
  __device__ __forceinline__ void write_at(int a, C v) const { z[a] = v; }
  __device__ __forceinline__ C read(int i) const { return read_at(map(i)); }
  __device__ __forceinline__ void write(int i, C v) const { write_at(map(i), v); }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// Exchange for a group of T threads (one warp, T <= 32) that owns a private
// buffer of N + N/32 complex slots (one pad slot per 32 elements, as GroupEx)
// accessed one complex value at a time.  Warp-synchronous.
template <typename Rl, int T> struct GroupExC {
  cplx_t<Rl>* z;
  using C = cplx_t<Rl>;
  static_assert(T <= 32, "GroupExC is warp-synchronous");
  static constexpr int kL = 5;
  static constexpr bool kFold = true;
  __device__ __forceinline__ static int map(int i) { return i + (i >> 5); }
  __device__ __forceinline__ static constexpr int delta(int d) { return d + (d >> 5); }
  __device__ __forceinline__ C read_at(int a) const { return z[a]; }
  __device__ __forceinline__ void write_at(int a, C v) const { z[a] = v; }
  __device__ __forceinline__ C read(int i) const { return read_at(map(i)); }
  __device__ __forceinline__ void write(int i, C v) const { write_at(map(i), v); }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
};

// Sum NB complex values over the CP adjacent lanes of a row group (CP a power
// of two, NB a multiple of CP) by recursive halving: at every level a lane
// keeps one half of its current values, sends the other half to the partner
// lane and adds what it receives, so the sum over CP lanes of NB values costs
// 2 (NB - NB/CP) shuffles per lane instead of 2 NB log2(CP).  On return lane c
// (= lane % CP) holds in u[0 .. NB/CP) the sums of entries c*NB/CP + i.
template <int CP, int NB, typename C>
__device__ __forceinline__ void halving_sum(C (&u)[NB], const int c) {
  static_assert(NB % CP == 0, "halving_sum: NB must be a multiple of CP");
#pragma unroll
  for (int lv = 0; (CP >> (lv + 1)) >= 1; ++lv) {
    const int off = CP >> (lv + 1);
    const int half = NB >> (lv + 1);
    const bool up = (c & off) != 0;
#pragma unroll
    for (int i = 0; i < half; ++i) {
      C send = up ? u[i] : u[i + half];
      const C keep = up ? u[i + half] : u[i];
      send.x = __shfl_xor_sync(0xffffffffu, send.x, off);
      send.y = __shfl_xor_sync(0xffffffffu, send.y, off);
      u[i] = cadd(keep, send);
    }
  }
}

}  // namespace fw
