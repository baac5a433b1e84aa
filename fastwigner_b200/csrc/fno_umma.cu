// Tensor-core GEMM (tcgen05 / TMEM) for the FNO surrogate's dense
// contractions: the truncated DFTs, the pointwise channel maps, the
// projection and the weight gradients.  C[b] = alpha op(A[b]) op(B[b]) +
// beta C[b] in FP32 with the products on the 5th-generation tensor cores in
// TF32, split three ways (a = a_hi + a_lo with a_hi the TF32 part:
// a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi) so the result keeps FP32 accuracy
// (~1e-6 relative) rather than TF32's ~1e-3.
//
// One CTA of four warps computes a 128 x BN tile of D = U V^T in the tensor
// core's orientation: U (128 rows x K) and V (BN rows x K), K-major in shared
// memory in the canonical no-swizzle layout -- 8-row x 16-byte core matrices,
// 128 bytes apart along the rows, the two K halves of one instruction LBO
// bytes apart.  U runs along C's contiguous dimension (N) when N >= M, so the
// epilogue's lanes store consecutive elements; else along M.
//
// Pipeline per 32-wide K chunk: every thread holds its share of the chunk in
// registers (float4 loads where the operand is K-contiguous, four strided
// loads otherwise, zero-filled at the edges), waits for the previous chunk's
// MMAs, splits and stores it to shared memory (each group of eight lanes
// writes one 128-byte run: no bank conflicts), and thread 0 issues the twelve
// MMAs (4 x K = 8, three products each) and commits them to an mbarrier;
// meanwhile the threads load the next chunk.  The accumulator lives in TMEM
// (128 lanes x BN columns); the four warps read their 32 lanes back with
// tcgen05.ld.  A CTA walks several row tiles (grid-stride), the next tile's
// first chunk loading while the current tile's epilogue runs.  The tensor
// core's FP32 accumulation truncates, so its error
// grows linearly with the number of accumulating MMAs (3.2e-5 of max |C| at
// K = 4096, random operands); tiles up to 32 columns wide therefore give each
// chunk a fresh accumulator (two TMEM halves in turn: one is read while the
// next chunk's MMAs fill the other) and sum the chunks in registers with
// round-to-nearest adds.  Wider tiles (the surrogate uses them only with
// K <= 32, one chunk) accumulate in TMEM.  A CTA may contract only a slice of
// K (split-K for the weight gradients, whose K is the whole grid); the slices
// are summed afterwards in FP64.
//
// Epilogue options: + bias (per row m of C), store of the pre-activation,
// GELU, multiplication by GELU'(aux) (the backward of a GELU), and a
// projection mode that reduces each D row against a weight vector
// (out = c + sum_j w_j GELU(t_j)), so the FNO's 128-wide hidden layer never
// leaves the chip.
//
// Every mbarrier wait is bounded: on expiry the CTA records FW_FNO_TIMEOUT in
// the FNO status word, writes NaN into the tile it was computing (its later
// tiles are left unwritten), waits once more (bounded) for its MMAs, frees its
// TMEM and returns.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include "fno_act.cuh"
#include "fw_internal.h"
#include "tma.cuh"

namespace fw {

__device__ int g_fno_status;  // FW_FNO_TIMEOUT when a tensor-core GEMM gave up waiting

// arguments of one tensor-core GEMM launch
struct UmmaArgs {
  int urows, vrows, K;  // D = U V^T is urows x vrows; contraction length K
  int ksplit, kchunk;   // CTA z = b ksplit + s contracts k in [s kchunk, min(K, (s + 1) kchunk))
  float alpha, beta;
  const float* U;  // U(r, k) = U[b usb + r usr + k usk]
  long long usr, usk, usb;
  const float* V;  // V(c, k) = V[b vsb + c vsr + k vsk]
  long long vsr, vsk, vsb;
  const float* Cin;  // D(r, c) of output batch z: z dsb + r dsr + c dsc (Cin, Cout, pre, aux alike)
  float* Cout;
  float* pre;
  const float* aux;
  long long dsr, dsc, dsb;
  const float* bias;  // indexed by D's row (bias_r) or column
  int bias_r;
  int act;            // EPI_*
  const float* dotw;  // projection mode: Cout[z dsb + r dsr] = dotb[0] + sum_c dotw[c] GELU(t(r, c))
  const float* dotb;
  int uvec, vvec;  // K-contiguous operand with 16-byte aligned rows: float4 loads
};

namespace umma {  // named (external linkage): host helpers take lambdas over these types

constexpr int UM = 128;  // tile rows (tensor-core M)
constexpr int UK = 32;   // K per shared-memory chunk (four MMAs of K = 8)
constexpr long long kUmmaMaxPolls = 1LL << 20;

enum { EPI_NONE = 0, EPI_GELU = 1, EPI_DGELU = 2 };


// canonical K-major no-swizzle offset (floats) of the 4-float row (r, k-group
// g) of a tile with `rows` rows: core matrix (r/8, g) of 8 x 4 floats
__device__ __forceinline__ int canon4(int r, int g, int rows) { return g * (rows * 4) + (r >> 3) * 32 + (r & 7) * 4; }

// shared-memory matrix descriptor: start address, LBO (the two K halves of
// one MMA), SBO = 128 bytes (neighbouring 8-row core matrices), sm100 version
// bits, no swizzle
__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t lbo_bytes) {
  const uint64_t a = (smem_u32(p) >> 4) & 0x3FFFu;
  const uint64_t l = (lbo_bytes >> 4) & 0x3FFFu;
  const uint64_t s = (128u >> 4) & 0x3FFFu;
  return a | (l << 16) | (s << 32) | (1ull << 46);
}

// instruction descriptor of kind::tf32: F32 accumulator, TF32 A and B, both
// K-major, N = bn, M = 128
__host__ __device__ constexpr uint32_t instr_desc(int bn) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(UM >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&r)[16]) {
  uint32_t u[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]), "=r"(u[8]),
        "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) r[i] = __uint_as_float(u[i]);
}

// TF32 part of x (the 19 leading bits; the tensor core reads no more) and the rest
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
  hi = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
  lo = x - hi;
}

// The (row, k-group) that thread (warp, lane) holds as its i-th float4 of a
// ROWS x UK chunk.  K-contiguous source: a warp covers 8 rows x 4 k-groups
// (eight rows of 64 bytes per load); row-contiguous source: R rows x 32/R
// k-groups (R consecutive elements per k).  Either way each group of eight
// lanes stores 8 consecutive rows of one k-group: one 128-byte run.
template <int ROWS>
__device__ __forceinline__ void item_rg(bool kfast, int warp, int i, int lane, int& r, int& g) {
  constexpr int NI = ROWS / 16;
  const int bi = warp * NI + i;
  if (kfast) {
    r = (bi >> 1) * 8 + (lane & 7);
    g = (bi & 1) * 4 + (lane >> 3);
  } else {
    constexpr int R = ROWS < 32 ? ROWS : 32;
    constexpr int RB = ROWS / R;
    constexpr int GPI = 32 / R;
    r = (bi % RB) * R + (lane % R);
    g = (bi / RB) * GPI + lane / R;
  }
}

// ragged edges (rows past the end, a partial K chunk, unaligned rows): element by element, zero-filled
template <int ROWS>
__device__ __noinline__ void load_chunk_edge(float4 (&v)[ROWS / 16], const float* base, long long sr, long long sk,
                                             int nrows, int k0, int kend, bool kfast, int warp, int lane) {
#pragma unroll
  for (int i = 0; i < ROWS / 16; ++i) {
    int r, g;
    item_rg<ROWS>(kfast, warp, i, lane, r, g);
    const int k = k0 + 4 * g;
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    if (r < nrows) {
      const float* p = base + (long long)r * sr + (long long)k * sk;
      if (k < kend) t.x = __ldg(p);
      if (k + 1 < kend) t.y = __ldg(p + sk);
      if (k + 2 < kend) t.z = __ldg(p + 2 * sk);
      if (k + 3 < kend) t.w = __ldg(p + 3 * sk);
    }
    v[i] = t;
  }
}

template <int ROWS>
__device__ __forceinline__ void load_chunk(float4 (&v)[ROWS / 16], const float* base, long long sr, long long sk,
                                           int nrows, int k0, int kend, bool kfast, bool vec, int warp, int lane) {
  const bool kfull = k0 + UK <= kend;
  if (kfull && kfast && vec) {
#pragma unroll
    for (int i = 0; i < ROWS / 16; ++i) {
      int r, g;
      item_rg<ROWS>(true, warp, i, lane, r, g);
      v[i] = r < nrows ? __ldg(reinterpret_cast<const float4*>(base + (long long)r * sr + k0 + 4 * g))
                       : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  } else if (kfull && !kfast) {
#pragma unroll
    for (int i = 0; i < ROWS / 16; ++i) {
      int r, g;
      item_rg<ROWS>(false, warp, i, lane, r, g);
      const float* p = base + (long long)r * sr + (long long)(k0 + 4 * g) * sk;
      v[i] = r < nrows ? make_float4(__ldg(p), __ldg(p + sk), __ldg(p + 2 * sk), __ldg(p + 3 * sk))
                       : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  } else {
    load_chunk_edge<ROWS>(v, base, sr, sk, nrows, k0, kend, kfast, warp, lane);
  }
}

template <int ROWS>
__device__ __forceinline__ void store_chunk(const float4 (&v)[ROWS / 16], float* hi, float* lo, bool kfast, int warp,
                                            int lane) {
#pragma unroll
  for (int i = 0; i < ROWS / 16; ++i) {
    int r, g;
    item_rg<ROWS>(kfast, warp, i, lane, r, g);
    const int o = canon4(r, g, ROWS);
    float4 h, l;
    split_tf32(v[i].x, h.x, l.x);
    split_tf32(v[i].y, h.y, l.y);
    split_tf32(v[i].z, h.z, l.z);
    split_tf32(v[i].w, h.w, l.w);
    *reinterpret_cast<float4*>(hi + o) = h;
    *reinterpret_cast<float4*>(lo + o) = l;
  }
}

// out of line: an inlined erff per column of a 128-wide epilogue overflows the instruction cache
__device__ __noinline__ float gelu_call(float x) { return gelu(x); }
__device__ __noinline__ float gelu_d_call(float x) { return gelu_d(x); }

template <int BN>
__global__ void __launch_bounds__(128, 3) umma_gemm_kernel(UmmaArgs g) {
  // FLUSH: each K chunk accumulates into a fresh TMEM half (alternating), and
  // the chunks are summed in registers with round-to-nearest FP32 adds
  constexpr bool FLUSH = BN <= 32;
  constexpr int TC1 = BN < 32 ? 32 : BN;        // TMEM columns of one accumulator
  constexpr int TCOLS = FLUSH ? 2 * TC1 : TC1;  // allocated (a power of two >= 32)
  extern __shared__ __align__(128) unsigned char sm_dyn[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  unsigned char* sm = sm_dyn + ((128u - (smem_u32(sm_dyn) & 127u)) & 127u);
  float* Uh = reinterpret_cast<float*>(sm);
  float* Ul = Uh + UM * UK;
  float* Vh = Ul + UM * UK;
  float* Vl = Vh + BN * UK;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int z = blockIdx.z, b = z / g.ksplit, s = z - b * g.ksplit;
  const int col0 = blockIdx.x * BN;
  const int nyt = (g.urows + UM - 1) / UM;  // row tiles; this CTA takes blockIdx.y, + gridDim.y, ...
  const int kbeg = s * g.kchunk;
  const int kend = min(g.K, kbeg + g.kchunk);
  const float* Ubase = g.U + (long long)b * g.usb;
  const float* Vb = g.V + (long long)b * g.vsb + (long long)col0 * g.vsr;
  const int vn = g.vrows - col0;
  const bool ukf = g.usk == 1, vkf = g.vsk == 1;
  const bool uvec = g.uvec != 0, vvec = g.vvec != 0;
  const long long zo = (long long)z * g.dsb;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"((uint32_t)TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_fence_init();
    abort_flag = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = instr_desc(BN);
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
  uint32_t phase = 0;
  bool pending = false;  // MMAs committed and not yet seen complete by this thread
  float accr[FLUSH ? BN : 1];
  // adds the accumulator half of chunk c into the registers
  auto flush = [&](int c) {
#pragma unroll
    for (int cb = 0; cb < BN / 16; ++cb) {
      float t[16];
      tmem_ld16(trow + (uint32_t)((c & 1) * TC1 + cb * 16), t);
#pragma unroll
      for (int i = 0; i < 16; ++i) accr[cb * 16 + i] += t[i];
    }
  };

  const int nch = (kend - kbeg + UK - 1) / UK;  // >= 1 by construction of the split
  int yt = blockIdx.y;                          // < nyt by construction of the grid
  int row0 = yt * UM;
  float4 ru[UM / 16], rv[BN / 16];
  load_chunk<UM>(ru, Ubase + (long long)row0 * g.usr, g.usr, g.usk, g.urows - row0, kbeg, kend, ukf, uvec, warp,
                 lane);
  load_chunk<BN>(rv, Vb, g.vsr, g.vsk, vn, kbeg, kend, vkf, vvec, warp, lane);
  for (;;) {  // row tiles
    const int nyt_next = yt + (int)gridDim.y;
    const bool more = nyt_next < nyt;
#pragma unroll
    for (int i = 0; i < (FLUSH ? BN : 1); ++i) accr[i] = 0.f;
    for (int c = 0; c < nch; ++c) {
      // the previous chunk's MMAs must be done before its tiles are overwritten
      if (pending) {
        if (mbar_wait_bounded(&mbar, phase, kUmmaMaxPolls)) {
          phase ^= 1u;
          pending = false;
        } else {
          abort_flag = 1;
        }
      }
      store_chunk<UM>(ru, Uh, Ul, ukf, warp, lane);
      store_chunk<BN>(rv, Vh, Vl, vkf, warp, lane);
      proxy_fence_smem();  // the generic stores become visible to the tensor core
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (abort_flag) break;
      if (tid == 0) {
        const uint32_t td = FLUSH ? tmem + (uint32_t)((c & 1) * TC1) : tmem;
#pragma unroll
        for (int q = 0; q < UK / 8; ++q) {
          const uint64_t dUh = smem_desc(Uh + q * 2 * UM * 4, UM * 16), dUl = smem_desc(Ul + q * 2 * UM * 4, UM * 16);
          const uint64_t dVh = smem_desc(Vh + q * 2 * BN * 4, BN * 16), dVl = smem_desc(Vl + q * 2 * BN * 4, BN * 16);
          umma_tf32(td, dUh, dVh, idesc, ((FLUSH ? 0 : c) > 0 || q > 0) ? 1u : 0u);
          umma_tf32(td, dUh, dVl, idesc, 1u);
          umma_tf32(td, dUl, dVh, idesc, 1u);
        }
        umma_commit(&mbar);
      }
      pending = true;
      // the previous chunk's half (complete: waited for above) while these MMAs run
      if (FLUSH && c > 0) flush(c - 1);
      // the next chunk, of this tile or the next one, in flight during the MMAs
      // (and during this tile's epilogue)
      if (c + 1 < nch) {
        const int k0 = kbeg + (c + 1) * UK;
        load_chunk<UM>(ru, Ubase + (long long)row0 * g.usr, g.usr, g.usk, g.urows - row0, k0, kend, ukf, uvec, warp,
                       lane);
        load_chunk<BN>(rv, Vb, g.vsr, g.vsk, vn, k0, kend, vkf, vvec, warp, lane);
      } else if (more) {
        const int nrow0 = nyt_next * UM;
        load_chunk<UM>(ru, Ubase + (long long)nrow0 * g.usr, g.usr, g.usk, g.urows - nrow0, kbeg, kend, ukf, uvec,
                       warp, lane);
        if (nch > 1) load_chunk<BN>(rv, Vb, g.vsr, g.vsk, vn, kbeg, kend, vkf, vvec, warp, lane);
      }
    }
    if (pending && !abort_flag) {
      if (mbar_wait_bounded(&mbar, phase, kUmmaMaxPolls)) {
        phase ^= 1u;
        pending = false;
      } else {
        abort_flag = 1;
      }
    }
    __syncthreads();
    tc_fence_after();
    if (abort_flag) break;
    if (FLUSH) flush(nch - 1);

    // ---- epilogue: warp w holds D rows 32w .. 32w+31 (its TMEM lanes).
    // FLUSH tiles read their accumulator from registers (cb unrolled, at most
    // two blocks); wider ones from TMEM, one 16-column block per iteration.
    const int gr = row0 + warp * 32 + lane;
    const bool rok = gr < g.urows;
    const long long rbase = zo + (long long)gr * g.dsr;
    if (g.dotw != nullptr) {
      float sum = 0.f;
#pragma unroll(FLUSH ? BN / 16 : 1)
      for (int cb = 0; cb < BN / 16; ++cb) {
        float acc[16];
        if (FLUSH) {
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = accr[FLUSH ? cb * 16 + i : 0];
        } else {
          tmem_ld16(trow + (uint32_t)(cb * 16), acc);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int cc = col0 + cb * 16 + i;
          if (cc < g.vrows) sum += __ldg(g.dotw + cc) * gelu_call(g.alpha * acc[i] + __ldg(g.bias + cc));
        }
      }
      if (rok) g.Cout[rbase] = sum + __ldg(g.dotb);
    } else {
      const bool plain = g.beta == 0.f && g.bias == nullptr && g.pre == nullptr && g.act == EPI_NONE;
#pragma unroll(FLUSH ? BN / 16 : 1)
      for (int cb = 0; cb < BN / 16; ++cb) {
        float acc[16];
        if (FLUSH) {
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = accr[FLUSH ? cb * 16 + i : 0];
        } else {
          tmem_ld16(trow + (uint32_t)(cb * 16), acc);
        }
        const int c0 = col0 + cb * 16;
        if (plain) {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (rok && c0 + i < g.vrows) g.Cout[rbase + (long long)(c0 + i) * g.dsc] = g.alpha * acc[i];
          continue;
        }
        // each group of 8 elements' operands is read before any is written (C
        // may be the output itself: each element is read and written by this thread)
#pragma unroll
        for (int h = 0; h < 16; h += 8) {
          float cin[8], ax[8], bi[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int cc = c0 + h + i;
            const bool ok = rok && cc < g.vrows;
            const long long off = rbase + (long long)cc * g.dsc;
            cin[i] = (ok && g.beta != 0.f) ? g.Cin[off] : 0.f;
            ax[i] = (ok && g.act == EPI_DGELU) ? g.aux[off] : 0.f;
            bi[i] = (ok && g.bias != nullptr) ? __ldg(g.bias + (g.bias_r ? gr : cc)) : 0.f;
          }
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int cc = c0 + h + i;
            if (rok && cc < g.vrows) {
              const long long off = rbase + (long long)cc * g.dsc;
              float t = g.alpha * acc[h + i] + g.beta * cin[i] + bi[i];
              if (g.pre != nullptr) g.pre[off] = t;
              if (g.act == EPI_GELU) t = gelu_call(t);
              else if (g.act == EPI_DGELU) t *= gelu_d_call(ax[i]);
              g.Cout[off] = t;
            }
          }
        }
      }
    }
    if (!more) break;
    yt = nyt_next;
    row0 = yt * UM;
    // this tile's TMEM reads complete before the next tile's first MMA: the
    // fence + barrier after the next chunk's shared-memory stores order them
  }

  if (abort_flag) {
    if (tid == 0) {
      atomicCAS(&g_fno_status, 0, FW_FNO_TIMEOUT);
      if (pending) mbar_wait_bounded(&mbar, phase, kUmmaMaxPolls);
    }
    const float nan = __int_as_float(0x7fc00000);
    const int gr = row0 + warp * 32 + lane;
    if (gr < g.urows) {
      if (g.dotw != nullptr) {
        g.Cout[zo + (long long)gr * g.dsr] = nan;
      } else {
        for (int i = 0; i < BN && col0 + i < g.vrows; ++i)
          g.Cout[zo + (long long)gr * g.dsr + (long long)(col0 + i) * g.dsc] = nan;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TCOLS) : "memory");
}

int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return 148;
  }
  return n;
}

template <int BN>
cudaError_t launch_bn(const UmmaArgs& g, int zdim, cudaStream_t st) {
  const size_t smem = (size_t)2 * (UM + BN) * UK * 4 + 128;
  auto kern = umma_gemm_kernel<BN>;
  static PerDeviceOnce attr;
  // the whole carveout as shared memory, so several CTAs fit on an SM
  cudaError_t e = attr.run([&] {
    cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r == cudaSuccess)
      r = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    return r;
  });
  if (e != cudaSuccess) return e;
  // row tiles beyond about eight CTAs per SM are looped over inside the CTAs
  const int gx = (g.vrows + BN - 1) / BN, nyt = (g.urows + UM - 1) / UM;
  const long long cap = (8LL * sm_count() + (long long)gx * zdim - 1) / ((long long)gx * zdim);
  const int gy = (int)(nyt < cap ? nyt : (cap < 1 ? 1 : cap));
  dim3 grid(gx, gy > 65535 ? 65535 : gy, zdim);
  kern<<<grid, 128, smem, st>>>(g);
  return cudaGetLastError();
}

int tile_bn(int vrows) { return vrows <= 16 ? 16 : vrows <= 32 ? 32 : vrows <= 64 ? 64 : 128; }

// sums Z partial tiles of E elements (FP64): out[e] (+)= sum_z work[z E + e]
__global__ void split_sum_kernel(int Z, int E, const float* __restrict__ work, float* out, int accumulate) {
  const int e = blockIdx.x * 32 + threadIdx.x;
  double s = 0.0;
  if (e < E)
    for (int zz = threadIdx.y; zz < Z; zz += 8) s += (double)work[(long long)zz * E + e];
  __shared__ double red[8][33];
  red[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && e < E) {
    double t = 0.0;
#pragma unroll
    for (int y = 0; y < 8; ++y) t += red[y][threadIdx.x];
    out[e] = (float)(t + (accumulate ? (double)out[e] : 0.0));
  }
}

struct Epi {
  const float* bias = nullptr;
  float* pre = nullptr;
  const float* aux = nullptr;
  int act = EPI_NONE;
  float* out = nullptr;
  const float* dotw = nullptr;
  const float* dotb = nullptr;
};

bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// C (M x N per batch) = alpha op(A) op(B) + beta C, with the epilogue `ep`;
// with ksplit > 1 the output batch z = b ksplit + s holds the partial product
// of K slice s.
cudaError_t gemm(int ta, int tb, int M, int N, int K, float alpha, const float* A, long long lda, long long sA,
                 const float* B, long long ldb, long long sB, float beta, const float* Cin, long long ldc,
                 long long sC, int batch, int ksplit, int kchunk, const Epi& ep, bool force_swap, cudaStream_t st) {
  // op(A)(m, k) at m am + k ak; op(B)(k, n) at n bnn + k bk
  const long long am = ta ? 1 : lda, ak = ta ? lda : 1;
  const long long bnn = tb ? ldb : 1, bk = tb ? 1 : ldb;
  const bool swap = force_swap || N >= M;
  UmmaArgs g{};
  g.K = K;
  g.ksplit = ksplit;
  g.kchunk = kchunk;
  g.alpha = alpha;
  g.beta = beta;
  if (swap) {
    g.urows = N, g.vrows = M;
    g.U = B, g.usr = bnn, g.usk = bk, g.usb = sB;
    g.V = A, g.vsr = am, g.vsk = ak, g.vsb = sA;
    g.dsr = 1, g.dsc = ldc;
    g.bias_r = 0;
  } else {
    g.urows = M, g.vrows = N;
    g.U = A, g.usr = am, g.usk = ak, g.usb = sA;
    g.V = B, g.vsr = bnn, g.vsk = bk, g.vsb = sB;
    g.dsr = ldc, g.dsc = 1;
    g.bias_r = 1;
  }
  g.dsb = sC;
  g.uvec = g.usk == 1 && al16(g.U) && (g.usr % 4 == 0 || g.urows == 1) && g.usb % 4 == 0;
  g.vvec = g.vsk == 1 && al16(g.V) && (g.vsr % 4 == 0 || g.vrows == 1) && g.vsb % 4 == 0;
  g.Cin = Cin;
  g.Cout = ep.out;
  g.pre = ep.pre;
  g.aux = ep.aux;
  g.bias = ep.bias;
  g.act = ep.act;
  g.dotw = ep.dotw;
  g.dotb = ep.dotb;
  const int zdim = batch * ksplit;
  switch (tile_bn(g.vrows)) {
    case 16: return launch_bn<16>(g, zdim, st);
    case 32: return launch_bn<32>(g, zdim, st);
    case 64: return launch_bn<64>(g, zdim, st);
    default: return launch_bn<128>(g, zdim, st);
  }
}


// K slices of a weight gradient: about four CTAs per SM over the whole launch,
// at least 256 of K per slice, a multiple of the 32-wide chunk
void wgrad_split(int rows, int cols, long long L, int batch, int* ksplit, int* kchunk) {
  const bool swap = cols >= rows;
  const int ur = swap ? cols : rows, vr = swap ? rows : cols;
  const int bn = tile_bn(vr);
  const long long tiles = (long long)((ur + UM - 1) / UM) * ((vr + bn - 1) / bn) * batch;
  long long want = (4LL * sm_count() + tiles - 1) / tiles;
  const long long maxs = (L + 255) / 256;
  if (want > maxs) want = maxs;
  if (want > 65535 / batch) want = 65535 / batch;
  if (want < 1) want = 1;
  long long kc = (L + want - 1) / want;
  kc = (kc + UK - 1) / UK * UK;
  *kchunk = (int)kc;
  *ksplit = (int)((L + kc - 1) / kc);
}

int check_gemm_args(long long M, long long N, long long K, int batch, const void* A, const void* B, const char* who) {
  const std::string w(who);
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0) return fail(FW_EINVAL, w + ": non-positive size");
  if (M > (1LL << 30) || N > (1LL << 30) || K > (1LL << 30)) return fail(FW_EINVAL, w + ": size above 2^30");
  if (A == nullptr || B == nullptr) return fail(FW_EINVAL, w + ": NULL operand");
  if (batch > 65535) return fail(FW_EINVAL, w + ": batch > 65535");
  return FW_OK;
}
}  // namespace umma

int fno_status_read(int* out, int clear) {
  cudaError_t e = cudaMemcpyFromSymbol(out, g_fno_status, sizeof(int));
  if (e == cudaSuccess && clear) {
    const int z = 0;
    e = cudaMemcpyToSymbol(g_fno_status, &z, sizeof(int));
  }
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_status");
}

}  // namespace fw

using namespace fw;
using namespace fw::umma;

extern "C" int fw_fno_sgemm(int transA, int transB, int M, int N, int K, float alpha, const float* A, long long lda,
                            long long strideA, const float* B, long long ldb, long long strideB, float beta, float* C,
                            long long ldc, long long strideC, int batch, void* stream) {
  if (int rc = check_gemm_args(M, N, K, batch, A, B, "fw_fno_sgemm")) return rc;
  if (C == nullptr) return fail(FW_EINVAL, "fw_fno_sgemm: NULL C");
  Epi ep;
  ep.out = C;
  cudaError_t e = gemm(transA, transB, M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, batch,
                       1, K, ep, false, static_cast<cudaStream_t>(stream));
  count_launch(1);
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_sgemm");
}

extern "C" int fw_fno_sgemm_ex(int transA, int transB, int M, int N, int K, float alpha, const float* A, long long lda,
                               long long strideA, const float* B, long long ldb, long long strideB, float beta,
                               const float* C, long long ldc, long long strideC, int batch, const float* bias,
                               float* pre, const float* aux, int act, float* out, void* stream) {
  if (int rc = check_gemm_args(M, N, K, batch, A, B, "fw_fno_sgemm_ex")) return rc;
  if (out == nullptr) return fail(FW_EINVAL, "fw_fno_sgemm_ex: NULL out");
  if (beta != 0.f && C == nullptr) return fail(FW_EINVAL, "fw_fno_sgemm_ex: beta != 0 needs C");
  if (act < 0 || act > 2) return fail(FW_EINVAL, "fw_fno_sgemm_ex: act must be 0 (none), 1 (GELU) or 2 (x GELU'(aux))");
  if (act == 2 && aux == nullptr) return fail(FW_EINVAL, "fw_fno_sgemm_ex: act 2 needs aux");
  Epi ep;
  ep.bias = bias;
  ep.pre = pre;
  ep.aux = aux;
  ep.act = act;
  ep.out = out;
  cudaError_t e = gemm(transA, transB, M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, batch,
                       1, K, ep, false, static_cast<cudaStream_t>(stream));
  count_launch(1);
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_sgemm_ex");
}

extern "C" int fw_fno_wgrad_work(int rows, int cols, long long L, int batch, long long* floats_out) {
  if (floats_out == nullptr) return fail(FW_EINVAL, "fw_fno_wgrad_work: NULL argument");
  if (int rc = check_gemm_args(rows, cols, L, batch, floats_out, floats_out, "fw_fno_wgrad_work")) return rc;
  int ks, kc;
  wgrad_split(rows, cols, L, batch, &ks, &kc);
  *floats_out = (long long)batch * ks * rows * cols;
  return FW_OK;
}

extern "C" int fw_fno_wgrad(int rows, int cols, long long L, const float* dY, long long strideY, const float* X,
                            long long strideX, int batch, float* work, long long work_floats, float* out,
                            int accumulate, void* stream) {
  if (int rc = check_gemm_args(rows, cols, L, batch, dY, X, "fw_fno_wgrad")) return rc;
  if (work == nullptr || out == nullptr) return fail(FW_EINVAL, "fw_fno_wgrad: NULL buffer");
  int ks, kc;
  wgrad_split(rows, cols, L, batch, &ks, &kc);
  const long long need = (long long)batch * ks * rows * cols;
  if (work_floats < need)
    return fail(FW_EINVAL, "fw_fno_wgrad: work buffer of " + std::to_string(work_floats) + " floats, " +
                               std::to_string(need) + " needed");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Epi ep;
  ep.out = work;
  // dY X^T: op(A) = dY_b (rows x L), op(B) = X_b^T; partial tiles of z = b ksplit + s
  cudaError_t e = gemm(0, 1, rows, cols, (int)L, 1.f, dY, L, strideY, X, L, strideX, 0.f, nullptr, cols,
                       (long long)rows * cols, batch, ks, kc, ep, false, st);
  if (e == cudaSuccess) {
    const int E = rows * cols;
    split_sum_kernel<<<(E + 31) / 32, dim3(32, 8), 0, st>>>(batch * ks, E, work, out, accumulate);
    e = cudaGetLastError();
  }
  count_launch(2);
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_wgrad");
}

extern "C" int fw_fno_project(int hidden, int C, long long L, const float* V, long long strideV, int batch,
                              const float* Q1, const float* c1, const float* Q2, const float* c2, float* out,
                              long long strideOut, void* stream) {
  if (int rc = check_gemm_args(hidden, L, C, batch, V, Q1, "fw_fno_project")) return rc;
  if (c1 == nullptr || Q2 == nullptr || c2 == nullptr || out == nullptr)
    return fail(FW_EINVAL, "fw_fno_project: NULL argument");
  if (hidden > UM) return fail(FW_EINVAL, "fw_fno_project: hidden width above 128");
  Epi ep;
  ep.bias = c1;
  ep.out = out;
  ep.dotw = Q2;
  ep.dotb = c2;
  // h = Q1 V_b (hidden x L) with the points along the tensor core's rows; the
  // epilogue reduces each point's hidden vector
  cudaError_t e = gemm(0, 0, hidden, (int)L, C, 1.f, Q1, C, 0, V, L, strideV, 0.f, nullptr, L, strideOut, batch, 1, C,
                       ep, true, static_cast<cudaStream_t>(stream));
  count_launch(1);
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_project");
}
