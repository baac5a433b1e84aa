// Tensor-core GEMM (tcgen05 / TMEM) for the FNO surrogate's dense
// contractions: the truncated DFTs, the pointwise channel maps and the
// projection.  C[b] = alpha op(A[b]) op(B[b]) + beta C[b] in FP32 with the
// products on the 5th-generation tensor cores in TF32, split three ways
// (a = a_hi + a_lo with a_hi the TF32 part: a b ~ a_hi b_hi + a_hi b_lo +
// a_lo b_hi) so the result keeps FP32 accuracy (~1e-6 relative) rather than
// TF32's ~1e-3.
//
// One CTA of four warps computes a 128 x BN tile of the product D = U V^T in
// the tensor core's orientation: U (128 rows x K) and V (BN rows x K), both
// K-major in shared memory in the canonical no-swizzle layout -- 8-row x
// 16-byte core matrices, 128 bytes apart along the rows, the K halves of one
// instruction LBO bytes apart.  The D tile accumulates in TMEM (128 lanes x
// BN columns); thread 0 issues the MMAs, a tcgen05.commit arrives on an
// mbarrier when they complete, and the four warps read their 32 lanes back
// with tcgen05.ld for the epilogue.  U is C's contiguous dimension (N) when
// N >= M (SWAP), so each lane stores a run of consecutive C elements; else M.
// Tiles are loaded with ordinary loads (any transpose, any leading dimension,
// zero-filled at the edges), converted and stored in the canonical layout.
// Every mbarrier wait is bounded: on expiry the CTA records FW_FNO_TIMEOUT in
// the FNO status word, writes NaN into its tile, waits once more (bounded)
// for its MMAs, frees its TMEM and returns.
#include <cuda_runtime.h>
#include <stdint.h>
#include "fw_internal.h"
#include "tma.cuh"

namespace fw {

__device__ int g_fno_status;  // FW_FNO_TIMEOUT when a tensor-core GEMM gave up waiting

namespace {

constexpr int UM = 128;   // tile rows (tensor-core M)
constexpr int UK = 32;    // K per shared-memory chunk (four MMAs of K = 8)
constexpr long long kUmmaMaxPolls = 1LL << 20;

struct UmmaArgs {
  int ta, tb, M, N, K;
  float alpha, beta;
  const float* A;
  long long lda, sA;
  const float* B;
  long long ldb, sB;
  float* C;
  long long ldc, sC;
};

// canonical K-major no-swizzle offset (floats) of element (r, k) of a tile
// with `rows` rows and UK columns: core matrix (r/8, k/4) of 8 x 4 floats
__device__ __forceinline__ int canon(int r, int k, int rows) {
  return (k >> 2) * (rows * 4) + (r >> 3) * 32 + (r & 7) * 4 + (k & 3);
}

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

template <int BN, bool SWAP>
__global__ void __launch_bounds__(128) umma_gemm_kernel(UmmaArgs g) {
  constexpr int TCOLS = BN < 32 ? 32 : BN;  // TMEM columns allocated (a power of two >= 32)
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
  const long long bz = blockIdx.z;
  const float* A = g.A + bz * g.sA;
  const float* B = g.B + bz * g.sB;
  float* C = g.C + bz * g.sC;
  const int rows = SWAP ? g.N : g.M;  // tensor-core M side (U)
  const int cols = SWAP ? g.M : g.N;  // tensor-core N side (V)
  const int row0 = blockIdx.y * UM, col0 = blockIdx.x * BN;
  // op(A)(m, k) and op(B)(k, n)
  auto opA = [&](int m, int k) -> float {
    return (m < g.M && k < g.K) ? (g.ta ? A[(size_t)k * g.lda + m] : A[(size_t)m * g.lda + k]) : 0.f;
  };
  auto opB = [&](int k, int n) -> float {
    return (n < g.N && k < g.K) ? (g.tb ? B[(size_t)n * g.ldb + k] : B[(size_t)k * g.ldb + n]) : 0.f;
  };
  // U(r, k) and V(c, k) of the product D = U V^T
  auto U = [&](int r, int k) { return SWAP ? opB(k, r) : opA(r, k); };
  auto V = [&](int c, int k) { return SWAP ? opA(c, k) : opB(k, c); };

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
  uint32_t phase = 0;
  bool pending = false;  // MMAs in flight (uniform)

  for (int k0 = 0; k0 < g.K; k0 += UK) {
    // ---- stage the chunk: U (UM x UK) and V (BN x UK), hi and lo parts
    // consecutive threads take consecutive k when the source is K-contiguous,
    // consecutive rows otherwise
    const bool u_kfast = SWAP ? (g.tb != 0) : (g.ta == 0);
    const bool v_kfast = SWAP ? (g.ta == 0) : (g.tb != 0);
    for (int e = tid; e < UM * UK; e += 128) {
      const int r = u_kfast ? e / UK : e % UM, k = u_kfast ? e % UK : e / UM;
      float hi, lo;
      split_tf32(U(row0 + r, k0 + k), hi, lo);
      const int o = canon(r, k, UM);
      Uh[o] = hi;
      Ul[o] = lo;
    }
    for (int e = tid; e < BN * UK; e += 128) {
      const int c = v_kfast ? e / UK : e % BN, k = v_kfast ? e % UK : e / BN;
      float hi, lo;
      split_tf32(V(col0 + c, k0 + k), hi, lo);
      const int o = canon(c, k, BN);
      Vh[o] = hi;
      Vl[o] = lo;
    }
    proxy_fence_smem();  // the generic stores above become visible to the tensor core
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < UK / 8; ++s) {
        const uint64_t dUh = smem_desc(Uh + s * 2 * UM * 4, UM * 16), dUl = smem_desc(Ul + s * 2 * UM * 4, UM * 16);
        const uint64_t dVh = smem_desc(Vh + s * 2 * BN * 4, BN * 16), dVl = smem_desc(Vl + s * 2 * BN * 4, BN * 16);
        umma_tf32(tmem, dUh, dVh, idesc, (k0 > 0 || s > 0) ? 1u : 0u);
        umma_tf32(tmem, dUh, dVl, idesc, 1u);
        umma_tf32(tmem, dUl, dVh, idesc, 1u);
      }
      umma_commit(&mbar);
    }
    pending = true;
    // the next chunk overwrites the tiles: wait for this chunk's MMAs
    if (!mbar_wait_bounded(&mbar, phase, kUmmaMaxPolls)) abort_flag = 1;
    __syncthreads();
    if (abort_flag) break;
    phase ^= 1u;
    pending = false;
    tc_fence_after();
  }

  // ---- epilogue: warp w holds D rows 32w .. 32w+31 (its TMEM lanes)
  const int r = row0 + warp * 32 + lane;
  if (!abort_flag) {
#pragma unroll
    for (int cb = 0; cb < BN / 16; ++cb) {
      float acc[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16), acc);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int c = col0 + cb * 16 + i;
        if (r < rows && c < cols) {
          float* dst = SWAP ? C + (size_t)c * g.ldc + r : C + (size_t)r * g.ldc + c;
          *dst = g.alpha * acc[i] + (g.beta == 0.f ? 0.f : g.beta * *dst);
        }
      }
    }
  } else {
    if (tid == 0) {
      atomicCAS(&g_fno_status, 0, FW_FNO_TIMEOUT);
      if (pending) mbar_wait_bounded(&mbar, phase, kUmmaMaxPolls);
    }
    for (int i = 0; i < BN; ++i) {
      const int c = col0 + i;
      if (r < rows && c < cols) (SWAP ? C[(size_t)c * g.ldc + r] : C[(size_t)r * g.ldc + c]) = __int_as_float(0x7fc00000);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TCOLS) : "memory");
}

template <int BN, bool SWAP>
cudaError_t launch_bn(const UmmaArgs& g, int batch, cudaStream_t st) {
  const size_t smem = (size_t)2 * (UM + BN) * UK * 4 + 128;
  auto kern = umma_gemm_kernel<BN, SWAP>;
  static PerDeviceOnce attr;
  cudaError_t e = set_smem_once(attr, kern, smem);
  if (e != cudaSuccess) return e;
  const int rows = SWAP ? g.N : g.M, cols = SWAP ? g.M : g.N;
  dim3 grid((cols + BN - 1) / BN, (rows + UM - 1) / UM, batch);
  kern<<<grid, 128, smem, st>>>(g);
  return cudaGetLastError();
}

template <bool SWAP>
cudaError_t launch_swap(const UmmaArgs& g, int batch, cudaStream_t st) {
  const int cols = SWAP ? g.M : g.N;
  if (cols <= 16) return launch_bn<16, SWAP>(g, batch, st);
  if (cols <= 32) return launch_bn<32, SWAP>(g, batch, st);
  if (cols <= 64) return launch_bn<64, SWAP>(g, batch, st);
  return launch_bn<128, SWAP>(g, batch, st);
}
}  // namespace

// The tensor-core path takes products with at least 64 rows on one side (the
// other side is tiled 16 to 128 wide) and K >= 8; smaller ones stay on the
// SIMT kernel.
bool umma_gemm_eligible(int M, int N, int K) { return (M >= 64 || N >= 64) && K >= 8; }

cudaError_t launch_umma_gemm(int ta, int tb, int M, int N, int K, float alpha, const float* A, long long lda,
                             long long sA, const float* B, long long ldb, long long sB, float beta, float* C,
                             long long ldc, long long sC, int batch, cudaStream_t st) {
  UmmaArgs g{ta, tb, M, N, K, alpha, beta, A, lda, sA, B, ldb, sB, C, ldc, sC};
  return N >= M ? launch_swap<true>(g, batch, st) : launch_swap<false>(g, batch, st);
}

int fno_status_read(int* out, int clear) {
  cudaError_t e = cudaMemcpyFromSymbol(out, g_fno_status, sizeof(int));
  if (e == cudaSuccess && clear) {
    const int z = 0;
    e = cudaMemcpyToSymbol(g_fno_status, &z, sizeof(int));
  }
  return e == cudaSuccess ? FW_OK : cuda_fail(e, "fw_fno_status");
}

}  // namespace fw
