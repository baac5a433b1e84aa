// Persistent, TMA-staged column pass for FP32 Wigner functions.
//
// The fused column pass (closing exp(V) of step k, observables from the
// mid-point spectrum, opening exp(V) of step k+1, between one forward and one
// inverse FFT along p) is latency bound when every tile loads its state and
// its phase-table rows from global memory as it starts: a CTA's warps all
// wait on the same loads, then all compete for issue.  This kernel runs one
// CTA per SM over a contiguous range of (column tile, instance) work items
// and keeps the next item's data in flight while it computes the current one:
//
//   * the state tile (N rows x 2*CP columns) arrives in shared memory by
//     bulk-tensor copies (TMA) issued as soon as the current tile has been
//     read into registers, so the copy overlaps the whole transform pair;
//   * the phase-table tile ((N/2+1) rows x CP column pairs) arrives the same
//     way after the current item's mid-point has read its own; consecutive
//     items of a CTA share the column tile (work items are column-tile major),
//     so with one table for the whole batch it is fetched once per column tile
//     a CTA visits rather than once per item;
//   * the stage twiddles live in shared memory for the life of the CTA.
//
// All copies are loads from this GPU's own memory without multicast.  Every
// wait on an mbarrier is bounded; if a copy never completes the CTA records
// FW_PASS_TIMEOUT in the plan's status word and returns.
#include <mutex>
#include <vector>
#include "fw_internal.h"
#include "tma.cuh"
#include "wigner_tiles.cuh"

namespace fw {

constexpr long long kTmaMaxPolls = 1LL << 22;  // polls of one mbarrier wait before the CTA gives up

// Rows of the phase-table tile one bulk copy moves, and the copies per tile
// (a box dimension may not exceed 256).  ROWS is a multiple of 4, so that
// every copy's shared-memory destination (ROWS rows of 32, 64 or 128 bytes)
// starts on 128 bytes; the last copy may run past the table's N/2+1 rows,
// which the copy fills with zeros.
template <int N> struct TabBox {
  static constexpr int H = N / 2 + 1;
  static constexpr int NL = (H + 255) / 256;
  static constexpr int ROWS = ((H + NL - 1) / NL + 3) / 4 * 4;
  static_assert(ROWS <= 256, "table box too tall");
};

// Launch shapes of the persistent column pass.  MINB CTAs of CP*T threads per
// SM.  BMAJOR: work items instance-major (consecutive items of a CTA are
// neighbouring column tiles of one instance, so a tile whose rows are narrower
// than a 64-byte DRAM line finds the rest of the line in L2; the table tile is
// fetched for every item) instead of column-tile major (consecutive items share
// the table tile).  PSUM_ALIAS: the per-bin p-weight sums live in the table
// tile's buffer once the mid-point has read the table (only with a table fetch
// per item).
template <int N> struct ColpShape;
// 1024: one CTA of 16 warps per SM, eight column pairs (64-byte state rows),
// column-tile-major items so a shared table tile is fetched once per column
// tile a CTA visits.  (Four pairs at two CTAs per SM, instance-major with a
// table fetch per item and the sums in the table buffer, measured 0.330 vs
// 0.315 ms per 64 x 1024^2 launch.)
template <> struct ColpShape<1024> {
  static constexpr int T = 64, CP = 8, MINB = 1;
  static constexpr bool BMAJOR = false, PSUM_ALIAS = false;
};

template <int N, int T, int CP, bool PSUM_ALIAS> struct ColpLayout {
  static constexpr int WROWB = 2 * CP;                        // floats per state-tile row
  static constexpr size_t W_FLOATS = (size_t)N * WROWB;
  static constexpr size_t T_FLOATS = (size_t)TabBox<N>::NL * TabBox<N>::ROWS * 4 * CP;  // complex tables
  static constexpr size_t EX_FLOATS = col_ex_reals<float, N, T, CP>();
  static constexpr size_t PSUM_FLOATS = PSUM_ALIAS ? 0 : (size_t)2 * N;
  // + twiddles, + 128 bytes to align the base of the buffers
  static constexpr size_t BYTES = (W_FLOATS + T_FLOATS + EX_FLOATS + PSUM_FLOATS) * 4 + (size_t)N * 8 + 128;
  static_assert(!PSUM_ALIAS || T_FLOATS >= (size_t)2 * N, "psum must fit in the table buffer");
  // every bulk-tensor destination on 128 bytes: the state boxes, the table
  // buffer and each table box (complex and real tables)
  static_assert((W_FLOATS * 4) % 128 == 0 && ((size_t)(N < 256 ? N : 256) * WROWB * 4) % 128 == 0,
                "state boxes off 128 bytes");
  static_assert(((size_t)TabBox<N>::ROWS * 4 * CP * 4) % 128 == 0 && ((size_t)TabBox<N>::ROWS * 2 * CP * 4) % 128 == 0,
                "table boxes off 128 bytes");
};

// Mid-point of the fused column pass with the phase-table tile in shared
// memory (Ts: row kk holds the CP column pairs' complex entries, 4 floats per
// pair; real Bloch tables take the regular column pass).  The same factor
// closes step k and opens step k+1 (time-independent Hamiltonian).  Otherwise
// as fused_mid.  Without FUSED the pass is one potential half-step (the
// opening one of a call, or the closing one with the observables of the
// result).  OBS: the observable sums are taken (a compile-time switch, like
// the table kind: 0.3127 -> 0.3045 ms per 64 x 1024^2 launch).  v holds
// the spectrum of the unscaled tile: the input scale sc multiplies the
// closing factor and the observable sums instead of every element.  The
// table row min(k, N-k), its Hermitian fold and the mirrored exchange slot of
// N-k are resolved per m at compile time (k = j + m T, j < T), with the
// mirror slots one per-thread base minus an immediate.
template <int N, int T, int RV, int CP, bool FUSED, bool OBS, typename EX>
__device__ __forceinline__ void fused_mid_staged(const PassArgs& a, int b, float2 (&v)[RV], const int j, EX& ex,
                                                 int c, const float* Ts, float2* psum, MidSums<float>& o,
                                                 double sc) {
  using C = float2;
  static_assert(N == RV * T && RV % 2 == 0 && T % RV == 0 && EX::kFold && EX::kL == ilog2_c(RV),
                "folded mirror addressing needs T a multiple of RV and a layout padded per RV");
  const C* G = reinterpret_cast<const C*>(a.wph) + (size_t)b * a.wph_bs;
  constexpr bool obs = OBS;
  const float hs = (float)(0.5 / (double)N * sc);
  C u[RV];
  ex_write_natural<T, RV>(ex, j, v);
  ex.sync();
  o.s2 = 0;
  o.ca = 0;
  o.cb = 0;
#pragma unroll
  for (int q = 0; q < MAXO; ++q) o.sq[q] = 0;
  const int mbase = ex.map(N - j);  // slot of N - j (virtual for j = 0); N - k is mbase - delta(m T)
#pragma unroll
  for (int m = 0; m < RV; ++m) {
    // k = j + m T: below N/2 for m < RV/2, else the table holds row N - k (conjugated, except at k = N/2)
    constexpr int H = RV / 2;
    const int kk = m < H ? j + m * T : N - j - m * T;
    C ea, eb;
    {
      const float4 e = *reinterpret_cast<const float4*>(Ts + (size_t)kk * (4 * CP) + 4 * c);
      ea = mk<C>(e.x, e.y);
      eb = mk<C>(e.z, e.w);
      if (m == 0 || m == H) {  // k = 0 or k = N/2 when j = 0: real entries
        if (j == 0) {
          ea.y = 0.f;
          eb.y = 0.f;
        } else if (m == H) {
          ea.y = -ea.y;
          eb.y = -eb.y;
        }
      } else if (m > H) {
        ea.y = -ea.y;
        eb.y = -eb.y;
      }
    }
    const int ms = m == 0 ? (j == 0 ? ex.map(0) : mbase) : mbase - EX::delta(m * T);
    const C zc = cconj(ex.read_at(ms));
    const C A = cmul(cadd(v[m], zc), ea);   // 2/sc x spectrum of column a at the mid-point
    const C Bi = cmul(csub(v[m], zc), eb);  // 2i/sc x spectrum of column b at the mid-point
    if (obs) {
      o.s2 += (double)(A.x * A.x + A.y * A.y + Bi.x * Bi.x + Bi.y * Bi.y);
      if (m == 0 && j == 0) {
        o.ca = A.x;
        o.cb = Bi.y;
      }
      u[m] = mk<C>(A.x + Bi.y, A.y - Bi.x);  // 2/sc x (spectrum a + spectrum b)
    }
    // fused: close step k and open step k+1 with the same factor; a single
    // half-step (the opening one of a call, or its closing one) repacks A, Bi
    v[m] = FUSED ? cscale(cadd(cmul(A, ea), cmul(Bi, eb)), hs) : cscale(cadd(A, Bi), hs);
  }
  // per-bin sums over the tile's CP column pairs; lane c ends with bins
  // m = c * RV/CP + i
  if (obs && a.Mp > 0) halving_sum<CP, RV>(u, c);
  ex.sync();  // the table tile and the exchange buffer are no longer read
  if (obs && a.Mp > 0) {
#pragma unroll
    for (int i = 0; i < RV / CP; ++i) psum[j + (c * (RV / CP) + i) * T] = u[i];
    ex.sync();
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
      const C u = psum[k];
      C g[MAXO];
      load_bin_weights<float>(G + (size_t)k * MAXO, a.Mp, g);
#pragma unroll
      for (int q = 0; q < MAXO; ++q)
        if (q < a.Mp) o.sq[q] += (double)u.x * (double)g[q].x + (double)u.y * (double)g[q].y;
    }
  }
  if (obs) {  // the sums of the unscaled spectrum, scaled once
    o.s2 *= sc * sc;
    o.ca *= sc;
    o.cb *= sc;
#pragma unroll
    for (int q = 0; q < MAXO; ++q) o.sq[q] *= sc;
  }
}

struct ColpCtl {
  int ntiles;    // column tiles per instance
  int tab_inst;  // phase tables per instance (1) or one for the batch (0)
};

template <int N, int T, int CP, int MINB, bool BMAJOR, bool PSUM_ALIAS, bool FUSED, bool OBS>
__global__ void __launch_bounds__(CP* T, MINB)
    col_persist_kernel(const __grid_constant__ CUtensorMap mW, const __grid_constant__ CUtensorMap mT, PassArgs a,
                       ColpCtl ctl) {
  using C = float2;
  using L = ColpLayout<N, T, CP, PSUM_ALIAS>;
  constexpr int RV = N / T;
  constexpr int NTHR = CP * T;
  constexpr int WBOX = N < 256 ? N : 256;  // state rows per bulk copy
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t bars[2];  // [0] state tile, [1] table tile
  __shared__ double red[34];
  __shared__ double ored[NTHR / 32][2 + 2 * MAXO];
  __shared__ int abort_flag;
  // bulk-tensor copies land on 128-byte boundaries: align the buffers' base
  unsigned char* smem = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
  float* Ws = reinterpret_cast<float*>(smem);
  float* Ts = Ws + L::W_FLOATS;
  float* exb = Ts + L::T_FLOATS;
  C* tw = reinterpret_cast<C*>(exb + L::EX_FLOATS);
  C* psum = PSUM_ALIAS ? reinterpret_cast<C*>(Ts) : tw + N;

  const int n_items = a.batch * ctl.ntiles;
  const int first = (int)((long long)blockIdx.x * n_items / gridDim.x);
  const int last = (int)((long long)(blockIdx.x + 1) * n_items / gridDim.x);
  if (first >= last) return;  // the same for every thread of the CTA
  const int tid = threadIdx.x;
  constexpr int tab_rowf = 4 * CP;  // floats per table-tile row (complex tables)
  const uint32_t w_bytes = (uint32_t)(L::W_FLOATS * 4);
  const uint32_t t_bytes = (uint32_t)(TabBox<N>::NL * TabBox<N>::ROWS * tab_rowf * 4);
  auto item_t = [&](int it) { return BMAJOR ? it % ctl.ntiles : it / a.batch; };
  auto item_b = [&](int it) { return BMAJOR ? it / ctl.ntiles : it % a.batch; };
  // key of the table tile an item reads; with the p-weight sums in the table
  // buffer every item fetches its tile
  auto tab_key = [&](int it) { return (ctl.tab_inst || PSUM_ALIAS) ? it : item_t(it) * a.batch; };
  auto issue_w = [&](int it) {
    mbar_arrive_expect_tx(&bars[0], w_bytes);
#pragma unroll
    for (int r = 0; r < N; r += WBOX) tma_load_3d(Ws + (size_t)r * L::WROWB, &mW, &bars[0], item_t(it) * 2 * CP, r, item_b(it));
  };
  auto issue_t = [&](int it) {
    mbar_arrive_expect_tx(&bars[1], t_bytes);
    const int tb = ctl.tab_inst ? item_b(it) : 0;
#pragma unroll
    for (int l = 0; l < TabBox<N>::NL; ++l)
      tma_load_3d(Ts + (size_t)l * TabBox<N>::ROWS * tab_rowf, &mT, &bars[1], item_t(it) * tab_rowf,
                  l * TabBox<N>::ROWS, tb);
  };

  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
    abort_flag = 0;
  }
  for (int i = tid; i < N; i += NTHR) tw[i] = reinterpret_cast<const C*>(a.tw)[i];
  __syncthreads();
  if (tid == 0) {
    issue_w(first);
    issue_t(first);
  }
  // parity of the next completion of each barrier, and whether a copy is in
  // flight on it (the same on every thread: issue decisions are uniform)
  uint32_t ph_w = 0, ph_t = 0;
  bool w_pending = true, t_pending = true;

  const int c = tid % CP;
  const int j = tid / CP;
  __builtin_assume(j >= 0 && j < T);
  using EXT = ColPadExC<float, CP, ilog2_c(RV)>;
  EXT ex{reinterpret_cast<C*>(exb), c};

  for (int it = first; it < last; ++it) {
    const int tile = item_t(it), b = item_b(it);
    const double sc = prev_scale(a, b, red, tile == 0);
    // ---- state tile: wait, read into registers, release the buffer to the next copy
    const bool ok_w = mbar_wait_bounded(&bars[0], ph_w, kTmaMaxPolls);
    if (ok_w) {
      ph_w ^= 1u;
      w_pending = false;
    } else {
      abort_flag = 1;
    }
    C v[RV];  // unscaled: the input scale is applied at the mid-point
#pragma unroll
    for (int m = 0; m < RV; ++m) {
      const float2 w = *reinterpret_cast<const float2*>(Ws + (size_t)(j + m * T) * L::WROWB + 2 * c);
      v[m] = mk<C>(w.x, w.y);
    }
    // release the buffer at once, so the next copy overlaps the whole transform
    // pair (issuing it after the forward transform, one barrier fewer, measured
    // 0.341 vs 0.315 ms per 64 x 1024^2 launch)
    __syncthreads();
    if (abort_flag) break;
    if (it + 1 < last) {
      if (tid == 0) issue_w(it + 1);
      w_pending = true;
    }
    // ---- forward transform along p
    fft<N, T, RV, -1, C, EXT>(v, j, ex, tw);
    // ---- mid-point: wait for this item's table tile if one is in flight
    if (t_pending) {
      const bool ok_t = mbar_wait_bounded(&bars[1], ph_t, kTmaMaxPolls);
      if (ok_t) {
        ph_t ^= 1u;
        t_pending = false;
      } else {
        abort_flag = 1;
      }
      __syncthreads();
      if (abort_flag) break;
    }
    MidSums<float> o;
    fused_mid_staged<N, T, RV, CP, FUSED, OBS>(a, b, v, j, ex, c, Ts, psum, o, sc);  // ends with a CTA barrier
    const int xa = tile * 2 * CP + 2 * c;
    if (OBS) mid_store<float, N, CP, NTHR>(a, b, tile, ctl.ntiles, o, xa, ored);
    // the next item's table tile (the p-weight sums in the table buffer have
    // been read before mid_store's barrier)
    t_pending = it + 1 < last && tab_key(it + 1) != tab_key(it);
    if (PSUM_ALIAS && !OBS) __syncthreads();  // no mid_store barrier to lean on
    if (tid == 0 && t_pending) issue_t(it + 1);
    // ---- inverse transform and store
    fft<N, T, RV, +1, C, EXT>(v, j, ex, tw);
    float* W = reinterpret_cast<float*>(a.W) + (size_t)b * a.w_bs;
    col_store<float, N, T, RV>(a, v, W, j, xa);
  }
  if (abort_flag && tid == 0) {
    if (a.status != nullptr) atomicCAS(a.status, 0, FW_PASS_TIMEOUT);
    // copies still in flight: wait for them once more, bounded, before the CTA's shared memory is released
    if (w_pending) mbar_wait_bounded(&bars[0], ph_w, kTmaMaxPolls);
    if (t_pending) mbar_wait_bounded(&bars[1], ph_t, kTmaMaxPolls);
  }
}

// ---------------------------------------------------------------------------
// host side

namespace {
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

// FP32 3-D tensor map: dims {d0 (innermost), d1, d2}, byte strides of dims 1
// and 2, box {b0, b1, 1}.
bool encode_3d(CUtensorMap* m, const void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1, uint64_t s2,
               uint32_t b0, uint32_t b1, CUtensorMapL2promotion promo) {
  EncodeTiled enc = encoder();
  if (enc == nullptr) return false;
  const cuuint64_t dims[3] = {d0, d1, d2};
  const cuuint64_t strides[2] = {s1, s2};
  const cuuint32_t box[3] = {b0, b1, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <int N>
cudaError_t launch_colp_cfg(const PassArgs& a, cudaStream_t st, int* nparts) {
  using S = ColpShape<N>;
  constexpr int T = S::T, CP = S::CP;
  using L = ColpLayout<N, T, CP, S::PSUM_ALIAS>;
  const int P = a.P, X = a.X;
  const int ntiles = X / (2 * CP);
  const int tab_rowf = (a.tab_real ? 2 : 4) * CP;
  const uint64_t tab_cols = (uint64_t)X * (a.tab_real ? 1 : 2);  // floats per table row
  const int ntab = a.tab_bs != 0 ? a.batch : 1;
  CUtensorMap mW, mT;
  const uint64_t wrow = (uint64_t)X * 4, winst = (uint64_t)a.w_bs * 4;
  const uint64_t trow = tab_cols * 4;
  const uint64_t tinst = a.tab_bs != 0 ? (uint64_t)a.tab_bs * (a.tab_real ? 4 : 8) : trow * (uint64_t)(P / 2 + 1);
  // state rows of a tile are 2*CP floats: fetch exactly those sectors from DRAM
  // (the neighbouring tile's half of each line is read by another CTA at
  // another time); table rows are whole 128-byte lines
  if (!encode_3d(&mW, a.W, (uint64_t)X, (uint64_t)P, (uint64_t)a.batch, wrow, winst, 2 * CP, N < 256 ? N : 256,
                 CU_TENSOR_MAP_L2_PROMOTION_L2_64B) ||
      !encode_3d(&mT, a.tab1, tab_cols, (uint64_t)(P / 2 + 1), (uint64_t)ntab, trow, tinst, (uint32_t)tab_rowf,
                 (uint32_t)TabBox<N>::ROWS, CU_TENSOR_MAP_L2_PROMOTION_L2_128B))
    return cudaErrorInvalidValue;
  const bool obs = a.part_out != nullptr;
  auto kern = a.fuse_mid ? (obs ? col_persist_kernel<N, T, CP, S::MINB, S::BMAJOR, S::PSUM_ALIAS, true, true>
                                : col_persist_kernel<N, T, CP, S::MINB, S::BMAJOR, S::PSUM_ALIAS, true, false>)
                         : (obs ? col_persist_kernel<N, T, CP, S::MINB, S::BMAJOR, S::PSUM_ALIAS, false, true>
                                : col_persist_kernel<N, T, CP, S::MINB, S::BMAJOR, S::PSUM_ALIAS, false, false>);
  static PerDeviceOnce attr[4];
  cudaError_t e = set_smem_once(attr[(a.fuse_mid ? 2 : 0) + (obs ? 1 : 0)], kern, L::BYTES);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  ColpCtl ctl{ntiles, a.tab_bs != 0 ? 1 : 0};
  const int items = a.batch * ntiles;
  const int ctas = sms * S::MINB;
  const int grid = items < ctas ? items : ctas;
  kern<<<grid, CP * T, L::BYTES, st>>>(mW, mT, a, ctl);
  if (nparts) *nparts = ntiles;
  return cudaGetLastError();
}
}  // namespace

// The persistent column pass handles an FP32 column pass with one
// time-independent table (tab1 == tab2 when fused, or a single half-step
// without tab2; no separable factors, no x-p mask, no blends; the p-weight
// spectra when p-observables are taken) whose tiles and strides meet the
// bulk-copy rules, over enough work
// items to fill the GPU at least twice; it uses the regular launch shape
// (ColCfg) of the transform length, so the partial-sum records per instance
// are the ones the plan sized for.
bool colp_eligible(const PassArgs& a, int dtype) {
  if (dtype != FW_F32 || a.tab1 == nullptr || a.g1 != nullptr || a.g2 != nullptr) return false;
  if (a.fuse_mid ? a.tab1 != a.tab2 : a.tab2 != nullptr) return false;
  if (a.part_out != nullptr && a.Mp > 0 && a.wph == nullptr) return false;  // p-observables need the weight spectra
  if (a.tab_real) return false;  // Bloch tables: the regular column pass
  if (a.bxp != nullptr || a.blend_pre || a.blend_post || a.small_shape) return false;
  if (a.P != 1024) return false;
  const uintptr_t mis = reinterpret_cast<uintptr_t>(a.W) | reinterpret_cast<uintptr_t>(a.tab1);
  if ((mis & 15) != 0 || (a.w_bs % 4) != 0) return false;
  if (a.tab_bs != 0 && (a.tab_bs * (a.tab_real ? 4 : 8)) % 16 != 0) return false;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  using S = ColpShape<1024>;
  if (a.X % (2 * S::CP) != 0 || col_parts(dtype, a.P, a.X, 0) != a.X / (2 * S::CP)) return false;
  return (long long)a.batch * (a.X / (2 * S::CP)) >= 2LL * S::MINB * sms && encoder() != nullptr;
}

cudaError_t launch_col_persist(const PassArgs& a, cudaStream_t st, int* nparts) {
  return launch_colp_cfg<1024>(a, st, nparts);
}

}  // namespace fw
