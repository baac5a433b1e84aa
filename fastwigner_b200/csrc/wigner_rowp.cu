// Persistent FP32 row pass (the kinetic half of the split-operator step).
//
// A row pass transforms pairs of rows along x, multiplies by exp(K) and
// transforms back; one warp owns one row pair, so its transforms need no
// barrier wider than the warp.  This kernel gives every warp its own
// pipeline over a contiguous range of (row pair, instance) work items: the
// next item's two rows (8 KiB at X = 1024) arrive in the warp's shared-memory
// staging buffer by a bulk copy issued as soon as the current rows are in
// registers, so the copy overlaps the item's whole transform pair.  The two
// rows of the phase table an item needs can be staged the same way
// (kRowStageTable; items are row-pair major, so with one table for the batch a
// warp would fetch a table pair once per row pair it visits), or read from L2
// during the spectral multiply, which leaves room for more warps per SM.  The
// stage twiddles live in shared memory for the life of the CTA.  Copies are plain bulk loads from this GPU's own
// memory; every wait is bounded (FW_PASS_TIMEOUT in the plan status word, then
// the warp returns).
#include "fw_internal.h"
#include "tma.cuh"
#include "wigner_tiles.cuh"

namespace fw {

constexpr long long kRowMaxPolls = 1LL << 22;
// warps (independent pipelines) per CTA, one CTA per SM: 12 x 168 registers
// fill the register file; the phase-table rows are then read from L2 (a
// warp-private staged copy would leave room for 8 warps only)
constexpr int kRowWarps = 12;
constexpr bool kRowStageTable = false;

template <int N> struct RowpLayout {
  static constexpr int T = 32, RV = N / T;
  static constexpr size_t W_BYTES = (size_t)2 * N * 4;                                  // the item's two rows
  static constexpr size_t T_BYTES = kRowStageTable ? (size_t)2 * (N / 2 + 1) * 8 : 0;  // their two table rows
  static constexpr size_t EX_BYTES = (size_t)(N + N / 32) * 8;                          // GroupExC exchange
  static constexpr size_t WARP_BYTES = ((W_BYTES + T_BYTES + EX_BYTES + 127) / 128) * 128;
  static constexpr int STW = stage_off(N, RV, N);  // stage-layout twiddles (complex entries)
  static constexpr size_t BYTES = (size_t)kRowWarps * WARP_BYTES + (size_t)STW * 8 + 128;  // + base alignment
};

template <int N>
__global__ void __launch_bounds__(32 * kRowWarps, 1) row_persist_kernel(PassArgs a, int npairs) {
  using C = float2;
  using L = RowpLayout<N>;
  constexpr int T = 32, RV = N / T;
  constexpr size_t HS = N / 2 + 1;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t bars[kRowWarps][2];  // per warp: [0] rows, [1] table rows
  unsigned char* smem = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);  // 128-byte aligned base
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* mine = smem + (size_t)w * L::WARP_BYTES;
  float* Ws = reinterpret_cast<float*>(mine);
  C* Ts = reinterpret_cast<C*>(mine + L::W_BYTES);
  C* exz = reinterpret_cast<C*>(mine + L::W_BYTES + L::T_BYTES);
  C* tws = reinterpret_cast<C*>(smem + (size_t)kRowWarps * L::WARP_BYTES);
  for (int i = threadIdx.x; i < L::STW; i += blockDim.x) tws[i] = reinterpret_cast<const C*>(a.tw)[i];
  if (lane == 0) {
    mbar_init(&bars[w][0], 1);
    mbar_init(&bars[w][1], 1);
    mbar_fence_init();
  }
  __syncthreads();  // the last CTA-wide barrier: from here on every warp runs alone

  const long long n_items = (long long)npairs * a.batch;
  const long long gw = (long long)blockIdx.x * kRowWarps + w, GW = (long long)gridDim.x * kRowWarps;
  const int first = (int)(gw * n_items / GW), last = (int)((gw + 1) * n_items / GW);
  if (first >= last) return;
  auto ipair = [&](int it) { return it / a.batch; };
  auto iinst = [&](int it) { return it % a.batch; };
  auto tkey = [&](int it) { return a.tab_bs != 0 ? it : ipair(it); };
  auto issue_w = [&](int it) {
    const float* src =
        reinterpret_cast<const float*>(a.W) + (size_t)iinst(it) * a.w_bs + (size_t)(2 * ipair(it)) * N;
    mbar_arrive_expect_tx(&bars[w][0], (uint32_t)L::W_BYTES);
    bulk_load(Ws, src, (uint32_t)L::W_BYTES, &bars[w][0]);
  };
  auto issue_t = [&](int it) {
    const C* src = reinterpret_cast<const C*>(a.tab1) + (size_t)iinst(it) * a.tab_bs + (size_t)(2 * ipair(it)) * HS;
    mbar_arrive_expect_tx(&bars[w][1], (uint32_t)L::T_BYTES);
    bulk_load(Ts, src, (uint32_t)L::T_BYTES, &bars[w][1]);
  };
  if (lane == 0) {
    issue_w(first);
    if (kRowStageTable) issue_t(first);
  }
  uint32_t ph_w = 0, ph_t = 0;
  bool w_pending = true, t_pending = kRowStageTable, failed = false;
  GroupExC<float, T> ex{exz};
  const int j = lane;
  const float f = (float)(a.out_scale / (double)N);

  for (int it = first; it < last; ++it) {
    const int rp = ipair(it), b = iinst(it);
    const double sc = a.prev_tot != nullptr ? 1.0 / (__ldcg(a.prev_tot + (size_t)b * a.M) * a.dxdp) : a.scale_const;
    // ---- the item's rows: wait (bounded, decided for the whole warp), into registers, release the buffer
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[w][0], ph_w, kRowMaxPolls))) {
      failed = true;
      break;
    }
    ph_w ^= 1u;
    w_pending = false;
    C v[RV];
    const float s = (float)sc;
#pragma unroll
    for (int m = 0; m < RV; ++m) {
      const int x = j + m * T;
      v[m] = mk<C>(Ws[x] * s, Ws[N + x] * s);
    }
    __syncwarp();
    if (it + 1 < last) {
      if (lane == 0) issue_w(it + 1);
      w_pending = true;
    }
    fft<N, T, RV, -1, C, GroupExC<float, T>, true>(v, j, ex, tws);
    // ---- exp(K) from the staged table rows (Hermitian-unpacked pair multiply)
    if (kRowStageTable && t_pending) {
      if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[w][1], ph_t, kRowMaxPolls))) {
        failed = true;
        break;
      }
      ph_t ^= 1u;
      t_pending = false;
    }
    ex_write_natural<T, RV>(ex, j, v);
    ex.sync();
    const C* tab = kRowStageTable
                       ? Ts
                       : reinterpret_cast<const C*>(a.tab1) + (size_t)b * a.tab_bs + (size_t)(2 * rp) * HS;
    // bin k = j + m T: table row k below N/2 (m < RV/2), row N - k conjugated
    // above it, at m = RV/2 row N/2 - j (N/2 itself, real, for j = 0); the
    // mirrored exchange slot of N - k is one per-thread base minus an
    // immediate, except k = 0 (slot 0).  Resolved per m at compile time: the
    // row pass from 0.1648 to 0.1584 ms per 64 x 1024^2 launch.
    const C* tlo = tab + j;
    const C* thi = tab + (N - j);
    auto ld = [&](const C* p) { return kRowStageTable ? *p : __ldg(p); };
    const int mbase = GroupExC<float, T>::map(N - j);
#pragma unroll
    for (int m = 0; m < RV; ++m) {
      constexpr int H = RV / 2;
      C ea, eb;
      if (m < H) {
        ea = ld(tlo + m * T);
        eb = ld(tlo + HS + m * T);
        if (m == 0 && j == 0) {
          ea.y = 0.f;
          eb.y = 0.f;
        }
      } else {
        ea = ld(thi - m * T);
        eb = ld(thi + HS - m * T);
        if (m == H && j == 0) {
          ea.y = 0.f;
          eb.y = 0.f;
        } else {
          ea.y = -ea.y;
          eb.y = -eb.y;
        }
      }
      const int ms = m == 0 ? (j == 0 ? 0 : mbase) : mbase - GroupExC<float, T>::delta(m * T);
      const C znk = ex.read_at(ms);
      v[m] = two_real_mul(v[m], znk, ea, eb, f);
    }
    ex.sync();  // every lane is done with Ts and the exchange buffer
    if (kRowStageTable && it + 1 < last && tkey(it + 1) != tkey(it)) {
      if (lane == 0) issue_t(it + 1);
      t_pending = true;
    }
    fft<N, T, RV, +1, C, GroupExC<float, T>, true>(v, j, ex, tws);
    float* W = reinterpret_cast<float*>(a.W) + (size_t)b * a.w_bs + (size_t)(2 * rp) * N;
#pragma unroll
    for (int m = 0; m < RV; ++m) {
      const int x = j + m * T;
      W[x] = v[m].x;
      W[N + x] = v[m].y;
    }
  }
  if (failed && lane == 0) {
    if (a.status != nullptr) atomicCAS(a.status, 0, FW_PASS_TIMEOUT);
    // copies still in flight: wait for them once more, bounded, before the warp's buffers are released
    if (w_pending) mbar_wait_bounded(&bars[w][0], ph_w, kRowMaxPolls);
    if (t_pending) mbar_wait_bounded(&bars[w][1], ph_t, kRowMaxPolls);
  }
}

// The persistent row pass takes an FP32 row pass of 1024-point rows with one
// static complex table per instance or per batch, no separable factor, its
// input scale from the per-instance totals (or a constant), 16-byte aligned
// rows and table pairs, and enough row pairs to give every warp of the GPU a
// few items.
bool rowp_eligible(const PassArgs& a, int dtype) {
  if (dtype != FW_F32 || a.X != 1024 || a.tab_real || a.g1 != nullptr || a.prev_part != nullptr) return false;
  if (a.small_shape || a.out_scale != 1.0) return false;
  const uintptr_t mis = reinterpret_cast<uintptr_t>(a.W) | reinterpret_cast<uintptr_t>(a.tab1);
  if ((mis & 15) != 0 || (a.w_bs % 4) != 0 || (a.tab_bs % 2) != 0 || (a.P % 2) != 0) return false;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (long long)a.batch * (a.P / 2) >= 4LL * sms * kRowWarps;
}

cudaError_t launch_row_persist(const PassArgs& a, cudaStream_t st) {
  constexpr int N = 1024;
  using L = RowpLayout<N>;
  auto kern = row_persist_kernel<N>;
  static PerDeviceOnce attr;
  cudaError_t e = set_smem_once(attr, kern, L::BYTES);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int npairs = a.P / 2;
  kern<<<sms, 32 * kRowWarps, L::BYTES, st>>>(a, npairs);
  return cudaGetLastError();
}

}  // namespace fw
