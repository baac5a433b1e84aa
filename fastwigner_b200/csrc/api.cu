// C ABI of libfastwigner: plan objects, step sequencing, error reporting.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <vector>
#include "fw_internal.h"
#include "passes.cuh"

namespace fw {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
int fail(int code, const std::string& msg) { set_error(msg); return code; }
int cuda_fail(cudaError_t e, const char* where) {
  return fail(FW_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// exp(-2 pi i k / N), k < N, computed in FP64 with the angle reduced exactly
// through integer arithmetic on k (so the table is accurate to FP64 rounding).
static std::vector<double> twiddles(int n) {
  std::vector<double> t(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    t[2 * k] = cos(a);
    t[2 * k + 1] = sin(a);
  }
  return t;
}

// Stage-layout twiddle table of an n-point transform with rv values per
// thread (fft.cuh, stage_off): the entries of twiddles(n) at k = bm r n/(ns R),
// computed by the same expression, so both tables hold identical values.
static std::vector<double> stage_twiddles(int n, int rv) {
  std::vector<double> t;
  for (int ns = rv; ns < n; ns *= rv) {
    const int R = n / ns >= rv ? rv : n / ns;
    const int s = n / (ns * R);
    for (int r = 1; r < R; ++r)
      for (int bm = 0; bm < ns; ++bm) {
        const double a = -2.0 * M_PI * (double)(bm * r * s) / (double)n;
        t.push_back(cos(a));
        t.push_back(sin(a));
      }
  }
  if (t.empty()) t.assign(2, 0.0);
  return t;
}

static int upload_twiddles(int n, int dtype, void** dev, int rv = 0) {
  std::vector<double> t = rv > 0 ? stage_twiddles(n, rv) : twiddles(n);
  cudaError_t e;
  if (dtype == FW_F64) {
    e = cudaMalloc(dev, t.size() * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(twiddles)");
    e = cudaMemcpy(*dev, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice);
  } else {
    std::vector<float> f(t.begin(), t.end());
    e = cudaMalloc(dev, f.size() * sizeof(float));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(twiddles)");
    e = cudaMemcpy(*dev, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(twiddles)");
  return FW_OK;
}

}  // namespace fw

using namespace fw;

struct fw_wigner_plan {
  int P, X, batch, dtype;
  int small = 0;       // small-batch launch shapes (small_shapes)
  int nparts;          // column-pass CTAs per instance (partials per instance)
  void* twP = nullptr; // twiddles for length P
  void* twX = nullptr; // twiddles for length X
  void* twsX = nullptr; // stage-layout twiddles of the row pass (length X)
  double* ring = nullptr;  // 2 x batch x nparts x MMAX partial sums
  double* wsum = nullptr;  // scratch for fw_wigner_weighted_sum partials
  int wsum_blocks = 0;
  void* wph = nullptr;  // spectra of the p-observable weights (wph_nb x 4 x P complex)
  int wph_nb = 0;
  double* tot = nullptr;  // per-instance reduced partial sums (batch x MMAX)
  int* status = nullptr;  // device status word (FW_PASS_TIMEOUT); may be null
};

static constexpr int MMAX = 2 + 8;

extern "C" int fw_abi_version(void) { return FW_ABI_VERSION; }
extern "C" const char* fw_last_error(void) { return g_err.c_str(); }
extern "C" int fw_wigner_num_obs(int Mx, int Mp) { return 2 + Mx + Mp; }

extern "C" int fw_wigner_plan_create(int P, int X, int batch, int dtype, fw_wigner_plan** out) {
  if (out == nullptr) return fail(FW_EINVAL, "fw_wigner_plan_create: out is NULL");
  *out = nullptr;
  if (dtype != FW_F32 && dtype != FW_F64) return fail(FW_EINVAL, "fw_wigner_plan_create: dtype must be FW_F32 or FW_F64");
  if (!size_supported(P) || !size_supported(X))
    return fail(FW_EINVAL, "fw_wigner_plan_create: P_gridDIM and X_gridDIM must be even and in [4, 4096] (got " +
                               std::to_string(P) + " x " + std::to_string(X) + ")");
  if (batch < 1 || batch > 65535) return fail(FW_EINVAL, "fw_wigner_plan_create: batch must be in [1, 65535]");
  const int small = small_shapes(dtype, P, X, batch);
  const int np = col_parts(dtype, P, X, small);
  if (np <= 0) return fail(FW_EINVAL, "fw_wigner_plan_create: unsupported X for the column pass tile");
  fw_wigner_plan* p = new fw_wigner_plan();
  p->P = P; p->X = X; p->batch = batch; p->dtype = dtype; p->nparts = np; p->small = small;
  int rc = upload_twiddles(P, dtype, &p->twP);
  if (rc == FW_OK) rc = upload_twiddles(X, dtype, &p->twX);
  if (rc == FW_OK) rc = upload_twiddles(X, dtype, &p->twsX, row_rv(dtype, X, small));
  if (rc == FW_OK) {
    cudaError_t e = cudaMalloc(&p->ring, sizeof(double) * 2 * (size_t)batch * np * MMAX);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc(partials)");
  }
  if (rc == FW_OK) {
    p->wsum_blocks = 256;
    cudaError_t e = cudaMalloc(&p->wsum, sizeof(double) * 2 * (size_t)batch * p->wsum_blocks);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc(weighted-sum scratch)");
  }
  if (rc == FW_OK) {
    // per-instance weight spectra while they fit in 64 MiB, else shared weights only
    const size_t per = (size_t)4 * P * 2 * (dtype == FW_F64 ? sizeof(double) : sizeof(float));
    p->wph_nb = per * (size_t)batch <= ((size_t)64 << 20) ? batch : 1;
    cudaError_t e = cudaMalloc(&p->wph, per * p->wph_nb);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc(weight spectra)");
  }
  if (rc == FW_OK) {
    cudaError_t e = cudaMalloc(&p->tot, sizeof(double) * (size_t)batch * MMAX);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc(instance totals)");
  }
  if (rc == FW_OK) {
    cudaError_t e = cudaMalloc(&p->status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->status, 0, sizeof(int));
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc(plan status)");
  }
  if (rc != FW_OK) {
    fw_wigner_plan_destroy(p);
    return rc;
  }
  *out = p;
  return FW_OK;
}

extern "C" int fw_wigner_plan_destroy(fw_wigner_plan* p) {
  if (p == nullptr) return FW_OK;
  cudaFree(p->twP);
  cudaFree(p->twX);
  cudaFree(p->twsX);
  cudaFree(p->ring);
  cudaFree(p->wsum);
  cudaFree(p->wph);
  cudaFree(p->tot);
  cudaFree(p->status);
  delete p;
  return FW_OK;
}

extern "C" int fw_wigner_plan_status(fw_wigner_plan* p, int* status_out, int clear) {
  if (p == nullptr || status_out == nullptr) return fail(FW_EINVAL, "fw_wigner_plan_status: NULL argument");
  *status_out = 0;
  if (p->status == nullptr) return FW_OK;
  cudaError_t e = cudaMemcpy(status_out, p->status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && clear) e = cudaMemset(p->status, 0, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "fw_wigner_plan_status");
  return FW_OK;
}

static inline const void* advance(const void* base, long long elems, size_t esz) {
  return base == nullptr ? nullptr : static_cast<const char*>(base) + (ptrdiff_t)(elems * (long long)esz);
}

namespace fw {
static long long g_launches = 0;
// optional per-launch timing hook used by fw_wigner_propagate_timed
struct LaunchTimer {
  std::vector<cudaEvent_t> ev;
  std::vector<int> kind;
  cudaStream_t st = nullptr;
  bool on = false;
  void mark(int k) {
    if (!on) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, st);
    ev.push_back(e);
    kind.push_back(k);
  }
};
static thread_local LaunchTimer* g_timer = nullptr;
}  // namespace fw

void fw::count_launch(long long n) { g_launches += n; }
extern "C" long long fw_launch_count(void) { return g_launches; }

extern "C" int fw_wigner_propagate(fw_wigner_plan* plan, const fw_wigner_desc* d, int steps, void* stream) {
  if (plan == nullptr || d == nullptr) return fail(FW_EINVAL, "fw_wigner_propagate: NULL plan or desc");
  if (steps < 0) return fail(FW_EINVAL, "fw_wigner_propagate: steps must be >= 0");
  if (steps == 0) return FW_OK;
  if (d->W == nullptr || d->tabV == nullptr || d->tabK == nullptr)
    return fail(FW_EINVAL, "fw_wigner_propagate: W, tabV and tabK are required");
  if (d->Mx < 0 || d->Mx > 4 || d->Mp < 0 || d->Mp > 4) return fail(FW_EINVAL, "fw_wigner_propagate: Mx, Mp must be in [0, 4]");
  if ((d->Mx > 0 && d->wx == nullptr) || (d->Mp > 0 && d->wp == nullptr))
    return fail(FW_EINVAL, "fw_wigner_propagate: observable weights missing");
  if (d->step_kind == FW_STEP_SPLIT && d->s0 == nullptr) return fail(FW_EINVAL, "fw_wigner_propagate: split steps need s0");
  if (d->step_kind != FW_STEP_FUSED && d->step_kind != FW_STEP_SPLIT) return fail(FW_EINVAL, "fw_wigner_propagate: bad step_kind");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t rs = plan->dtype == FW_F64 ? sizeof(double) : sizeof(float);
  const size_t tes = d->tab_real ? rs : 2 * rs;
  const int M = 2 + d->Mx + d->Mp;
  const int B = plan->batch;
  const size_t ring_slot = (size_t)B * plan->nparts * M;

  PassArgs base{};
  base.W = d->W;
  base.w_bs = d->w_bstride;
  base.P = plan->P;
  base.X = plan->X;
  base.batch = B;
  base.tab_bs = d->tab_bstride;
  base.tab_real = d->tab_real;
  base.dxdp = d->dxdp;
  base.scale_const = 1.0;
  base.M = M;
  base.Mx = d->Mx;
  base.Mp = d->Mp;
  base.wx_bs = d->wx_bstride;
  base.wp_bs = d->wp_bstride;
  base.s0 = d->s0;
  base.s0_bs = d->s0_bstride;
  base.blend_c = d->blend_c;
  base.out_scale = 1.0;
  base.small_shape = plan->small;
  base.status = plan->status;

  auto tabV = [&](int k) { return advance(d->tabV, (long long)k * d->tabV_step, tes); };
  auto tabK = [&](int k) { return advance(d->tabK, (long long)k * d->tabK_step, tes); };
  auto gV = [&](int k) { return advance(d->gV, (long long)k * d->gV_step, 2 * rs); };
  auto gK = [&](int k) { return advance(d->gK, (long long)k * d->gK_step, 2 * rs); };
  auto ring = [&](int k) { return plan->ring + (size_t)(k & 1) * ring_slot; };
  auto hist = [&](int k) { return d->obs_out == nullptr ? nullptr : d->obs_out + (size_t)k * B * M; };

  // With a totals buffer, a batch of 4 or more and more than 8 partial records
  // per instance, a small kernel after each column pass with partial sums
  // reduces them per instance (and records the observable history); the next
  // pass reads one total per instance.  For smaller batches or few records
  // (where that launch costs more than it saves: about 1 us per step for
  // 14-18 instances of 256 x 128 ... 512 x 256) and for fixed-scratch plans
  // every CTA of the next pass reduces the partials itself.
  const bool totals = plan->tot != nullptr && B >= 4 && plan->nparts > 8;
  auto col = [&](PassArgs a) -> int {
    a.tw = plan->twP;
    int np = 0;
    cudaError_t e = launch_col(a, plan->dtype, st, &np);
    if (e != cudaSuccess) return cuda_fail(e, "column pass launch");
    ++g_launches;
    if (g_timer) g_timer->mark(0);
    if (totals && a.part_out != nullptr) {
      e = launch_totals(a.part_out, plan->nparts, M, B, plan->tot, a.obs_hist, st);
      if (e != cudaSuccess) return cuda_fail(e, "totals launch");
      ++g_launches;
      if (g_timer) g_timer->mark(3);
    }
    return FW_OK;
  };
  auto row = [&](PassArgs a) -> int {
    a.tw = plan->twsX;
    cudaError_t e = launch_row(a, plan->dtype, st);
    if (e != cudaSuccess) return cuda_fail(e, "row pass launch");
    ++g_launches;
    if (g_timer) g_timer->mark(1);
    return FW_OK;
  };
  auto obs_args = [&](PassArgs& a, int k) {
    a.part_out = ring(k);
    a.wx = d->wx == nullptr ? nullptr : d->wx + (size_t)k * d->wx_step;
    a.wp = d->wp == nullptr ? nullptr : d->wp + (size_t)k * d->wp_step;
    if (totals) a.obs_hist = hist(k);  // read by the totals kernel, not by the pass
  };
  auto prev_args = [&](PassArgs& a, int k) {  // normalisation from the partials of step k
    if (totals) {
      a.prev_tot = plan->tot;
      return;
    }
    a.prev_part = ring(k);
    a.prev_nparts = plan->nparts;
    a.obs_hist = hist(k);
  };
  int rc = FW_OK;
  if (d->step_kind == FW_STEP_FUSED) {
    // The two potential half-steps between kinetic steps share one transform
    // pair (observables from the mid-point spectrum) unless an x-p mask
    // (bxp) sits between them, or the p-weights change with the step or do
    // not fit the plan's spectrum buffer.
    bool fuse = d->bxp == nullptr && !col_generic(plan->dtype, plan->P, plan->X);
    if (fuse && d->Mp > 0) {
      const int nb = d->wp_bstride != 0 ? B : 1;
      if (d->wp_step != 0 || plan->wph == nullptr || nb > plan->wph_nb) {
        fuse = false;
      } else {
        base.wph = plan->wph;
        base.wph_bs = d->wp_bstride != 0 ? 4LL * plan->P : 0;
        cudaError_t e = launch_pweight_dft(d->wp, d->wp_bstride, d->Mp, plan->P, nb, plan->wph, 4LL * plan->P,
                                           plan->dtype, st);
        if (e != cudaSuccess) return cuda_fail(e, "weight spectrum launch");
        ++g_launches;
      }
    }
    PassArgs a = base;  // opening V/2 of step 0
    a.tab1 = tabV(0);
    a.g1 = gV(0);
    a.scale_const = d->in_scale;
    if ((rc = col(a)) != FW_OK) return rc;
    for (int k = 0; k < steps; ++k) {
      PassArgs r = base;
      r.tab1 = tabK(k);
      r.g1 = gK(k);
      if (k > 0) prev_args(r, k - 1);
      if ((rc = row(r)) != FW_OK) return rc;
      PassArgs c = base;
      c.tab1 = tabV(k);
      c.g1 = gV(k);
      c.bxp = d->bxp;
      c.bxp_bs = d->bxp_bstride;
      obs_args(c, k);
      if (k + 1 < steps) {
        c.tab2 = tabV(k + 1);
        c.g2 = gV(k + 1);
        c.fuse_mid = fuse ? 1 : 0;
        // a column pair's two table entries load as one vector when both
        // tables start on 16 bytes and the instance stride keeps pairs aligned
        auto a16 = [](const void* t) { return (reinterpret_cast<uintptr_t>(t) & 15) == 0; };
        c.tab_vec = (d->tab_bstride % 2 == 0 && a16(c.tab1) && a16(c.tab2)) ? 1 : 0;
      }
      if ((rc = col(c)) != FW_OK) return rc;
    }
  } else {
    for (int k = 0; k < steps; ++k) {
      PassArgs c1 = base;
      c1.tab1 = tabV(k);
      c1.g1 = gV(k);
      c1.blend_pre = 1;
      if (k > 0) prev_args(c1, k - 1);
      else c1.scale_const = d->in_scale;
      if ((rc = col(c1)) != FW_OK) return rc;
      PassArgs r = base;
      r.tab1 = tabK(k);
      r.g1 = gK(k);
      if ((rc = row(r)) != FW_OK) return rc;
      PassArgs c2 = base;
      c2.tab1 = tabV(k);
      c2.g1 = gV(k);
      c2.bxp = d->bxp;
      c2.bxp_bs = d->bxp_bstride;
      c2.blend_post = 1;
      obs_args(c2, k);
      if ((rc = col(c2)) != FW_OK) return rc;
    }
  }
  PassArgs f = base;
  prev_args(f, steps - 1);
  cudaError_t e = launch_finalize(f, plan->dtype, st);
  if (e != cudaSuccess) return cuda_fail(e, "finalize launch");
  ++g_launches;
  if (g_timer) g_timer->mark(2);
  return FW_OK;
}

extern "C" int fw_wigner_propagate_timed(fw_wigner_plan* plan, const fw_wigner_desc* d, int steps, void* stream,
                                         float* ms_out, int* kind_out, int n_out) {
  if (ms_out == nullptr || kind_out == nullptr) return fail(FW_EINVAL, "fw_wigner_propagate_timed: NULL output");
  LaunchTimer t;
  t.st = static_cast<cudaStream_t>(stream);
  t.on = true;
  t.mark(-1);  // start marker
  g_timer = &t;
  int rc = fw_wigner_propagate(plan, d, steps, stream);
  g_timer = nullptr;
  cudaError_t e = cudaStreamSynchronize(t.st);
  if (rc == FW_OK && e != cudaSuccess) rc = cuda_fail(e, "fw_wigner_propagate_timed sync");
  const int n = (int)t.ev.size() - 1;
  if (rc == FW_OK && n > n_out) rc = fail(FW_EINVAL, "fw_wigner_propagate_timed: output arrays too small");
  for (int i = 0; rc == FW_OK && i < n; ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t.ev[i], t.ev[i + 1]);
    ms_out[i] = ms;
    kind_out[i] = t.kind[i + 1];
  }
  for (cudaEvent_t ev : t.ev) cudaEventDestroy(ev);
  return rc;
}

// ---------------------------------------------------------------------------
namespace fw {
template <typename Rl>
__global__ void weighted_sum_kernel(const Rl* W, long long w_bs, const double* F, size_t n, double* part) {
  const int b = blockIdx.y;
  const Rl* w = W + (size_t)b * w_bs;
  double s = 0.0, s2 = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = (double)w[i];
    s += F ? v * F[i] : v;
    s2 += v * v;
  }
  __shared__ double r1[32], r2[32];
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) { r1[threadIdx.x >> 5] = s; r2[threadIdx.x >> 5] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, c = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += r1[k]; c += r2[k]; }
    part[((size_t)b * gridDim.x + blockIdx.x) * 2 + 0] = a;
    part[((size_t)b * gridDim.x + blockIdx.x) * 2 + 1] = c;
  }
}
__global__ void sum_parts_kernel(const double* part, int nparts, double* out) {
  const int b = blockIdx.x;
  if (threadIdx.x < 2) {
    double a = 0;
    for (int k = 0; k < nparts; ++k) a += part[((size_t)b * nparts + k) * 2 + threadIdx.x];
    out[b * 2 + threadIdx.x] = a;
  }
}
}  // namespace fw

extern "C" int fw_wigner_weighted_sum(fw_wigner_plan* plan, const void* W, long long w_bstride, const double* F,
                                      double* out, void* stream) {
  if (plan == nullptr || W == nullptr || out == nullptr) return fail(FW_EINVAL, "fw_wigner_weighted_sum: NULL argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t n = (size_t)plan->P * plan->X;
  dim3 grid(plan->wsum_blocks, plan->batch);
  if (plan->dtype == FW_F32)
    weighted_sum_kernel<float><<<grid, 256, 0, st>>>(static_cast<const float*>(W), w_bstride, F, n, plan->wsum);
  else
    weighted_sum_kernel<double><<<grid, 256, 0, st>>>(static_cast<const double*>(W), w_bstride, F, n, plan->wsum);
  sum_parts_kernel<<<plan->batch, 32, 0, st>>>(plan->wsum, plan->wsum_blocks, out);
  g_launches += 2;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "weighted sum launch");
  return FW_OK;
}

// ---------------------------------------------------------------------------
// Propagation without device allocation.
//
// Some callers cannot call cudaMalloc: a host program that gives this library
// only buffers carved from its own fixed device-memory pool (instrument or
// real-time control loops that size all GPU memory once at start-up), or a
// loop that must not hit the implicit device-wide synchronisation of
// cudaMalloc / cudaFree between propagation calls.  For them,
// fw_wigner_propagate_noalloc runs the same passes as fw_wigner_propagate
// with the plan scratch (twiddle tables, the partial-sum ring, the
// per-instance totals and the p-weight spectra) placed in the fixed array
// below instead of plan allocations.
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;  // 4 MiB per device, held until process exit
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
// device address of g_noalloc_scratch per device, looked up once per device
static unsigned char* g_noalloc_ptr[kMaxDevices] = {};
static PerDeviceOnce g_noalloc_once;

__global__ void noalloc_twiddles_kernel(int n, int dtype, void* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double s, c;
  sincospi(-2.0 * (double)k / (double)n, &s, &c);
  if (dtype == FW_F64) {
    reinterpret_cast<double*>(out)[2 * k] = c;
    reinterpret_cast<double*>(out)[2 * k + 1] = s;
  } else {
    reinterpret_cast<float*>(out)[2 * k] = (float)c;
    reinterpret_cast<float*>(out)[2 * k + 1] = (float)s;
  }
}

// Stage-layout table (fft.cuh, stage_off) of an n-point transform with rv
// values per thread, gathered from the k-indexed table tw; total entries.
__global__ void noalloc_stage_kernel(int n, int rv, int dtype, const void* tw, void* out, int total) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int ns = rv, off = 0, R = rv;
  for (;;) {  // i < total bounds the walk over the stages
    R = n / ns >= rv ? rv : n / ns;
    const int sz = (R - 1) * ns;
    if (i < off + sz) break;
    off += sz;
    ns *= rv;
  }
  const int r = (i - off) / ns + 1, bm = (i - off) % ns;
  const int k = bm * r * (n / (ns * R));
  if (dtype == FW_F64) reinterpret_cast<double2*>(out)[i] = reinterpret_cast<const double2*>(tw)[k];
  else reinterpret_cast<float2*>(out)[i] = reinterpret_cast<const float2*>(tw)[k];
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Byte offsets of the no-allocation scratch regions of one call, in the
// order they sit in the array, each starting on 256 bytes.
struct NoAllocLayout {
  int small, np, rvX, nsX, wph_nb;
  size_t twP, twX, twsX, ring, tot, wph, need;
};

// Layout for a call with these sizes and descriptor; returns FW_OK or an
// FW_EINVAL message (sizes the plan entry point would also reject).
int noalloc_layout(int P, int X, int batch, int dtype, const fw_wigner_desc* d, NoAllocLayout* L) {
  if (dtype != FW_F32 && dtype != FW_F64) return fail(FW_EINVAL, "fw_wigner_propagate_noalloc: bad dtype");
  if (!size_supported(P) || !size_supported(X))
    return fail(FW_EINVAL, "fw_wigner_propagate_noalloc: P and X must be even and in [4, 4096]");
  if (batch < 1 || batch > 65535) return fail(FW_EINVAL, "fw_wigner_propagate_noalloc: batch must be in [1, 65535]");
  L->small = small_shapes(dtype, P, X, batch);
  L->np = col_parts(dtype, P, X, L->small);
  if (L->np <= 0) return fail(FW_EINVAL, "fw_wigner_propagate_noalloc: unsupported X for the column pass tile");
  const size_t rs = dtype == FW_F64 ? sizeof(double) : sizeof(float);
  L->rvX = row_rv(dtype, X, L->small);
  L->nsX = stage_off(X, L->rvX, X);
  // p-weight spectra (fused mid-point column pass): shared or per-instance weights
  const bool pw = d != nullptr && d->Mp > 0;
  L->wph_nb = pw ? (d->wp_bstride != 0 ? batch : 1) : 0;
  size_t off = 0;
  L->twP = off;  off += align256(2 * rs * (size_t)P);
  L->twX = off;  off += align256(2 * rs * (size_t)X);
  L->twsX = off; off += align256(2 * rs * (size_t)(L->nsX > 0 ? L->nsX : 1));
  L->ring = off; off += align256(sizeof(double) * 2 * (size_t)batch * L->np * MMAX);
  L->tot = off;  off += align256(sizeof(double) * (size_t)batch * MMAX);
  L->wph = off;  off += align256((size_t)4 * P * 2 * rs * (size_t)L->wph_nb);
  L->need = off;
  return FW_OK;
}
}  // namespace

extern "C" size_t fw_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

extern "C" size_t fw_noalloc_scratch_needed(int P, int X, int batch, int dtype, const fw_wigner_desc* desc) {
  NoAllocLayout L;
  return noalloc_layout(P, X, batch, dtype, desc, &L) == FW_OK ? L.need : 0;
}

extern "C" int fw_wigner_propagate_noalloc(int P, int X, int batch, int dtype, const fw_wigner_desc* desc, int steps,
                                           void* stream) {
  if (desc == nullptr) return fail(FW_EINVAL, "fw_wigner_propagate_noalloc: NULL desc");
  NoAllocLayout L;
  int rc = noalloc_layout(P, X, batch, dtype, desc, &L);
  if (rc != FW_OK) return rc;
  if (L.need > kNoAllocScratchBytes)
    return fail(FW_EINVAL, "fw_wigner_propagate_noalloc: needs " + std::to_string(L.need) +
                               " bytes of scratch for this grid and batch, more than the fixed " +
                               std::to_string(kNoAllocScratchBytes) + " bytes; use fw_wigner_propagate");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(FW_EINVAL, "fw_wigner_propagate_noalloc: device index too large");
  // once per device, with that device current (thread-safe)
  e = g_noalloc_once.run([&] {
    void* p = nullptr;
    cudaError_t r = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (r == cudaSuccess) g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    return r;
  });
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
  unsigned char* base = g_noalloc_ptr[dev];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (steps > 0) {
    // every call rewrites the twiddles (earlier calls may have left other
    // sizes); the partial-sum ring, the totals and the weight spectra are
    // always written before they are read
    noalloc_twiddles_kernel<<<(P + 255) / 256, 256, 0, st>>>(P, dtype, base + L.twP);
    noalloc_twiddles_kernel<<<(X + 255) / 256, 256, 0, st>>>(X, dtype, base + L.twX);
    if (L.nsX > 0)
      noalloc_stage_kernel<<<(L.nsX + 255) / 256, 256, 0, st>>>(X, L.rvX, dtype, base + L.twX, base + L.twsX, L.nsX);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "noalloc twiddle launch");
    count_launch(2 + (L.nsX > 0));
  }
  fw_wigner_plan tmp;
  tmp.P = P;
  tmp.X = X;
  tmp.batch = batch;
  tmp.dtype = dtype;
  tmp.nparts = L.np;
  tmp.small = L.small;
  tmp.twP = base + L.twP;
  tmp.twX = base + L.twX;
  tmp.twsX = base + L.twsX;
  tmp.ring = reinterpret_cast<double*>(base + L.ring);
  tmp.tot = reinterpret_cast<double*>(base + L.tot);
  tmp.wph = L.wph_nb > 0 ? base + L.wph : nullptr;
  tmp.wph_nb = L.wph_nb;
  tmp.wsum = nullptr;
  tmp.wsum_blocks = 0;
  return fw_wigner_propagate(&tmp, desc, steps, stream);
}
