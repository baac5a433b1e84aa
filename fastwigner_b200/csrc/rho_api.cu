// C ABI for density-matrix plans (von Neumann / Bloch rho propagation and
// generic row/column passes).
#include <cuda_runtime.h>
#include <math.h>
#include <string>
#include <vector>
#include "fw_internal.h"

namespace fw {
struct Factor;
struct RhoArgs;
}
#include "rho_passes.cu"

using namespace fw;

struct fw_rho_plan {
  int N, batch, dtype;
  int nparts;           // row-pass CTAs per instance
  void* tw = nullptr;   // twiddles for length N
  double* ring = nullptr;
  int ring_M = 0;
};

namespace {
constexpr int RHO_MMAX = 4 + 4 * RMAXO;

int upload_tw(int n, int dtype, void** dev) {
  std::vector<double> t(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    t[2 * k] = cos(a);
    t[2 * k + 1] = sin(a);
  }
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

Factor to_factor(const fw_rho_factor* f) {
  Factor r{};
  if (f == nullptr || !f->on) return r;
  r.on = 1;
  r.s_re = f->s_re;
  r.s_im = f->s_im;
  r.u = f->u;
  r.w = f->w;
  r.tab = f->tab;
  r.tab_bs = f->tab_bstride;
  r.shear_c = f->shear_c;
  r.shear_a = f->shear_a;
  r.shear_b = f->shear_b;
  r.sign = f->sign;
  return r;
}
}  // namespace

extern "C" int fw_rho_plan_create(int N, int batch, int dtype, fw_rho_plan** out) {
  if (out == nullptr) return fail(FW_EINVAL, "fw_rho_plan_create: out is NULL");
  *out = nullptr;
  if (dtype != FW_F32 && dtype != FW_F64) return fail(FW_EINVAL, "fw_rho_plan_create: bad dtype");
  if (!size_pow2_supported(N))
    return fail(FW_EINVAL, "fw_rho_plan_create: X_gridDIM must be a power of two in [128, 4096] (got " +
                               std::to_string(N) + ")");
  if (batch < 1 || batch > 65535) return fail(FW_EINVAL, "fw_rho_plan_create: batch must be in [1, 65535]");
  fw_rho_plan* p = new fw_rho_plan();
  p->N = N;
  p->batch = batch;
  p->dtype = dtype;
  p->nparts = rho_row_parts(dtype, N);
  int rc = upload_tw(N, dtype, &p->tw);
  if (rc == FW_OK) {
    cudaError_t e = cudaMalloc(&p->ring, sizeof(double) * 2 * (size_t)batch * p->nparts * RHO_MMAX);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc(partials)");
  }
  if (rc != FW_OK) {
    fw_rho_plan_destroy(p);
    return rc;
  }
  *out = p;
  return FW_OK;
}

extern "C" int fw_rho_plan_destroy(fw_rho_plan* p) {
  if (p == nullptr) return FW_OK;
  cudaFree(p->tw);
  cudaFree(p->ring);
  delete p;
  return FW_OK;
}

extern "C" int fw_rho_num_parts(const fw_rho_plan* p) { return p == nullptr ? -1 : p->nparts; }

extern "C" int fw_rho_pass(fw_rho_plan* p, void* R, long long r_bstride, int axis, const fw_rho_factor* f0, int t1,
                           const fw_rho_factor* f1, const fw_rho_factor* f2, int t2, const fw_rho_factor* f3,
                           double* part_out, double* sum_out, void* stream) {
  if (p == nullptr || R == nullptr) return fail(FW_EINVAL, "fw_rho_pass: NULL plan or state");
  if (axis != 0 && axis != 1) return fail(FW_EINVAL, "fw_rho_pass: axis must be 0 (columns) or 1 (rows)");
  if (axis == 0 && (part_out != nullptr || sum_out != nullptr))
    return fail(FW_EINVAL, "fw_rho_pass: reductions are available on row passes only");
  RhoArgs a{};
  a.R = R;
  a.r_bs = r_bstride;
  a.N = p->N;
  a.batch = p->batch;
  a.dX = 1.0;
  a.dP = 1.0;
  a.f0 = to_factor(f0);
  a.f1 = to_factor(f1);
  a.f2 = to_factor(f2);
  a.f3 = to_factor(f3);
  a.t1 = t1 < 0 ? -1 : (t1 > 0 ? 1 : 0);
  a.t2 = t2 < 0 ? -1 : (t2 > 0 ? 1 : 0);
  a.M = 4;
  a.part_out = part_out;
  a.sum_out = sum_out;
  a.tw = p->tw;
  for (const fw_rho_factor* f : {f0, f1, f2, f3})
    if (f && f->on && f->shear_c != 0.0) { a.dX = f->shear_dx; a.dP = f->shear_dp; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = axis == 1 ? launch_rho_row(a, p->dtype, st, nullptr) : launch_rho_col(a, p->dtype, st);
  if (e != cudaSuccess) return cuda_fail(e, "fw_rho_pass launch");
  count_launch(1);
  return FW_OK;
}

extern "C" int fw_rho_propagate(fw_rho_plan* p, const fw_rho_desc* d, int steps, void* stream) {
  if (p == nullptr || d == nullptr) return fail(FW_EINVAL, "fw_rho_propagate: NULL plan or desc");
  if (steps < 0) return fail(FW_EINVAL, "fw_rho_propagate: steps must be >= 0");
  if (steps == 0) return FW_OK;
  if (d->R == nullptr || d->uV == nullptr || d->wV == nullptr || d->uK == nullptr || d->wK == nullptr)
    return fail(FW_EINVAL, "fw_rho_propagate: R and the four phase vectors are required");
  if (d->Mx < 0 || d->Mx > RMAXO || d->Mp < 0 || d->Mp > RMAXO)
    return fail(FW_EINVAL, "fw_rho_propagate: Mx, Mp must be in [0, 4]");
  if ((d->Mx > 0 && d->wx == nullptr) || (d->Mp > 0 && d->gp == nullptr))
    return fail(FW_EINVAL, "fw_rho_propagate: observable weights missing");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t cs = (p->dtype == FW_F64 ? 16 : 8);  // bytes per complex
  const int N = p->N, B = p->batch;
  const int M = 4 + 2 * d->Mx + 2 * d->Mp;
  const size_t slot = (size_t)B * p->nparts * M;
  auto vec = [&](const void* base, long long step, int k) -> const void* {
    return static_cast<const char*>(base) + (size_t)k * (size_t)step * cs;
  };
  auto ring = [&](int k) { return p->ring + (size_t)(k & 1) * slot; };
  auto hist = [&](int k) { return d->obs_out == nullptr ? nullptr : d->obs_out + (size_t)k * B * M; };
  auto expV = [&](int k, double s) {
    Factor f{};
    f.on = 1;
    f.s_re = s;
    f.u = vec(d->uV, d->V_step, k);
    f.w = vec(d->wV, d->V_step, k);
    f.tab = d->bx;
    f.tab_bs = d->b_bstride;
    return f;
  };
  auto expK = [&](int k, double s) {
    Factor f{};
    f.on = 1;
    f.s_re = s;
    f.u = vec(d->uK, d->K_step, k);
    f.w = vec(d->wK, d->K_step, k);
    f.tab = d->bp;
    f.tab_bs = d->b_bstride;
    return f;
  };
  RhoArgs base{};
  base.R = d->R;
  base.r_bs = d->r_bstride;
  base.N = N;
  base.batch = B;
  base.dX = d->dX;
  base.dP = 1.0;
  base.M = M;
  base.Mx = d->Mx;
  base.Mp = d->Mp;
  base.tw = p->tw;
  const double invN = 1.0 / (double)N;
  int np = 0;
  auto row = [&](RhoArgs a) -> int {
    cudaError_t e = launch_rho_row(a, p->dtype, st, &np);
    if (e != cudaSuccess) return cuda_fail(e, "rho row pass launch");
    count_launch(1);
    return FW_OK;
  };
  auto col = [&](RhoArgs a) -> int {
    cudaError_t e = launch_rho_col(a, p->dtype, st);
    if (e != cudaSuccess) return cuda_fail(e, "rho column pass launch");
    count_launch(1);
    return FW_OK;
  };
  int rc;
  {
    RhoArgs a = base;  // opening expV of step 0, then FFT along x
    a.f1 = expV(0, 1.0);
    a.t2 = -1;
    if ((rc = row(a)) != FW_OK) return rc;
  }
  for (int k = 0; k < steps; ++k) {
    RhoArgs c = base;
    c.t1 = -1;
    c.f1 = expK(k, invN);
    c.t2 = +1;
    if (k > 0) {
      c.prev_part = ring(k - 1);
      c.prev_nparts = p->nparts;
      c.obs_hist = hist(k - 1);
    }
    if ((rc = col(c)) != FW_OK) return rc;
    RhoArgs r = base;
    r.t1 = +1;
    r.f1 = expV(k, invN);
    r.part_out = ring(k);
    r.wx = d->wx == nullptr ? nullptr : d->wx + (size_t)k * d->wx_step;
    r.gp = d->gp == nullptr ? nullptr : d->gp + (size_t)k * d->gp_step;
    if (k + 1 < steps) {
      r.f2 = expV(k + 1, 1.0);
      r.t2 = -1;
    }
    if ((rc = row(r)) != FW_OK) return rc;
  }
  RhoArgs f = base;  // final normalisation
  f.prev_part = ring(steps - 1);
  f.prev_nparts = p->nparts;
  f.obs_hist = hist(steps - 1);
  return row(f);
}
