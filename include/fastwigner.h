/*
 * fastwigner.h -- C ABI of libfastwigner (B200 / sm_100a split-operator
 * propagators for phase-space quantum dynamics).
 *
 * Plain C: opaque handles, raw device pointers, sizes and an int status
 * (0 = success; otherwise fw_last_error() holds a message).  Device pointers
 * are caller-owned (the Python layer passes torch CUDA tensor storage); the
 * library owns only its plan scratch (twiddle tables, partial-sum rings).
 * All work is enqueued on the caller's stream (cudaStream_t passed as void*,
 * NULL = legacy default stream).  A handle must not be used from two host
 * threads at once.
 *
 * Reference interfaces replaced (dibondar/FastWigner, paths within that project):
 *   - cuFFT ctypes binding + plans  cufft.py:105-342
 *   - WignerMoyalCUDA1D.single_step_propagation / propagate
 *                                   wigner_moyal_cuda_1d.py:496-540
 *   - WignerMoyalFTTW1D.single_step_propagation / propagate
 *                                   wigner_moyal_fftw_1d.py:397-440
 *   - WignerBlochCUDA1D.bloch_single_step_propagation
 *                                   wigner_bloch_cuda_1d.py:229-254
 *   - WignerRandomCollisionModelFFTW1D.single_step_propagation
 *                                   wigner_random_collision_model_fftw_1d.py:56-76
 */
#ifndef FASTWIGNER_H
#define FASTWIGNER_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FW_ABI_VERSION 1

/* element types of the state buffers */
#define FW_F32 0 /* float state, complex64 spectra (FP64 phase arguments) */
#define FW_F64 1 /* double state, complex128 spectra */

/* status codes */
#define FW_OK 0
#define FW_EINVAL 1   /* bad argument (size, null pointer, unsupported grid) */
#define FW_ECUDA 2    /* a CUDA runtime call failed */
#define FW_ENVRTC 3   /* run-time compilation of a user expression failed */
#define FW_ESTATE 4   /* handle in the wrong state */

/* device status words: of a batched launch (fw_batch_status) and of a plan (fw_wigner_plan_status) */
#define FW_BATCH_TIMEOUT 1  /* a grid barrier gave up waiting; the launch returned early */
#define FW_PASS_TIMEOUT 2   /* a pass's bulk copy into shared memory did not complete; its CTA returned early */
#define FW_FNO_TIMEOUT 3    /* a tensor-core GEMM of the FNO gave up waiting for its MMAs; its output is invalid (NaN where it stopped) */

/* step structure of fw_wigner_propagate */
#define FW_STEP_FUSED 0 /* V/2 K V/2 with the closing V/2 of step n fused with the
                           opening V/2 of step n+1 (Moyal, Bloch): 2 passes/step */
#define FW_STEP_SPLIT 1 /* blend V/2 K V/2 blend (random-collision model): 3 passes/step */

/* Library version of this header; fw_abi_version() must return it. */
int fw_abi_version(void);

/* Message of the last failed call on this host thread ("" if none). */
const char* fw_last_error(void);

/* ------------------------------------------------------------------------ */
/* Wigner-function (real P x X grid) split-operator plans                    */
/* ------------------------------------------------------------------------ */

typedef struct fw_wigner_plan fw_wigner_plan;

/*
 * Create a plan for `batch` Wigner functions of P x X points (p rows, x
 * fastest) in precision `dtype` (FW_F32 / FW_F64).  P and X must be powers of
 * two in [128, 4096].  Replaces the four cuFFT D2Z/Z2D axis plans and the
 * aliased theta-x / p-lambda buffers of WignerMoyalCUDA1D.__init__
 * (wigner_moyal_cuda_1d.py:285-339, cufft.py:160-213) and the pyFFTW plans of
 * WignerMoyalFTTW1D.__init__ (wigner_moyal_fftw_1d.py:303-366): the spectra
 * never leave the chip, so no spectrum buffer exists.
 */
int fw_wigner_plan_create(int P, int X, int batch, int dtype, fw_wigner_plan** out);
int fw_wigner_plan_destroy(fw_wigner_plan* plan);

/*
 * Synchronous read of the plan's device status word (0, or FW_PASS_TIMEOUT
 * when a pass gave up waiting for a bulk copy and its results are incomplete);
 * clear != 0 resets it to 0 afterwards.  No reference counterpart (the
 * reference's cuFFT calls report errors through their return status,
 * cufft.py:95-102).
 */
int fw_wigner_plan_status(fw_wigner_plan* plan, int* status_out, int clear);

/* Number of per-step observables (M) the plan writes for Mx x-weights and Mp p-weights: 2 + Mx + Mp.
 * Observable slots per instance and step: [sum W, sum W^2, sum W*wx_0(x) .., sum W*wp_0(p) ..]
 * (sums over the grid of the un-normalised state; ratios give normalised averages). */
int fw_wigner_num_obs(int Mx, int Mp);

typedef struct fw_wigner_desc {
  void* W;                  /* device state, batch x P x X */
  long long w_bstride;      /* elements between instances */
  int step_kind;            /* FW_STEP_FUSED or FW_STEP_SPLIT */
  /* phase tables, device; complex (re,im interleaved) unless tab_real:
     tabV: (P/2+1) x X half spectrum over (theta, x); tabK: P x (X/2+1) over (p, lambda).
     Table for step k is base + k * *_step elements; tab_bstride between instances. */
  const void* tabV;
  long long tabV_step;
  const void* tabK;
  long long tabK_step;
  long long tab_bstride;
  int tab_real;             /* 1: real exponent tables (Bloch) */
  /* optional separable per-step factors, complex, gV: P/2+1 over theta, gK: X/2+1 over lambda */
  const void* gV;
  long long gV_step;
  const void* gK;
  long long gK_step;
  /* optional real P x X multiplier applied after every step (abs_boundary_x_p) */
  const void* bxp;
  long long bxp_bstride;
  /* FW_STEP_SPLIT: W <- blend_c * W + s0 before and after every step */
  const void* s0;
  long long s0_bstride;
  double blend_c;
  /* observables: Mx x-weights (Mx x X doubles), Mp p-weights (Mp x P doubles); Mx, Mp <= 4 */
  int Mx;
  int Mp;
  const double* wx;
  long long wx_step;
  long long wx_bstride;
  const double* wp;
  long long wp_step;
  long long wp_bstride;
  double* obs_out;          /* device, steps x batch x M doubles (may be NULL: no history kept) */
  double dxdp;              /* phase-space cell, for the normalisation sum(W) dX dP = 1 */
  double in_scale;          /* factor applied to W on the first load (1.0) */
} fw_wigner_desc;

/*
 * Advance every instance by `steps` split-operator steps, renormalising after
 * each step and recording the per-step observable sums in obs_out.  All work
 * is enqueued on `stream`; no host synchronisation.  Replaces propagate()
 * of wigner_moyal_cuda_1d.py:521-540 / wigner_moyal_fftw_1d.py:418-440 and the
 * Bloch step loop of wigner_bloch_cuda_1d.py:129-165.
 */
int fw_wigner_propagate(fw_wigner_plan* plan, const fw_wigner_desc* desc, int steps, void* stream);

/*
 * fw_wigner_propagate, additionally timing every kernel launch with CUDA
 * events on `stream`; blocks until the work is done.  ms_out receives
 * 2*steps+2 (FW_STEP_FUSED) or 3*steps+1 (FW_STEP_SPLIT) per-launch durations
 * in milliseconds and kind_out the pass kind of each launch (0 column, 1 row,
 * 2 finalize).  n_out is the capacity of both arrays.  A profiling helper; no
 * reference counterpart.
 */
int fw_wigner_propagate_timed(fw_wigner_plan* plan, const fw_wigner_desc* desc, int steps, void* stream,
                              float* ms_out, int* kind_out, int n_out);

/* Number of kernels this library has launched in the process so far. */
long long fw_launch_count(void);

/*
 * fw_wigner_propagate for callers that cannot allocate device memory: no
 * counterpart in the reference.  Some hosts cannot call cudaMalloc -- a program
 * that hands this library only buffers from its own fixed device-memory pool
 * (instrument or real-time control loops that size all GPU memory at start-up),
 * or a loop that must not hit the device-wide synchronisation of cudaMalloc /
 * cudaFree between calls.  This entry point takes no plan and allocates
 * nothing: its scratch (twiddle tables, partial sums, per-instance totals and
 * the spectra of the p-observable weights) lives in a fixed array of
 * fw_noalloc_scratch_bytes() (4 MiB) that every GPU loading the library holds
 * until exit, and it runs the same passes as fw_wigner_propagate with a plan
 * of the same sizes.  A call whose scratch (fw_noalloc_scratch_needed) exceeds
 * the array is rejected with FW_EINVAL.  The first call on a device looks up
 * the array's device address (thread-safe, once per device; make that first
 * call before any stream capture; after cudaDeviceReset the recorded address
 * is stale, so a process that resets a device must not call this entry point
 * on it again).  All calls share the array: calls that overlap on the GPU
 * (other streams, other host threads) race and must be serialised by the
 * caller.  The caller still owns W, the tables, weights and obs_out exactly
 * as for fw_wigner_propagate.
 */
int fw_wigner_propagate_noalloc(int P, int X, int batch, int dtype, const fw_wigner_desc* desc, int steps,
                                void* stream);

/* Size in bytes of the fixed scratch array used by fw_wigner_propagate_noalloc. */
size_t fw_noalloc_scratch_bytes(void);

/*
 * Bytes of that array a fw_wigner_propagate_noalloc call with these sizes and
 * descriptor needs (only desc->Mp and desc->wp_bstride matter; desc may be
 * NULL for no p-observables): the twiddle tables of P and X, the row pass's
 * stage-layout table, 2 x batch x (column tiles per instance) x 10 partial
 * sums, batch x 10 totals and, with p-observables, 4 x P weight spectra per
 * weight set, each region rounded up to 256 bytes.  0 for invalid sizes.
 */
size_t fw_noalloc_scratch_needed(int P, int X, int batch, int dtype, const fw_wigner_desc* desc);

/*
 * out[b*2+0] = sum_{p,x} W[b] * F (F = NULL means F = 1), out[b*2+1] = sum W^2, in FP64.
 * F is a device P x X double array shared by the batch.  Replaces the
 * weighted_func kernel + gpuarray.sum of get_average and the gpuarray.dot of
 * get_purity (wigner_moyal_cuda_1d.py:378-403).  `out` is device memory.
 */
int fw_wigner_weighted_sum(fw_wigner_plan* plan, const void* W, long long w_bstride, const double* F, double* out,
                           void* stream);

/* ------------------------------------------------------------------------ */
/* Density-matrix plans: rho[b][i][j] = <x'_i| rho |x_j>, complex N x N       */
/* ------------------------------------------------------------------------ */

typedef struct fw_rho_plan fw_rho_plan;

/*
 * Plan for `batch` complex N x N density matrices (complex64 for FW_F32,
 * complex128 for FW_F64), N a power of two in [128, 4096].  Replaces the
 * cuFFT Z2Z plans of RhoVNeumannCUDA1D (rho_vneumann_cuda_1d.py:212, :238-239;
 * cufft.py:241-342).
 */
int fw_rho_plan_create(int N, int batch, int dtype, fw_rho_plan** out);
int fw_rho_plan_destroy(fw_rho_plan* plan);
/* Row-pass partial records per instance (the length of part_out / N for fw_rho_pass). */
int fw_rho_num_parts(const fw_rho_plan* plan);

/* Element-wise factor f(i, j) = s * u[j] * w[i] * tab[i][j] * exp(i shear_c A(j) B(i)) * (-1)^(i sign),
 * A, B grid coordinates (0: x = shear_dx (k - N/2), 1: p = shear_dp ((k + N/2) mod N - N/2)). */
typedef struct fw_rho_factor {
  int on;
  double s_re, s_im;
  const void* u;            /* complex N (state precision), over j; NULL = 1 */
  const void* w;            /* complex N, over i; NULL = 1 */
  const void* tab;          /* real N x N (state precision); NULL = 1 */
  long long tab_bstride;
  double shear_c;           /* 0: no shear factor */
  int shear_a, shear_b;
  double shear_dx, shear_dp;
  int sign;
} fw_rho_factor;

/*
 * One pass over rows (axis 1: transforms along j) or columns (axis 0: along i):
 * F0 -> T1 -> F1 -> F2 -> T2 -> F3, T = 0 none, -1 forward FFT, +1 unnormalised
 * inverse FFT.  Row passes may also write per-CTA partials part_out[b][c][4] =
 * [Re tr, Im tr, sum |rho|^2, 0] of the state after F1, and sum_out[b][c][2] =
 * complex sum of all elements after F3 (device arrays, fw_rho_num_parts records
 * per instance).  Replaces the observable, shear and sign-flip kernels with their
 * axis FFTs (rho_vneumann_cuda_1d.py:431-472, :502-592, :710-800).
 */
int fw_rho_pass(fw_rho_plan* plan, void* R, long long r_bstride, int axis, const fw_rho_factor* f0, int t1,
                const fw_rho_factor* f1, const fw_rho_factor* f2, int t2, const fw_rho_factor* f3, double* part_out,
                double* sum_out, void* stream);

typedef struct fw_rho_desc {
  void* R;                  /* device states, batch x N x N complex */
  long long r_bstride;      /* complex elements between instances */
  /* exp(V) in the x-representation: factor u[j] w[i] (vN: u = exp(-i dt V(x)/2), w = conj(u);
     Bloch: u = w = exp(-dbeta (V - V_min/2)/4)); step k uses base + k * V_step complex elements */
  const void* uV;
  const void* wV;
  long long V_step;
  /* exp(K) in the (fft-ordered) momentum representation, same structure */
  const void* uK;
  const void* wK;
  long long K_step;
  const void* bx;           /* optional real N x N factor with every exp(V) (abs_boundary_x) */
  const void* bp;           /* optional real N x N factor with every exp(K) (abs_boundary_p) */
  long long b_bstride;
  /* observables: Mx diagonal x-weights (Mx x N doubles) -> Tr[rho f(x)];
     Mp Toeplitz kernels G = ifft(g(p)) (Mp x N complex doubles) -> Tr[rho g(p)];
     wx_step and gp_step count doubles */
  int Mx;
  int Mp;
  const double* wx;
  long long wx_step;
  const double* gp;
  long long gp_step;
  double* obs_out;          /* steps x batch x M doubles, M = 4 + 2 Mx + 2 Mp:
                               [Re tr, Im tr, sum|rho|^2, 0, (Re, Im) of each x- then p-observable] */
  double dX;
} fw_rho_desc;

/*
 * Advance every density matrix by `steps` split-operator steps
 * (exp(V) -> FFT2 -> exp(K) -> iFFT2 -> exp(V), then rho /= Tr(rho) dX), two
 * fused passes per step, observables recorded per step.  Replaces
 * RhoVNeumannCUDA1D.single_step_propagation / propagate
 * (rho_vneumann_cuda_1d.py:340-374) and RhoBlochCUDA1D.bloch_single_step_propagation
 * (rho_bloch_cuda_1d.py:224-241).
 */
int fw_rho_propagate(fw_rho_plan* plan, const fw_rho_desc* desc, int steps, void* stream);

/* ------------------------------------------------------------------------ */
/* Persistent batched propagation over instances with uneven grids (FP32)   */
/* ------------------------------------------------------------------------ */

typedef struct fw_batch fw_batch;

/*
 * A batch of `ninst` independent FP32 Wigner functions, instance i on a
 * P[i] x X[i] grid with P, X in {128, 256, 512, 1024}.  fw_batch_propagate
 * advances all of them with ONE cooperative (persistent) launch: phases of
 * row / column passes separated by bounded software grid barriers, work items
 * (instance, tile) pulled from atomic queues and run with the tile code of each
 * instance's size.  `variant` selects the launch shape (fw_batch_num_variants();
 * chosen by the Python autotuner).  No reference counterpart (the reference runs
 * one instance per class, wigner_moyal_cuda_1d.py:521-540).
 */
int fw_batch_create(int ninst, const int* P, const int* X, int variant, fw_batch** out);
int fw_batch_destroy(fw_batch* batch);
int fw_batch_num_variants(void);
int fw_batch_set_variant(fw_batch* batch, int variant);
/* State W (P x X floats), complex64 tables tabV ((P/2+1) x X) and tabK (P x (X/2+1)) of instance i. */
int fw_batch_set_instance(fw_batch* batch, int i, void* W, const void* tabV, const void* tabK, double dxdp);
/*
 * Advance every instance by `steps` steps (Moyal/Bloch split operator with
 * per-step renormalisation); obs (device, may be NULL) receives steps x ninst x 2
 * doubles [sum W, sum W^2].  use_graph != 0 replays a CUDA graph of the launch
 * (captured on first use for this (steps, obs)).
 */
int fw_batch_propagate(fw_batch* batch, int steps, double* obs, int use_graph, void* stream);
/* Synchronous read of the device status word (0 or FW_BATCH_TIMEOUT). */
int fw_batch_status(fw_batch* batch, int* status_out);
/*
 * Synchronous write of the device status word.  0 clears a recorded timeout
 * so that the batch can run again; a non-zero value makes the next launch
 * return at its first grid barrier (every CTA reads the word there).  The
 * status word is this build's failure detection for the persistent launch;
 * the reference has no counterpart (its only recovery is the Bloch roll-back,
 * wigner_bloch_cuda_1d.py:188-225).
 */
int fw_batch_set_status(fw_batch* batch, int status);
/*
 * Polls (each followed by a 64 ns sleep) that a CTA waits at a grid barrier
 * before it records FW_BATCH_TIMEOUT and the launch returns; default 2^25
 * (a few seconds).  0 makes any CTA that has to wait give up at once.
 * Changing the limit drops a captured graph of the launch.
 */
int fw_batch_set_spin_limit(fw_batch* batch, long long polls);

/* ------------------------------------------------------------------------ */
/* Fourier-neural-operator surrogate kernels (training and inference, FP32)  */
/* No reference counterpart: the surrogate seeds the Bloch thermal-state      */
/* computation (wigner_bloch_cuda_1d.py:129-165).                             */
/* ------------------------------------------------------------------------ */

/* C[b] = alpha op(A[b]) op(B[b]) + beta C[b]; op(A) M x K, op(B) K x N, row-major,
 * leading dimensions lda/ldb/ldc, batch strides strideA/B/C (elements), batch <= 65535,
 * sizes <= 2^30.  Runs on the tensor cores (tcgen05 MMAs in TF32 with a three-way split
 * that keeps FP32 products).  Outputs up to 32 wide on the tensor core's short side
 * (min(M, N) <= 32) sum 32-wide K chunks in registers with round-to-nearest adds; wider
 * ones accumulate in tensor memory, whose truncating FP32 adds leave an error growing
 * with K (about 3e-5 of max |C| at K = 4096 for random operands). */
int fw_fno_sgemm(int transA, int transB, int M, int N, int K, float alpha, const float* A, long long lda,
                 long long strideA, const float* B, long long ldb, long long strideB, float beta, float* C,
                 long long ldc, long long strideC, int batch, void* stream);
/* The same product with a fused epilogue: t = alpha op(A) op(B) + beta C + bias[m]
 * (bias may be NULL; C may be NULL when beta == 0); pre = t when pre != NULL;
 * out = t (act 0), GELU(t) (act 1) or t GELU'(aux) (act 2).  pre, aux and out share
 * C's layout (ldc, strideC); out may be C itself. */
int fw_fno_sgemm_ex(int transA, int transB, int M, int N, int K, float alpha, const float* A, long long lda,
                    long long strideA, const float* B, long long ldb, long long strideB, float beta, const float* C,
                    long long ldc, long long strideC, int batch, const float* bias, float* pre, const float* aux,
                    int act, float* out, void* stream);
/* Weight gradient out[r][c] (+)= sum_b sum_l dY[b][r][l] X[b][c][l] (dY: rows x L per
 * sample, X: cols x L, batch strides strideY / strideX) as a split-K tensor-core product
 * into `work` and an FP64 sum of the slices; fw_fno_wgrad_work gives the floats `work`
 * must hold for these sizes. */
int fw_fno_wgrad_work(int rows, int cols, long long L, int batch, long long* floats_out);
int fw_fno_wgrad(int rows, int cols, long long L, const float* dY, long long strideY, const float* X,
                 long long strideX, int batch, float* work, long long work_floats, float* out, int accumulate,
                 void* stream);
/* Fused two-layer pointwise projection: out[b][l] = c2[0] + sum_j Q2[j] GELU(c1[j] +
 * sum_c Q1[j][c] V[b][c][l]) for j < hidden <= 128 (Q1: hidden x C); the hidden layer
 * stays in tensor memory. */
int fw_fno_project(int hidden, int C, long long L, const float* V, long long strideV, int batch, const float* Q1,
                   const float* c1, const float* Q2, const float* c2, float* out, long long strideOut, void* stream);
/* Synchronous read of the FNO status word (0 or FW_FNO_TIMEOUT); clear != 0 resets it. */
int fw_fno_status(int* status_out, int clear);
/* Per-mode complex channel mixing, [B][C][2][K] layouts (real block, imaginary block):
 * mode 0: out = sum_i X[b][i] Y[i][o]; mode 1: out[b][i] = sum_o X[b][o] conj(Y[i][o]);
 * mode 2: out[i][o] = sum_b conj(X[b][i]) Y[b][o]. */
int fw_fno_mix(int mode, int B, int Cin, int Cout, int K, const float* X, const float* Y, float* out, void* stream);
/* pre = X + bias[c] over [B][C][L]; Y = act ? GELU(pre) : pre (pre may be NULL). */
int fw_fno_bias_act(long long n, int C, long long L, const float* X, const float* bias, float* pre, float* Y, int act,
                    void* stream);
/* dpre = act ? dY GELU'(pre) : dY. */
int fw_fno_act_bwd(long long n, const float* dY, const float* pre, float* dpre, int act, void* stream);
/* out[c] (+)= sum over b, l of X[b][c][l] (FP64 accumulation). */
int fw_fno_channel_sum(int B, int C, long long L, const float* X, float* out, int accumulate, void* stream);
/* loss[b] = |Y_b - T_b|^2 / |T_b|^2 (doubles); dY = d(mean loss)/dY (may be NULL). */
int fw_fno_rel_l2(int B, long long L, const float* Y, const float* T, float* dY, double* loss, void* stream);
/* Adam with bias correction for step `step` (>= 1) and decoupled weight decay. */
int fw_fno_adam(long long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                int step, float weight_decay, void* stream);
/* Lift input [B][NP+2][G0][G1]: NP per-sample parameters broadcast, then xs[G1], ps[G0]. */
int fw_fno_features(int B, int NP, int G0, int G1, const float* params, const float* xs, const float* ps, float* out,
                    void* stream);

/* ------------------------------------------------------------------------ */
/* User C expressions (NVRTC)                                                */
/* ------------------------------------------------------------------------ */

typedef struct fw_expr fw_expr;

/*
 * Compile a CUDA C evaluation module with NVRTC for the current device and
 * load it.  Every kernel of the module has the C signature
 *   extern "C" __global__ void name(const double* in, long long n, double* re, double* im)
 * Replaces PyCUDA SourceModule compilation of the user strings V, K,
 * boundaries, initial states and observables (wigner_moyal_cuda_1d.py:250-277,
 * :389-391, :480-483; rho_vneumann_cuda_1d.py:196-204, :325-327, :425-427).
 */
int fw_expr_create(const char* source, fw_expr** out);
int fw_expr_destroy(fw_expr* mod);

/* Compile only (no device needed); the NVRTC log is copied to `log`. */
int fw_expr_check(const char* source, char* log, int log_len);

/* Launch kernel `name` over n points: in is 10 x n doubles (device), re/im n doubles each (im may be NULL). */
int fw_expr_eval(fw_expr* mod, const char* name, const double* in, long long n, double* out_re, double* out_im,
                 void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FASTWIGNER_H */
