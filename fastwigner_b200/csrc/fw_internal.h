// Internal declarations shared by the CUDA translation units of libfastwigner.
#pragma once
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include "../../include/fastwigner.h"

namespace fw {
constexpr int kMaxDevices = 64;

// A set-up call made once per device and remembered (thread-safe): e.g. the
// dynamic shared-memory limit of one kernel, which is a per-device attribute.
// The first call on a device runs `fn` with that device current; later calls
// on it return the recorded result.  cudaDeviceReset does not clear the record.
struct PerDeviceOnce {
  std::once_flag flag[kMaxDevices];
  cudaError_t err[kMaxDevices] = {};
  template <class Fn> cudaError_t run(Fn&& fn) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::call_once(flag[dev], [&] { err[dev] = fn(); });
    return err[dev];
  }
};

// Raise a kernel's dynamic shared-memory limit to `smem` bytes, once per
// device and kernel (each call site keeps its own PerDeviceOnce).
template <typename K> cudaError_t set_smem_once(PerDeviceOnce& once, K kern, size_t smem) {
  return once.run([&] { return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); });
}

struct PassArgs;
cudaError_t launch_row(const PassArgs& a, int dtype, cudaStream_t st);
cudaError_t launch_col(const PassArgs& a, int dtype, cudaStream_t st, int* nparts);
cudaError_t launch_finalize(const PassArgs& a, int dtype, cudaStream_t st);
cudaError_t launch_pweight_dft(const double* wp, long long wp_bs, int Mp, int P, int nb, void* out, long long out_bs,
                               int dtype, cudaStream_t st);
int fno_status_read(int* out, int clear);
bool colp_eligible(const PassArgs& a, int dtype);
bool rowp_eligible(const PassArgs& a, int dtype);
cudaError_t launch_row_persist(const PassArgs& a, cudaStream_t st);
cudaError_t launch_col_persist(const PassArgs& a, cudaStream_t st, int* nparts);
cudaError_t launch_totals(const double* part, int nparts, int M, int batch, double* tot, double* hist,
                          cudaStream_t st);
int col_parts(int dtype, int P, int X, int small);
int row_rv(int dtype, int N, int small);
int small_shapes(int dtype, int P, int X, int batch);
// Wigner plans: any even size in [4, 4096]; the register-resident passes take
// the powers of two in [128, 4096], the others run the generic passes
bool size_supported(int n);
bool size_pow2_supported(int n);
bool col_generic(int dtype, int P, int X);
inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
cudaError_t launch_generic_row(const PassArgs& a, int dtype, cudaStream_t st);
cudaError_t launch_generic_col(const PassArgs& a, int dtype, cudaStream_t st, int* nparts);

void set_error(const std::string& msg);
void count_launch(long long n);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);
}  // namespace fw
