// Run-time compilation of user C expressions (NVRTC -> CUBIN -> cudaLibrary).
//
// The reference's CUDA classes splice user strings (V, K, boundaries, initial
// states, observables) into CUDA C templates and compile them with PyCUDA's
// SourceModule (e.g. wigner_moyal_cuda_1d.py:250-277).  Here the Python layer
// generates an evaluation module (one extern "C" kernel per expression, all
// with the signature (const double* in, long long n, double* re, double* im))
// and this file compiles it for the current device and launches its kernels.
// The expression kernels only tabulate FP64 values (phase arguments,
// weights, initial states); the propagation itself runs in the precompiled
// pass kernels.
#include <cuda_runtime.h>
#include <nvrtc.h>
#include <string>
#include <vector>
#include "fw_internal.h"

using namespace fw;

struct fw_expr {
  cudaLibrary_t lib = nullptr;
  std::string log;
};

namespace {

int nvrtc_compile(const char* source, int arch_major, int arch_minor, std::vector<char>* cubin, std::string* log) {
  nvrtcProgram prog;
  nvrtcResult r = nvrtcCreateProgram(&prog, source, "fw_expr.cu", 0, nullptr, nullptr);
  if (r != NVRTC_SUCCESS) {
    *log = nvrtcGetErrorString(r);
    return FW_ENVRTC;
  }
  std::string arch = "--gpu-architecture=sm_" + std::to_string(arch_major * 10 + arch_minor);
  if (arch_major >= 9) arch += "a";
  const char* opts[] = {arch.c_str(), "-std=c++17", "--fmad=true"};
  r = nvrtcCompileProgram(prog, 3, opts);
  size_t ls = 0;
  nvrtcGetProgramLogSize(prog, &ls);
  log->assign(ls, '\0');
  if (ls) nvrtcGetProgramLog(prog, &(*log)[0]);
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    return FW_ENVRTC;
  }
  if (cubin != nullptr) {
    size_t cs = 0;
    nvrtcGetCUBINSize(prog, &cs);
    cubin->resize(cs);
    nvrtcGetCUBIN(prog, cubin->data());
  }
  nvrtcDestroyProgram(&prog);
  return FW_OK;
}

}  // namespace

extern "C" int fw_expr_check(const char* source, char* log, int log_len) {
  if (source == nullptr) return fail(FW_EINVAL, "fw_expr_check: NULL source");
  std::string lg;
  int rc = nvrtc_compile(source, 10, 0, nullptr, &lg);
  if (log != nullptr && log_len > 0) {
    const size_t n = lg.size() < (size_t)(log_len - 1) ? lg.size() : (size_t)(log_len - 1);
    for (size_t i = 0; i < n; ++i) log[i] = lg[i];
    log[n] = '\0';
  }
  if (rc != FW_OK) return fail(rc, "NVRTC compilation failed:\n" + lg);
  return FW_OK;
}

extern "C" int fw_expr_create(const char* source, fw_expr** out) {
  if (source == nullptr || out == nullptr) return fail(FW_EINVAL, "fw_expr_create: NULL argument");
  *out = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
  std::vector<char> cubin;
  std::string lg;
  int rc = nvrtc_compile(source, prop.major, prop.minor, &cubin, &lg);
  if (rc != FW_OK) return fail(rc, "NVRTC compilation failed:\n" + lg);
  fw_expr* x = new fw_expr();
  x->log = lg;
  e = cudaLibraryLoadData(&x->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
  if (e != cudaSuccess) {
    delete x;
    return cuda_fail(e, "cudaLibraryLoadData");
  }
  *out = x;
  return FW_OK;
}

extern "C" int fw_expr_destroy(fw_expr* x) {
  if (x == nullptr) return FW_OK;
  if (x->lib) cudaLibraryUnload(x->lib);
  delete x;
  return FW_OK;
}

extern "C" int fw_expr_eval(fw_expr* x, const char* name, const double* in, long long n, double* out_re,
                            double* out_im, void* stream) {
  if (x == nullptr || name == nullptr || in == nullptr || out_re == nullptr)
    return fail(FW_EINVAL, "fw_expr_eval: NULL argument");
  if (n <= 0) return FW_OK;
  cudaKernel_t k;
  cudaError_t e = cudaLibraryGetKernel(&k, x->lib, name);
  if (e != cudaSuccess) return cuda_fail(e, (std::string("cudaLibraryGetKernel(") + name + ")").c_str());
  void* args[] = {(void*)&in, (void*)&n, (void*)&out_re, (void*)&out_im};
  const int threads = 256;
  const long long blocks = (n + threads - 1) / threads;
  if (blocks > 0x7fffffffLL) return fail(FW_EINVAL, "fw_expr_eval: n too large");
  e = cudaLaunchKernel((const void*)k, dim3((unsigned)blocks), dim3(threads), args, 0,
                       static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "expression kernel launch");
  return FW_OK;
}
