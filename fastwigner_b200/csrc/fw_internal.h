// Internal declarations shared by the CUDA translation units of libfastwigner.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "../../include/fastwigner.h"

namespace fw {
struct PassArgs;
cudaError_t launch_row(const PassArgs& a, int dtype, cudaStream_t st);
cudaError_t launch_col(const PassArgs& a, int dtype, cudaStream_t st, int* nparts);
cudaError_t launch_finalize(const PassArgs& a, int dtype, cudaStream_t st);
cudaError_t launch_pweight_dft(const double* wp, long long wp_bs, int Mp, int P, int nb, void* out, long long out_bs,
                               int dtype, cudaStream_t st);
cudaError_t launch_totals(const double* part, int nparts, int M, int batch, double* tot, double* hist,
                          cudaStream_t st);
int col_parts(int dtype, int P, int X, int small);
int row_rv(int dtype, int N, int small);
int small_shapes(int dtype, int P, int X, int batch);
bool size_supported(int n);

void set_error(const std::string& msg);
void count_launch(long long n);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);
}  // namespace fw
