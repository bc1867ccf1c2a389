// The dense kernels of the operator build on the GPU (bit for bit the
// host's): a DenseBackend for build_operators.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "rtfmm_plan.h"

namespace rtfmm_b200 {

// returns the sweeps run by the one-launch (cooperative) form, -1 when the
// per-sweep graph (or the host, n < 2) ran them; one_launch = false asks for
// the graph form
int jacobi_sweeps_gpu(int n, std::vector<double>& W, std::vector<double>& Vc, cudaStream_t st,
                      bool one_launch = true);
void matmul_gpu(int n, const double* A, const double* B, double* C, cudaStream_t st);
void chain_gpu(int n, const double* A, const double* B, int nG, const double* const* G, double* const* out,
               cudaStream_t st);
void kernel_spectra_gpu(int N, int noff, const int* offs, double r0, double delta, double gsize, double* gk,
                        cudaStream_t st);
// Runs on `st`; throws std::runtime_error on a CUDA error.
DenseBackend gpu_dense_backend(cudaStream_t st);

}  // namespace rtfmm_b200
