// Dense kernels of the operator build on the GPU (LaplaceKernel::precompute,
// 3dpp/src/kernel.cpp:1638-1683): the one-sided Jacobi sweeps of the SVD of
// the equivalent-to-check operator and the products VSinv (UT G) of the M2M
// and image-M2M operators.
//
// Both give the host's results bit for bit, so an operator set built here
// equals one built by the host.  Every floating-point operation is the
// host's, in the host's order, with rounding to nearest and no contraction
// (__dmul_rn, __dadd_rn, __ddiv_rn, __dsqrt_rn): dot products and matrix
// sums run sequentially over their index in one thread, and only
// independent element updates are spread over threads.  The host code they
// mirror is jacobi_sweeps_host and matmul_host (rtfmm_plan.cpp).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "rtfmm_precompute.h"

namespace rtfmm_b200 {
namespace {

constexpr int kRoundThreads = 128;

// One round of the tournament: block b rotates the column pair
// (pairs[2b], pairs[2b+1]) of W (n rows) and Vc (m rows, first n updated).
__global__ void __launch_bounds__(kRoundThreads) k_jacobi_round(double* __restrict__ W, double* __restrict__ Vc,
                                                               int n, int m, const int* __restrict__ pairs,
                                                               unsigned long long* __restrict__ off_bits) {
  extern __shared__ double col[];  // 2n: columns p and q of W
  __shared__ double cs[2];
  __shared__ int go;
  const int p = pairs[2 * blockIdx.x], q = pairs[2 * blockIdx.x + 1];
  if (q >= n) return;  // the padding column
  double* sp = col;
  double* sq = col + n;
  double* wp = W + (size_t)p * n;
  double* wq = W + (size_t)q * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sp[i] = wp[i];
    sq[i] = wq[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double alpha = 0, beta = 0, gamma = 0;
    // in order over i (the host's sum); unrolled so the shared-memory loads
    // run ahead of the three dependent chains of adds
#pragma unroll 8
    for (int i = 0; i < n; ++i) {
      alpha = __dadd_rn(alpha, __dmul_rn(sp[i], sp[i]));
      beta = __dadd_rn(beta, __dmul_rn(sq[i], sq[i]));
      gamma = __dadd_rn(gamma, __dmul_rn(sp[i], sq[i]));
    }
    go = 0;
    if (!(alpha == 0.0 || beta == 0.0)) {
      const double rel = __ddiv_rn(fabs(gamma), __dsqrt_rn(__dmul_rn(alpha, beta)));
      // rel >= 0, so its bit pattern orders as its value (a NaN, which the
      // host's std::max would drop, is left out)
      if (!isnan(rel)) atomicMax(off_bits, (unsigned long long)__double_as_longlong(rel));
      if (!(rel < kJacobiTol)) {
        const double zeta = __ddiv_rn(__dsub_rn(beta, alpha), __dmul_rn(2.0, gamma));
        const double t = __ddiv_rn(zeta >= 0 ? 1.0 : -1.0,
                                   __dadd_rn(fabs(zeta), __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(zeta, zeta)))));
        const double c = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(t, t))));
        cs[0] = c;
        cs[1] = __dmul_rn(c, t);
        go = 1;
      }
    }
  }
  __syncthreads();
  if (!go) return;
  const double c = cs[0], sn = cs[1];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double a1 = sp[i], b1 = sq[i];
    wp[i] = __dsub_rn(__dmul_rn(c, a1), __dmul_rn(sn, b1));
    wq[i] = __dadd_rn(__dmul_rn(sn, a1), __dmul_rn(c, b1));
  }
  double* vp = Vc + (size_t)p * m;
  double* vq = Vc + (size_t)q * m;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double a1 = vp[i], b1 = vq[i];
    vp[i] = __dsub_rn(__dmul_rn(c, a1), __dmul_rn(sn, b1));
    vq[i] = __dadd_rn(__dmul_rn(sn, a1), __dmul_rn(c, b1));
  }
}

constexpr int kTile = 16;

// C = A B (n x n, row-major); C[i][j] accumulated over k in order from 0.0.
__global__ void __launch_bounds__(kTile* kTile) k_matmul_seq(int n, const double* __restrict__ A,
                                                            const double* __restrict__ B, double* __restrict__ C) {
  __shared__ double As[kTile][kTile + 1], Bs[kTile][kTile + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int row = blockIdx.y * kTile + ty, col = blockIdx.x * kTile + tx;
  double acc = 0.0;
  for (int k0 = 0; k0 < n; k0 += kTile) {
    As[ty][tx] = (row < n && k0 + tx < n) ? A[(size_t)row * n + k0 + tx] : 0.0;
    Bs[ty][tx] = (k0 + ty < n && col < n) ? B[(size_t)(k0 + ty) * n + col] : 0.0;
    __syncthreads();
    const int kend = min(kTile, n - k0);
    for (int kk = 0; kk < kend; ++kk) acc = __dadd_rn(acc, __dmul_rn(As[ty][kk], Bs[kk][tx]));
    __syncthreads();
  }
  if (row < n && col < n) C[(size_t)row * n + col] = acc;
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

struct Buf {
  void* p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
  template <typename T>
  T* get(size_t count) {
    check(cudaMalloc(&p, std::max<size_t>(1, count) * sizeof(T)), "cudaMalloc");
    return (T*)p;
  }
};

void launch_matmul(int n, const double* A, const double* B, double* C, cudaStream_t st) {
  const dim3 grid((n + kTile - 1) / kTile, (n + kTile - 1) / kTile), block(kTile, kTile);
  k_matmul_seq<<<grid, block, 0, st>>>(n, A, B, C);
  check(cudaGetLastError(), "k_matmul_seq");
}

}  // namespace

void jacobi_sweeps_gpu(int n, std::vector<double>& W, std::vector<double>& Vc, cudaStream_t st) {
  const int m = n + (n & 1);
  const size_t smem = sizeof(double) * 2 * (size_t)n;
  if (n < 2 || smem > 48 * 1024) {  // beyond one block's default shared memory: the host sweeps
    jacobi_sweeps_host(n, W, Vc);
    return;
  }
  const std::vector<int> pairs = jacobi_pairs(n);
  Buf bw, bv, bp, bo;
  double* dW = bw.get<double>(W.size());
  double* dV = bv.get<double>(Vc.size());
  int* dP = bp.get<int>(pairs.size());
  unsigned long long* dO = bo.get<unsigned long long>(1);
  check(cudaMemcpyAsync(dW, W.data(), sizeof(double) * W.size(), cudaMemcpyHostToDevice, st), "upload W");
  check(cudaMemcpyAsync(dV, Vc.data(), sizeof(double) * Vc.size(), cudaMemcpyHostToDevice, st), "upload V");
  check(cudaMemcpyAsync(dP, pairs.data(), sizeof(int) * pairs.size(), cudaMemcpyHostToDevice, st), "upload pairs");
  for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
    check(cudaMemsetAsync(dO, 0, sizeof(unsigned long long), st), "memset");
    for (int round = 0; round < m - 1; ++round) {
      k_jacobi_round<<<m / 2, kRoundThreads, smem, st>>>(dW, dV, n, m, dP + (size_t)round * m, dO);
      check(cudaGetLastError(), "k_jacobi_round");
    }
    unsigned long long bits = 0;
    check(cudaMemcpyAsync(&bits, dO, sizeof(bits), cudaMemcpyDeviceToHost, st), "off_max");
    check(cudaStreamSynchronize(st), "sweep");
    double off_max;
    std::memcpy(&off_max, &bits, sizeof(off_max));
    if (off_max < kJacobiTol) break;
  }
  check(cudaMemcpyAsync(W.data(), dW, sizeof(double) * W.size(), cudaMemcpyDeviceToHost, st), "download W");
  check(cudaMemcpyAsync(Vc.data(), dV, sizeof(double) * Vc.size(), cudaMemcpyDeviceToHost, st), "download V");
  check(cudaStreamSynchronize(st), "download");
}

void matmul_gpu(int n, const double* A, const double* B, double* C, cudaStream_t st) {
  const size_t nn = (size_t)n * n;
  Buf ba, bb, bc;
  double* dA = ba.get<double>(nn);
  double* dB = bb.get<double>(nn);
  double* dC = bc.get<double>(nn);
  check(cudaMemcpyAsync(dA, A, sizeof(double) * nn, cudaMemcpyHostToDevice, st), "upload A");
  check(cudaMemcpyAsync(dB, B, sizeof(double) * nn, cudaMemcpyHostToDevice, st), "upload B");
  launch_matmul(n, dA, dB, dC, st);
  check(cudaMemcpyAsync(C, dC, sizeof(double) * nn, cudaMemcpyDeviceToHost, st), "download C");
  check(cudaStreamSynchronize(st), "matmul");
}

void chain_gpu(int n, const double* A, const double* B, int nG, const double* const* G, double* const* out,
               cudaStream_t st) {
  const size_t nn = (size_t)n * n;
  Buf ba, bb, bg, bm, bc;
  double* dA = ba.get<double>(nn);
  double* dB = bb.get<double>(nn);
  double* dG = bg.get<double>(nn * nG);
  double* dM = bm.get<double>(nn);
  double* dC = bc.get<double>(nn * nG);
  check(cudaMemcpyAsync(dA, A, sizeof(double) * nn, cudaMemcpyHostToDevice, st), "upload A");
  check(cudaMemcpyAsync(dB, B, sizeof(double) * nn, cudaMemcpyHostToDevice, st), "upload B");
  for (int k = 0; k < nG; ++k)
    check(cudaMemcpyAsync(dG + nn * k, G[k], sizeof(double) * nn, cudaMemcpyHostToDevice, st), "upload G");
  for (int k = 0; k < nG; ++k) {
    launch_matmul(n, dB, dG + nn * k, dM, st);
    launch_matmul(n, dA, dM, dC + nn * k, st);
  }
  for (int k = 0; k < nG; ++k)
    check(cudaMemcpyAsync(out[k], dC + nn * k, sizeof(double) * nn, cudaMemcpyDeviceToHost, st), "download");
  check(cudaStreamSynchronize(st), "chain");
}

DenseBackend gpu_dense_backend(cudaStream_t st) {
  DenseBackend be;
  be.jacobi_sweeps = [st](int n, std::vector<double>& W, std::vector<double>& Vc) { jacobi_sweeps_gpu(n, W, Vc, st); };
  be.matmul = [st](int n, const double* A, const double* B, double* C) { matmul_gpu(n, A, B, C, st); };
  be.chain = [st](int n, const double* A, const double* B, int nG, const double* const* G, double* const* out) {
    chain_gpu(n, A, B, nG, G, out, st);
  };
  return be;
}

}  // namespace rtfmm_b200
