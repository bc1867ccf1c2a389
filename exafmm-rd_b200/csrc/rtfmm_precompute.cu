// Dense kernels of the operator build on the GPU (LaplaceKernel::precompute
// and precompute_m2l, 3dpp/src/kernel.cpp:1638-1769): the one-sided Jacobi
// sweeps of the SVD of the equivalent-to-check operator, the products
// VSinv (UT G) of the M2M and image-M2M operators, and the kernel spectra of
// the FFT-M2L.  (The Gram-Schmidt pass over the left singular vectors, a
// chain of n dependent steps, stays on the host cores, which run it faster.)
//
// All give the host's results bit for bit, so an operator set built here
// equals one built by the host.  Every floating-point operation is the
// host's, in the host's order, with rounding to nearest and no contraction
// (__dmul_rn, __dadd_rn, __ddiv_rn, __dsqrt_rn): sums run sequentially over
// their index in one thread, except the Jacobi inner products, which the host
// sums in a warp's order (jacobi_dots), and only independent element updates
// are spread over threads.  The host code they mirror is jacobi_sweeps_host,
// matmul_host and kernel_spectra_host (rtfmm_plan.cpp).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "rtfmm_precompute.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace rtfmm_b200 {
namespace {

constexpr int kRoundWarps = 4;

// The rotation of column pair (p, q) of W (n rows) and Vc (m rows, first n
// updated) by one warp.  Lane l sums the terms i = l, l + 32, ... of the three
// inner products in order, then the butterfly combines the lanes
// (jacobi_dots); every lane forms the same rotation.  The pair's
// |gamma|/sqrt(alpha beta) goes into *off_bits (a maximum of non-negative
// doubles taken on their bit patterns).
__device__ __forceinline__ void jacobi_pair(double* __restrict__ W, double* __restrict__ Vc, int n, int m, int p,
                                            int q, unsigned long long* __restrict__ off_bits) {
  const int lane = threadIdx.x & 31;
  double* wp = W + (size_t)p * n;
  double* wq = W + (size_t)q * n;
  double alpha = 0, beta = 0, gamma = 0;
  for (int i = lane; i < n; i += 32) {
    const double a = wp[i], b = wq[i];
    alpha = __dadd_rn(alpha, __dmul_rn(a, a));
    beta = __dadd_rn(beta, __dmul_rn(b, b));
    gamma = __dadd_rn(gamma, __dmul_rn(a, b));
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    alpha = __dadd_rn(alpha, __shfl_xor_sync(0xffffffffu, alpha, o));
    beta = __dadd_rn(beta, __shfl_xor_sync(0xffffffffu, beta, o));
    gamma = __dadd_rn(gamma, __shfl_xor_sync(0xffffffffu, gamma, o));
  }
  if (alpha == 0.0 || beta == 0.0) return;
  const double rel = __ddiv_rn(fabs(gamma), __dsqrt_rn(__dmul_rn(alpha, beta)));
  // a NaN, which the host's std::max would drop, is left out
  if (lane == 0 && !isnan(rel)) atomicMax(off_bits, (unsigned long long)__double_as_longlong(rel));
  if (rel < kJacobiTol) return;
  const double zeta = __ddiv_rn(__dsub_rn(beta, alpha), __dmul_rn(2.0, gamma));
  const double t =
      __ddiv_rn(zeta >= 0 ? 1.0 : -1.0, __dadd_rn(fabs(zeta), __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(zeta, zeta)))));
  const double c = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(t, t))));
  const double sn = __dmul_rn(c, t);
  for (int i = lane; i < n; i += 32) {
    const double a1 = wp[i], b1 = wq[i];
    wp[i] = __dsub_rn(__dmul_rn(c, a1), __dmul_rn(sn, b1));
    wq[i] = __dadd_rn(__dmul_rn(sn, a1), __dmul_rn(c, b1));
  }
  double* vp = Vc + (size_t)p * m;
  double* vq = Vc + (size_t)q * m;
  for (int i = lane; i < n; i += 32) {
    const double a1 = vp[i], b1 = vq[i];
    vp[i] = __dsub_rn(__dmul_rn(c, a1), __dmul_rn(sn, b1));
    vq[i] = __dadd_rn(__dmul_rn(sn, a1), __dmul_rn(c, b1));
  }
}

// One round of the tournament: warp w of block b rotates the pair
// pairs[2k], pairs[2k+1], k = 4 b + w.
__global__ void __launch_bounds__(32 * kRoundWarps) k_jacobi_round(double* __restrict__ W, double* __restrict__ Vc,
                                                                  int n, int m, const int* __restrict__ pairs,
                                                                  unsigned long long* __restrict__ off_bits) {
  const int k = blockIdx.x * kRoundWarps + (threadIdx.x >> 5);
  if (k >= m / 2) return;  // warp-uniform
  const int p = pairs[2 * k], q = pairs[2 * k + 1];
  if (q >= n) return;  // the padding column
  jacobi_pair(W, Vc, n, m, p, q, off_bits);
}

// Spins of a block at the grid barrier before it gives up (the blocks of a
// cooperative launch are all resident, so the barrier only gives up when
// something else has gone wrong).
constexpr long long kBarrierSpins = 1ll << 24;

// Grid-wide barrier of a cooperative launch: bar[0] counts arrivals, bar[1]
// is the generation.  A block that waits kBarrierSpins in vain sets *err and
// leaves; returns false when *err is set.
__device__ bool grid_barrier(unsigned* bar, int* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      bar[0] = 0;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long it = 0;
      while (*gen == g)
        if (++it > kBarrierSpins) {
          atomicExch(err, 1);
          break;
        }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int*)err == 0;
}

// Every sweep in one cooperative launch: the warps of the grid take the
// pairs of a round in turn, a grid barrier separates the rounds, and after a
// sweep's last round every block reads the sweep's maximum and stops when it
// is below the tolerance.  off_bits[s & 1] collects sweep s (the other slot
// is cleared for the next sweep once all blocks have read it).  status[0] =
// sweeps run, status[1] = 1 if a barrier gave up.
__global__ void __launch_bounds__(32 * kRoundWarps) k_jacobi_sweeps(double* __restrict__ W, double* __restrict__ Vc,
                                                                   int n, int m, const int* __restrict__ pairs,
                                                                   unsigned long long* __restrict__ off_bits,
                                                                   unsigned* __restrict__ bar, int* __restrict__ status) {
  const int nw = gridDim.x * kRoundWarps;
  const int w = blockIdx.x * kRoundWarps + (threadIdx.x >> 5);
  int sweep = 0;
  for (; sweep < kJacobiMaxSweeps; ++sweep) {
    unsigned long long* ob = off_bits + (sweep & 1);
    for (int round = 0; round < m - 1; ++round) {
      const int* pr = pairs + (size_t)round * m;
      for (int k = w; k < m / 2; k += nw) {
        const int p = pr[2 * k], q = pr[2 * k + 1];
        if (q < n) jacobi_pair(W, Vc, n, m, p, q, ob);
      }
      if (!grid_barrier(bar, status + 1)) return;
    }
    const unsigned long long bits = *(volatile unsigned long long*)ob;
    if (blockIdx.x == 0 && threadIdx.x == 0) off_bits[(sweep + 1) & 1] = 0;
    if (__longlong_as_double((long long)bits) < kJacobiTol) {
      ++sweep;
      break;
    }
    if (!grid_barrier(bar, status + 1)) return;  // every block has read the maximum
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) status[0] = sweep;
}

// Kernel spectra (kernel_spectra_host): block b takes offset b; the grid of
// 1/r and the two intermediate passes of the separable DFT live in the
// block's scratch (N^3 + 2 * 2 N^2 Nh doubles).  Thread per output, each sum
// sequential over its index as in dft3_r2c; cs/sn are the host's twiddles.
__global__ void __launch_bounds__(256) k_kernel_spectra(int N, const int* __restrict__ offs, double r0,
                                                        double delta, double gsize, const double* __restrict__ cs,
                                                        const double* __restrict__ sn, double* __restrict__ scratch,
                                                        double* __restrict__ gk) {
  const int Nh = N / 2 + 1;
  const size_t N3 = (size_t)N * N * N, Nc = (size_t)N * N * Nh;
  double* g = scratch + (size_t)blockIdx.x * (N3 + 4 * Nc);
  double* a = g + N3;
  double* b = a + 2 * Nc;
  double* out = gk + (size_t)blockIdx.x * 2 * Nc;
  const int* o = offs + 3 * blockIdx.x;
  const double rel0 = __dmul_rn(__dmul_rn((double)o[0], r0), 2.0);
  const double rel1 = __dmul_rn(__dmul_rn((double)o[1], r0), 2.0);
  const double rel2 = __dmul_rn(__dmul_rn((double)o[2], r0), 2.0);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (size_t e = tid; e < N3; e += nt) {
    const int i = (int)(e % N), j = (int)((e / N) % N), k = (int)(e / ((size_t)N * N));
    const double px = __dsub_rn(__dadd_rn(-gsize, __dmul_rn((double)i, delta)), rel0);
    const double py = __dsub_rn(__dadd_rn(-gsize, __dmul_rn((double)j, delta)), rel1);
    const double pz = __dsub_rn(__dadd_rn(-gsize, __dmul_rn((double)k, delta)), rel2);
    const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)), __dmul_rn(pz, pz)));
    g[e] = r == 0 ? 0.0 : __ddiv_rn(1.0, r);
  }
  __syncthreads();
  for (size_t e = tid; e < Nc; e += nt) {  // x -> kx: e = (z N + y) Nh + kx
    const int kx = (int)(e % Nh);
    const size_t zy = e / Nh;
    double re = 0, im = 0;
    for (int x = 0; x < N; ++x) {
      const int t = (kx * x) % N;
      const double v = g[zy * N + x];
      re = __dadd_rn(re, __dmul_rn(v, cs[t]));
      im = __dadd_rn(im, __dmul_rn(v, sn[t]));
    }
    a[2 * e] = re;
    a[2 * e + 1] = im;
  }
  __syncthreads();
  for (size_t e = tid; e < Nc; e += nt) {  // y -> ky: e = (z N + ky) Nh + kx
    const int kx = (int)(e % Nh), ky = (int)((e / Nh) % N), z = (int)(e / ((size_t)N * Nh));
    double re = 0, im = 0;
    for (int y = 0; y < N; ++y) {
      const int t = (ky * y) % N;
      const size_t s = ((size_t)z * N + y) * Nh + kx;
      re = __dadd_rn(re, __dsub_rn(__dmul_rn(a[2 * s], cs[t]), __dmul_rn(a[2 * s + 1], sn[t])));
      im = __dadd_rn(im, __dadd_rn(__dmul_rn(a[2 * s], sn[t]), __dmul_rn(a[2 * s + 1], cs[t])));
    }
    b[2 * e] = re;
    b[2 * e + 1] = im;
  }
  __syncthreads();
  for (size_t e = tid; e < Nc; e += nt) {  // z -> kz: e = (kz N + ky) Nh + kx
    const int kx = (int)(e % Nh), ky = (int)((e / Nh) % N), kz = (int)(e / ((size_t)N * Nh));
    double re = 0, im = 0;
    for (int z = 0; z < N; ++z) {
      const int t = (kz * z) % N;
      const size_t s = ((size_t)z * N + ky) * Nh + kx;
      re = __dadd_rn(re, __dsub_rn(__dmul_rn(b[2 * s], cs[t]), __dmul_rn(b[2 * s + 1], sn[t])));
      im = __dadd_rn(im, __dadd_rn(__dmul_rn(b[2 * s], sn[t]), __dmul_rn(b[2 * s + 1], cs[t])));
    }
    out[2 * e] = re;
    out[2 * e + 1] = im;
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

// A captured CUDA graph and its executable, released together.
struct Graph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  ~Graph() {
    if (x) cudaGraphExecDestroy(x);
    if (g) cudaGraphDestroy(g);
  }
};

int jacobi_sweeps_gpu(int n, std::vector<double>& W, std::vector<double>& Vc, cudaStream_t st, bool one_launch) {
  const int m = n + (n & 1);
  if (n < 2) {
    jacobi_sweeps_host(n, W, Vc);
    return -1;
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
  // all sweeps in one cooperative launch (its blocks all resident, so its
  // grid barriers can wait); a launch that is refused or a barrier that gives
  // up leaves it to the graph below, from the same inputs
  bool done = false;
  int sweeps_run = -1;
  {
    int dev = 0, nsm = 0, per = 0, coop = 0;
    check(cudaGetDevice(&dev), "device");
    check(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "attribute");
    check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "attribute");
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_jacobi_sweeps, 32 * kRoundWarps, 0), "occupancy");
    const int nblk = std::min((m / 2 + kRoundWarps - 1) / kRoundWarps, nsm * per);
    if (one_launch && coop && nblk >= 1) {
      Buf baux;
      unsigned long long* aux = baux.get<unsigned long long>(4);  // off_bits[2], bar[2], status[2]
      check(cudaMemsetAsync(aux, 0, sizeof(unsigned long long) * 4, st), "memset");
      unsigned long long* ob = aux;
      unsigned* bar = reinterpret_cast<unsigned*>(aux + 2);
      int* status = reinterpret_cast<int*>(aux + 3);
      int nn = n, mm = m;
      void* args[] = {&dW, &dV, &nn, &mm, &dP, &ob, &bar, &status};
      cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_jacobi_sweeps, dim3(nblk), dim3(32 * kRoundWarps),
                                                  args, 0, st);
      int hs[2] = {0, 0};
      if (e == cudaSuccess) e = cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e == cudaSuccess && hs[1] == 0) {
        done = true;
        sweeps_run = hs[0];
      } else if (e == cudaErrorCooperativeLaunchTooLarge || e == cudaErrorNotSupported || e == cudaSuccess) {
        cudaGetLastError();  // refused launch or a barrier that gave up: the graph path
        check(cudaMemcpyAsync(dW, W.data(), sizeof(double) * W.size(), cudaMemcpyHostToDevice, st), "upload W");
        check(cudaMemcpyAsync(dV, Vc.data(), sizeof(double) * Vc.size(), cudaMemcpyHostToDevice, st), "upload V");
      } else {
        check(e, "k_jacobi_sweeps");
      }
    }
  }
  if (!done) {
    // one sweep (the off-diagonal maximum cleared, then m - 1 rounds) as a
    // graph, replayed until the sweep leaves every pair below the tolerance
    Graph sweep;
    const int nblk = (m / 2 + kRoundWarps - 1) / kRoundWarps;
    check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
    cudaError_t e = cudaMemsetAsync(dO, 0, sizeof(unsigned long long), st);
    for (int round = 0; round < m - 1 && e == cudaSuccess; ++round) {
      k_jacobi_round<<<nblk, 32 * kRoundWarps, 0, st>>>(dW, dV, n, m, dP + (size_t)round * m, dO);
      e = cudaGetLastError();
    }
    const cudaError_t ec = cudaStreamEndCapture(st, &sweep.g);
    check(e, "k_jacobi_round");
    check(ec, "end capture");
    check(cudaGraphInstantiate(&sweep.x, sweep.g, 0), "instantiate");
    for (int s = 0; s < kJacobiMaxSweeps; ++s) {
      check(cudaGraphLaunch(sweep.x, st), "sweep");
      unsigned long long bits = 0;
      check(cudaMemcpyAsync(&bits, dO, sizeof(bits), cudaMemcpyDeviceToHost, st), "off_max");
      check(cudaStreamSynchronize(st), "sweep");
      double off_max;
      std::memcpy(&off_max, &bits, sizeof(off_max));
      if (off_max < kJacobiTol) break;
    }
  }
  check(cudaMemcpyAsync(W.data(), dW, sizeof(double) * W.size(), cudaMemcpyDeviceToHost, st), "download W");
  check(cudaMemcpyAsync(Vc.data(), dV, sizeof(double) * Vc.size(), cudaMemcpyDeviceToHost, st), "download V");
  check(cudaStreamSynchronize(st), "download");
  return sweeps_run;
}

void kernel_spectra_gpu(int N, int noff, const int* offs, double r0, double delta, double gsize, double* gk,
                        cudaStream_t st) {
  if (noff <= 0) return;
  const size_t N3 = (size_t)N * N * N, Nc = (size_t)N * N * (N / 2 + 1);
  // the host's twiddles (dft3_r2c)
  std::vector<double> cs(N), sn(N);
  for (int m = 0; m < N; ++m) {
    cs[m] = std::cos(2.0 * M_PI * m / N);
    sn[m] = -std::sin(2.0 * M_PI * m / N);
  }
  Buf bo, bc, bs, bw, bg;
  int* dOff = bo.get<int>(3 * (size_t)noff);
  double* dcs = bc.get<double>(N);
  double* dsn = bs.get<double>(N);
  double* dW = bw.get<double>((N3 + 4 * Nc) * noff);
  double* dG = bg.get<double>(2 * Nc * noff);
  check(cudaMemcpyAsync(dOff, offs, sizeof(int) * 3 * noff, cudaMemcpyHostToDevice, st), "upload offsets");
  check(cudaMemcpyAsync(dcs, cs.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st), "upload twiddles");
  check(cudaMemcpyAsync(dsn, sn.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st), "upload twiddles");
  k_kernel_spectra<<<noff, 256, 0, st>>>(N, dOff, r0, delta, gsize, dcs, dsn, dW, dG);
  check(cudaGetLastError(), "k_kernel_spectra");
  check(cudaMemcpyAsync(gk, dG, sizeof(double) * 2 * Nc * noff, cudaMemcpyDeviceToHost, st), "download spectra");
  check(cudaStreamSynchronize(st), "spectra");
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
  be.jacobi_sweeps = [st](int n, std::vector<double>& W, std::vector<double>& Vc) {
    (void)jacobi_sweeps_gpu(n, W, Vc, st);
  };
  be.matmul = [st](int n, const double* A, const double* B, double* C) { matmul_gpu(n, A, B, C, st); };
  be.chain = [st](int n, const double* A, const double* B, int nG, const double* const* G, double* const* out) {
    chain_gpu(n, A, B, nG, G, out, st);
  };
  be.spectra = [st](int N, int noff, const int* offs, double r0, double delta, double gsize, double* gk) {
    kernel_spectra_gpu(N, noff, offs, r0, delta, gsize, gk, st);
  };

  return be;
}

}  // namespace rtfmm_b200
