// Ewald and direct sums on sampled targets, FP64 on the GPU: the accuracy
// reference for the FMM at sizes where a CPU sum takes hours.
//
// rtfmm_b200_ewald_sampled restates EwaldSolver (3dpp/src/ewald.cpp): splitting
// parameter alpha = ksize / L (ewald.cpp:13), real-space sum over r < L/2
// (cutoff, ewald.cpp:14), reciprocal sum over the (2 ksize + 1)^3 - 1 integer
// waves (ewald.cpp:16-30, 94-109, 177-202) and the self term
// -2 alpha q / sqrt(pi) (ewald.cpp:112-118).  The real-space image of a pair
// is the per-particle minimum image, which makes this the converged Ewald
// sum.  The reference picks one image per pair of leaf cells from the cell
// centres with a strict |dx| > L/2 test (ewald.cpp:121-152), which drops pairs
// that are close only across the periodic boundary.
// Outputs are phi and grad(phi) at the targets, no 1/(4 pi), no dipole term.
//
// rtfmm_b200_direct_sampled is the free-space sum (kernel.cpp:258-311 without
// lists): phi_t = sum q / r, grad_t = -sum q d / r^3 over all r > 0.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "rtfmm_b200.h"

namespace rtfmm_b200 {
void set_last_error(const std::string& msg);
}

namespace {

using rtfmm_b200::set_last_error;

constexpr int kTile = 32;       // bodies per shared-memory tile (structure factor)
constexpr int kColThreads = 128;  // (n1, n2) wave columns per block
constexpr int kMaxK = 16;       // largest ksize supported (33 waves per axis)
constexpr int kSumThreads = 256;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }

// Partial structure factors S(k) = sum_j q_j exp(-i k.x_j), k = (2 pi / L) n,
// over one chunk of bodies.  Thread = wave column (n1, n2); it sweeps n3 by
// repeated multiplication.  Per-body powers E_d^m = exp(-i 2 pi m x_d / L),
// m <= K, are built in shared memory by repeated multiplication from one
// sincospi per axis.  part: [chunk][col][n3] complex.
template <int K>
__global__ void __launch_bounds__(kColThreads)
    k_structure(const double4* __restrict__ xq, int64_t n, int64_t chunk, double inv_l,
                double2* __restrict__ part) {
  __shared__ double2 pw[kTile][3][K + 1];
  constexpr int W = 2 * K + 1, ncol = W * W;
  const int col = blockIdx.x * kColThreads + threadIdx.x;
  const int n1 = col / W - K, n2 = col % W - K;
  const int64_t b0 = (int64_t)blockIdx.y * chunk;
  const int64_t b1 = b0 + chunk < n ? b0 + chunk : n;
  double2 acc[W];
#pragma unroll
  for (int m = 0; m < W; ++m) acc[m] = make_double2(0.0, 0.0);
  for (int64_t t0 = b0; t0 < b1; t0 += kTile) {
    const int cnt = (int)(b1 - t0 < kTile ? b1 - t0 : kTile);
    __syncthreads();
    for (int e = threadIdx.x; e < cnt * 3; e += kColThreads) {
      const int j = e / 3, d = e % 3;
      const double4 b = xq[t0 + j];
      const double c = d == 0 ? b.x : (d == 1 ? b.y : b.z);
      double s, co;
      sincospi(-2.0 * c * inv_l, &s, &co);
      const double2 e1 = make_double2(co, s);
      double2 cur = make_double2(1.0, 0.0);
#pragma unroll
      for (int m = 0; m <= K; ++m) {
        pw[j][d][m] = cur;
        cur = cmul(cur, e1);
      }
    }
    __syncthreads();
    if (col < ncol) {
      for (int j = 0; j < cnt; ++j) {
        const double q = xq[t0 + j].w;
        const double2 a = n1 >= 0 ? pw[j][0][n1] : conj2(pw[j][0][-n1]);
        const double2 bb = n2 >= 0 ? pw[j][1][n2] : conj2(pw[j][1][-n2]);
        const double2 e3 = pw[j][2][1];
        double2 cur = cmul(cmul(a, bb), conj2(pw[j][2][K]));  // n3 = -K
        cur.x *= q;
        cur.y *= q;
#pragma unroll
        for (int m = 0; m < W; ++m) {
          acc[m].x += cur.x;
          acc[m].y += cur.y;
          cur = cmul(cur, e3);
        }
      }
    }
  }
  if (col < ncol) {
#pragma unroll
    for (int m = 0; m < W; ++m) part[((size_t)blockIdx.y * ncol + col) * W + m] = acc[m];
  }
}

// Sum the chunk partials in a fixed order and fold in the reciprocal-space
// weight (4 pi / L^3) exp(-k^2 / (4 alpha^2)) / k^2 (zero for k = 0).
__global__ void k_structure_sum(const double2* __restrict__ part, int nchunk, int K, double scale, double alpha,
                                double inv_vol4pi, double2* __restrict__ S) {
  const int W = 2 * K + 1, nk = W * W * W;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  double2 s = make_double2(0.0, 0.0);
  for (int c = 0; c < nchunk; ++c) {
    const double2 v = part[(size_t)c * nk + k];
    s.x += v.x;
    s.y += v.y;
  }
  const int n1 = k / (W * W) - K, n2 = (k / W) % W - K, n3 = k % W - K;
  const double k2 = (double)(n1 * n1 + n2 * n2 + n3 * n3) * scale * scale;
  const double w = k2 > 0 ? inv_vol4pi * exp(-k2 / (4 * alpha * alpha)) / k2 : 0.0;
  S[k] = make_double2(s.x * w, s.y * w);
}

// Per target: real-space sum over every source (minimum image, 0 < r < L/2),
// reciprocal sum over the waves, self term.  One block per target.
__global__ void __launch_bounds__(kSumThreads)
    k_ewald_targets(const double4* __restrict__ xq, int64_t n, const int64_t* __restrict__ tidx, double L,
                    double alpha, const double2* __restrict__ S, int K, double* __restrict__ phi,
                    double* __restrict__ grad) {
  __shared__ double red[4][kSumThreads];
  const int64_t ti = tidx[blockIdx.x];
  const double4 t = xq[ti];
  const double cutoff = 0.5 * L, a2 = alpha * alpha, c2 = 2.0 * alpha / sqrt(M_PI);
  double p = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
  for (int64_t j = threadIdx.x; j < n; j += kSumThreads) {
    const double4 s = xq[j];
    double dx = t.x - s.x, dy = t.y - s.y, dz = t.z - s.z;
    dx -= L * rint(dx / L);
    dy -= L * rint(dy / L);
    dz -= L * rint(dz / L);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double r = sqrt(r2);
    if (r > 0.0 && r < cutoff) {
      const double e = erfc(alpha * r);
      p += s.w * e / r;
      const double cf = s.w * (e + c2 * r * exp(-a2 * r2)) / (r2 * r);
      gx -= cf * dx;
      gy -= cf * dy;
      gz -= cf * dz;
    }
  }
  // reciprocal space: sum_k Re[S'(k) e^{i k.x}] and its gradient
  const int W = 2 * K + 1, nk = W * W * W;
  const double scale = 2.0 * M_PI / L;
  for (int k = threadIdx.x; k < nk; k += kSumThreads) {
    const int n1 = k / (W * W) - K, n2 = (k / W) % W - K, n3 = k % W - K;
    double sn, cs;
    sincospi(2.0 * (n1 * t.x + n2 * t.y + n3 * t.z) / L, &sn, &cs);
    const double2 v = S[k];
    const double re = v.x * cs - v.y * sn, im = v.x * sn + v.y * cs;
    p += re;
    gx -= im * scale * n1;
    gy -= im * scale * n2;
    gz -= im * scale * n3;
  }
  red[0][threadIdx.x] = p;
  red[1][threadIdx.x] = gx;
  red[2][threadIdx.x] = gy;
  red[3][threadIdx.x] = gz;
  __syncthreads();
  for (int o = kSumThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    phi[blockIdx.x] = red[0][0] - c2 * t.w;
    grad[3 * blockIdx.x + 0] = red[1][0];
    grad[3 * blockIdx.x + 1] = red[2][0];
    grad[3 * blockIdx.x + 2] = red[3][0];
  }
}

// Free-space direct sum per target.  One block per target.
__global__ void __launch_bounds__(kSumThreads)
    k_direct_targets(const double4* __restrict__ xq, int64_t n, const int64_t* __restrict__ tidx,
                     double* __restrict__ phi, double* __restrict__ grad) {
  __shared__ double red[4][kSumThreads];
  const double4 t = xq[tidx[blockIdx.x]];
  double p = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
  for (int64_t j = threadIdx.x; j < n; j += kSumThreads) {
    const double4 s = xq[j];
    const double dx = t.x - s.x, dy = t.y - s.y, dz = t.z - s.z;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > 0.0) {
      const double ir = 1.0 / sqrt(r2);
      const double qir = s.w * ir;
      p += qir;
      const double q3 = qir * ir * ir;
      gx -= q3 * dx;
      gy -= q3 * dy;
      gz -= q3 * dz;
    }
  }
  red[0][threadIdx.x] = p;
  red[1][threadIdx.x] = gx;
  red[2][threadIdx.x] = gy;
  red[3][threadIdx.x] = gz;
  __syncthreads();
  for (int o = kSumThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    phi[blockIdx.x] = red[0][0];
    grad[3 * blockIdx.x + 0] = red[1][0];
    grad[3 * blockIdx.x + 1] = red[2][0];
    grad[3 * blockIdx.x + 2] = red[3][0];
  }
}

// Device buffers of one call, freed on every return path.
struct Scratch {
  std::vector<void*> p;
  ~Scratch() {
    for (void* q : p) cudaFree(q);
  }
  template <typename T>
  cudaError_t alloc(T** out, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * (count ? count : 1));
    if (e == cudaSuccess) p.push_back(q);
    *out = reinterpret_cast<T*>(q);
    return e;
  }
};

int cuda_fail(cudaError_t e, const char* what) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return RTFMM_ECUDA;
}

#define EW_CK(x)                             \
  do {                                       \
    cudaError_t e_ = (x);                    \
    if (e_ != cudaSuccess) return cuda_fail(e_, #x); \
  } while (0)

int check_inputs(int64_t n, const double* x, const double* q, int64_t nt, const int64_t* targets, double* phi,
                 double* grad) {
  if (n < 1 || nt < 1 || nt > (1 << 30)) {
    set_last_error("n and the number of targets must be positive");
    return RTFMM_EINVAL;
  }
  if (!x || !q || !targets || !phi || !grad) {
    set_last_error("null argument");
    return RTFMM_EINVAL;
  }
  for (int64_t i = 0; i < nt; ++i)
    if (targets[i] < 0 || targets[i] >= n) {
      set_last_error("target index out of range");
      return RTFMM_EINVAL;
    }
  for (int64_t i = 0; i < 3 * n; ++i)
    if (!std::isfinite(x[i])) {
      set_last_error("non-finite body position");
      return RTFMM_EINVAL;
    }
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(q[i])) {
      set_last_error("non-finite charge");
      return RTFMM_EINVAL;
    }
  return RTFMM_OK;
}

int upload_bodies(Scratch& sc, int64_t n, const double* x, const double* q, int64_t nt, const int64_t* targets,
                  double4** d_xq, int64_t** d_t, double** d_phi, double** d_grad) {
  std::vector<double4> h(n);
  for (int64_t i = 0; i < n; ++i) h[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], q[i]);
  EW_CK(sc.alloc(d_xq, n));
  EW_CK(sc.alloc(d_t, nt));
  EW_CK(sc.alloc(d_phi, nt));
  EW_CK(sc.alloc(d_grad, 3 * nt));
  EW_CK(cudaMemcpy(*d_xq, h.data(), sizeof(double4) * n, cudaMemcpyHostToDevice));
  EW_CK(cudaMemcpy(*d_t, targets, sizeof(int64_t) * nt, cudaMemcpyHostToDevice));
  return RTFMM_OK;
}

}  // namespace

extern "C" int rtfmm_b200_ewald_sampled(int device, int64_t n, const double* x, const double* q, double cycle,
                                        int ksize, int64_t nt, const int64_t* targets, double* phi, double* grad) {
  int rc = check_inputs(n, x, q, nt, targets, phi, grad);
  if (rc) return rc;
  if (!(cycle > 0) || !std::isfinite(cycle) || ksize < 1 || ksize > kMaxK) {
    set_last_error("cycle must be positive and ksize in [1, 16]");
    return RTFMM_EINVAL;
  }
  EW_CK(cudaSetDevice(device));
  Scratch sc;
  double4* d_xq;
  int64_t* d_t;
  double *d_phi, *d_grad;
  rc = upload_bodies(sc, n, x, q, nt, targets, &d_xq, &d_t, &d_phi, &d_grad);
  if (rc) return rc;
  const int K = ksize, W = 2 * K + 1, ncol = W * W, nk = W * W * W;
  const double L = cycle, alpha = ksize / L, scale = 2 * M_PI / L;
  // bodies split into chunks so that every column block sees many SMs
  const int nchunk = (int)std::min<int64_t>(256, (n + kTile - 1) / kTile);
  const int64_t chunk = (n + nchunk - 1) / nchunk;
  double2 *d_part, *d_S;
  EW_CK(sc.alloc(&d_part, (size_t)nchunk * nk));
  EW_CK(sc.alloc(&d_S, (size_t)nk));
  dim3 g1((ncol + kColThreads - 1) / kColThreads, nchunk);
  switch (K) {
#define EW_K(k) \
  case k: k_structure<k><<<g1, kColThreads>>>(d_xq, n, chunk, 1.0 / L, d_part); break;
    EW_K(1) EW_K(2) EW_K(3) EW_K(4) EW_K(5) EW_K(6) EW_K(7) EW_K(8)
    EW_K(9) EW_K(10) EW_K(11) EW_K(12) EW_K(13) EW_K(14) EW_K(15) EW_K(16)
#undef EW_K
  }
  EW_CK(cudaGetLastError());
  k_structure_sum<<<(nk + 255) / 256, 256>>>(d_part, nchunk, K, scale, alpha, 4 * M_PI / (L * L * L), d_S);
  EW_CK(cudaGetLastError());
  k_ewald_targets<<<(unsigned)nt, kSumThreads>>>(d_xq, n, d_t, L, alpha, d_S, K, d_phi, d_grad);
  EW_CK(cudaGetLastError());
  EW_CK(cudaMemcpy(phi, d_phi, sizeof(double) * nt, cudaMemcpyDeviceToHost));
  EW_CK(cudaMemcpy(grad, d_grad, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
  return RTFMM_OK;
}

extern "C" int rtfmm_b200_direct_sampled(int device, int64_t n, const double* x, const double* q, int64_t nt,
                                         const int64_t* targets, double* phi, double* grad) {
  int rc = check_inputs(n, x, q, nt, targets, phi, grad);
  if (rc) return rc;
  EW_CK(cudaSetDevice(device));
  Scratch sc;
  double4* d_xq;
  int64_t* d_t;
  double *d_phi, *d_grad;
  rc = upload_bodies(sc, n, x, q, nt, targets, &d_xq, &d_t, &d_phi, &d_grad);
  if (rc) return rc;
  k_direct_targets<<<(unsigned)nt, kSumThreads>>>(d_xq, n, d_t, d_phi, d_grad);
  EW_CK(cudaGetLastError());
  EW_CK(cudaMemcpy(phi, d_phi, sizeof(double) * nt, cudaMemcpyDeviceToHost));
  EW_CK(cudaMemcpy(grad, d_grad, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
  return RTFMM_OK;
}
