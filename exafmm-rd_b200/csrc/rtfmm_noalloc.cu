// P2M for a batch of leaves that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool or allocator (where a stray cudaMalloc would
// bypass its accounting or fail under its limits), or a host that has
// handed all device memory to that pool.  rtfmm_b200_p2m_noalloc serves them:
// the caller passes every input and the output as device pointers, and the
// scratch the stage needs (the leaves' check-surface potentials and the
// intermediate U^T p) lives in one file-scope __device__ array of fixed size
// that every GPU loading this library holds until the process exits.
//
// The arithmetic is that of the P2M stage of the evaluation pass
// (p2m_precompute, 3dpp/src/kernel.cpp:332-371): the same check-surface
// kernel and the same two batched operator applications, y = U^T p then
// q = 0.5^depth * (V S^-1) y, with the same summation order, so its output
// equals the pass's leaf equivalent densities.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/rtfmm_b200.h"
#include "rtfmm_kernels.cuh"

namespace rtfmm_b200 {

void set_last_error(const std::string& msg);  // rtfmm_capi.cu: rtfmm_b200_last_error()

namespace {

constexpr size_t kScratchDoubles = RTFMM_NOALLOC_SCRATCH_BYTES / sizeof(double);

// Shared by every call on a device; each call overwrites all of it that it
// reads, so nothing needs clearing between calls, and calls that overlap on
// the GPU (different streams, or different host threads) race on it.
static __device__ __align__(256) double g_p2m_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch[kMaxDevices] = {};  // device address of g_p2m_scratch, per device

static_assert(sizeof(rtfmm_leaf) == sizeof(LeafInfo), "rtfmm_leaf must match the internal leaf record");

// Unit-cube surface points (get_surface_points, 3dpp/src/surface.cpp:3-47),
// i outermost, k innermost; one thread, P^3 <= 4096 steps.
__global__ void k_na_surface(int P, double* unit) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int n = 0;
  for (int i = 0; i < P; ++i)
    for (int j = 0; j < P; ++j)
      for (int k = 0; k < P; ++k)
        if (i == 0 || i == P - 1 || j == 0 || j == P - 1 || k == 0 || k == P - 1) {
          unit[3 * n + 0] = -1.0 + i * 2.0 / (P - 1);
          unit[3 * n + 1] = -1.0 + j * 2.0 / (P - 1);
          unit[3 * n + 2] = -1.0 + k * 2.0 / (P - 1);
          ++n;
        }
}

// Row maps of the batched application: identity rows, one group, and the
// per-leaf 0.5^depth scale taken from the leaf records.
__global__ void k_na_rows(const LeafInfo* leaves, int nleaf, int* iota, int* group_off, double* scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nleaf) {
    iota[i] = i;
    scale[i] = leaves[i].scale;
  }
  if (i == 0) {
    group_off[0] = 0;
    group_off[1] = nleaf;
  }
}

int fail(int code, const char* msg) {
  set_last_error(msg);
  return code;
}

}  // namespace

}  // namespace rtfmm_b200

using namespace rtfmm_b200;

extern "C" int rtfmm_b200_p2m_noalloc(int P, int64_t nleaf, const rtfmm_leaf* d_leaves, const double* d_bodies,
                                      const double* d_U, const double* d_VSinvT, double* d_q_equiv,
                                      void* stream) {
  if (P < 2 || P > 16) return fail(RTFMM_EINVAL, "p2m_noalloc: P must be in [2, 16]");
  if (nleaf < 0) return fail(RTFMM_EINVAL, "p2m_noalloc: nleaf must be >= 0");
  if (nleaf == 0) return RTFMM_OK;
  if (!d_leaves || !d_bodies || !d_U || !d_VSinvT || !d_q_equiv)
    return fail(RTFMM_EINVAL, "p2m_noalloc: null device pointer");
  // the kernels read bodies as double4, copy operator rows in 16-byte pieces
  // and store q_equiv as double2; the leaf records are read as 8-byte fields
  auto misaligned = [](const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) != 0; };
  if (misaligned(d_bodies, 16) || misaligned(d_U, 16) || misaligned(d_VSinvT, 16) || misaligned(d_q_equiv, 16) ||
      misaligned(d_leaves, 8))
    return fail(RTFMM_EINVAL,
                "p2m_noalloc: d_bodies, d_U, d_VSinvT and d_q_equiv must be 16-byte aligned, d_leaves 8-byte");
  // bound nleaf before any product so that the size arithmetic cannot wrap
  if (nleaf > (int64_t)kScratchDoubles)
    return fail(RTFMM_EINVAL,
                "p2m_noalloc: batch too large for the fixed scratch; split the leaves into smaller batches");
  const int ns = 6 * (P - 1) * (P - 1) + 2;
  // scratch: check potentials and U^T p (nleaf*ns each), surface points
  // (3*ns), per-leaf scale (nleaf), then integer row maps (nleaf + 2 ints)
  const size_t need = 2 * (size_t)nleaf * ns + 3 * (size_t)ns + (size_t)nleaf + ((size_t)nleaf + 2 + 1) / 2;
  if (need > kScratchDoubles)
    return fail(RTFMM_EINVAL,
                "p2m_noalloc: batch too large for the fixed scratch (needs 2*nleaf*num_surf + 3*num_surf + "
                "1.5*nleaf doubles within RTFMM_NOALLOC_SCRATCH_BYTES); split the leaves into smaller batches");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(RTFMM_ECUDA, "p2m_noalloc: no current CUDA device");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Outside stream capture the scratch array's device address is looked up
  // on every call (it moves when the module is loaded again after a device
  // reset); during capture the address cached by an earlier call is used, so
  // the first call on a device must come before any capture.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess)
    return fail(RTFMM_ECUDA, "p2m_noalloc: cudaStreamIsCapturing failed");
  double* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (cap == cudaStreamCaptureStatusNone) {
      // the symbol's device address, taken with this device current (the
      // host-side name is not a device address)
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_p2m_scratch);
      if (e != cudaSuccess) return fail(RTFMM_ECUDA, "p2m_noalloc: cudaGetSymbolAddress failed");
      g_scratch[dev] = static_cast<double*>(p);
    } else if (!g_scratch[dev]) {
      return fail(RTFMM_EINVAL, "p2m_noalloc: the first call on a device must come before any stream capture");
    }
    base = g_scratch[dev];
  }
  const int nl = (int)nleaf;
  double* pcheck = base;
  double* ymid = pcheck + (size_t)nl * ns;
  double* unit = ymid + (size_t)nl * ns;
  double* scale = unit + 3 * (size_t)ns;
  int* iota = reinterpret_cast<int*>(scale + nl);
  int* group_off = iota + nl;
  const LeafInfo* leaves = reinterpret_cast<const LeafInfo*>(d_leaves);
  k_na_surface<<<1, 32, 0, st>>>(P, unit);
  k_na_rows<<<(nl + 255) / 256, 256, 0, st>>>(leaves, nl, iota, group_off, scale);
  if (cudaGetLastError() != cudaSuccess) return fail(RTFMM_ECUDA, "p2m_noalloc: launch failed");
  if (launch_p2m_check(reinterpret_cast<const double4*>(d_bodies), leaves, nl, unit, ns, pcheck, st) !=
      cudaSuccess)
    return fail(RTFMM_ECUDA, "p2m_noalloc: check-surface launch failed");
  ApplyBatch b;
  b.groups = 1;
  b.S = 1;
  b.ns = ns;
  b.beta = 0;
  b.max_rows = nl;
  b.inrow = iota;
  b.outrow = iota;
  b.group_off = group_off;
  b.A = pcheck;
  b.B = d_U;  // y[n] = sum_j U[j][n] p[j]
  b.scale = nullptr;
  b.C = ymid;
  if (launch_apply(b, st) != cudaSuccess) return fail(RTFMM_ECUDA, "p2m_noalloc: U^T launch failed");
  b.A = ymid;
  b.B = d_VSinvT;  // q[n] = scale * sum_j (V S^-1)[n][j] y[j]
  b.scale = scale;
  b.C = d_q_equiv;
  if (launch_apply(b, st) != cudaSuccess) return fail(RTFMM_ECUDA, "p2m_noalloc: V S^-1 launch failed");
  return RTFMM_OK;
}
