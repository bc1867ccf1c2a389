// Device kernels of the periodic KIFMM evaluation pass for sm_100a.
//
// Stage map (reference function -> kernel here):
//   p2p_1toN_256          (3dpp/src/kernel.cpp:258-311)   k_p2p32 / k_p2p64
//   p2m_precompute        (kernel.cpp:332-371)            k_p2m_check + k_apply_f64_tc
//   m2m_precompute / img  (kernel.cpp:395-404, 434-442)   k_apply_f64_tc per level
//   m2l_fft_precompute_t  (kernel.cpp:1140-1397)          k_m2l_up, k_m2l_hadamard8,
//     hadamard_8x8 / 1x27 (kernel.cpp:1012-1138)          k_m2l_hadamard27, k_m2l_down
//   l2l_precompute / img  (kernel.cpp:1419-1435)          k_apply_f64_tc per level
//   l2p_precompute        (kernel.cpp:1458-1511)          k_apply_f64_tc + k_l2p_eval
// (k_apply_f64 is the SIMT form of the operator GEMM, built with APPLY_TC=0.)
// The adjoint adds k_swap_charges, k_restore_charges, k_adj_combine; the
// device-buffer forward k_set_charges.
//   dipole_correction, scale_bodies, sort_bodies_by_idx
//                         (kernel.cpp:1580-1596, body.cpp:88-96,177-190)  k_dipole_*, k_post
//
// Every index a kernel forms is checked against the extent of the buffer it
// addresses; no kernel waits on another block.
#include "rtfmm_kernels.cuh"

#include <cuda_runtime.h>

#include <atomic>

#include <cub/cub.cuh>

// FP64 pair kernels: seed the reciprocal square root with the FP64 (1) or
// FP32 (0) hardware approximation
#ifndef RSQ_SEED64
#define RSQ_SEED64 1
#endif
// FP32 P2P: inner unroll and resident blocks per SM.  A block is one warp
// (P2P_WARPS): work items differ in cost several-fold, and a block of four
// held the slots of its finished warps until its slowest one was done
// (3.33 against 3.12 ms at N = 2^20, P = 8).
#ifndef P2P_UNROLL
#define P2P_UNROLL 4
#endif
#ifndef P2P_MINB
#define P2P_MINB 20
#endif
#ifndef P2P_PACKED
#define P2P_PACKED 1
#endif
#ifndef P2P_WARPS
#define P2P_WARPS 1
#endif
#ifndef P2P_TILE
#define P2P_TILE 32
#endif
// register-blocked FFT-M2L up: resident blocks per SM (FP32; FP64 keeps 2)
#ifndef UP_RB_MINB
#define UP_RB_MINB 3
#endif
// FP32 Hadamard: targets per thread, directions per FP32 partial sum,
// resident blocks per SM
#ifndef HAD_TT
#define HAD_TT 2
#endif
#ifndef HAD_DF
#define HAD_DF 8
#endif
#ifndef HAD_MINB
#define HAD_MINB 4
#endif
// FP32 Hadamard: FP64 accumulators in shared memory (1) or registers (0)
#ifndef HAD_ACC_SMEM
#define HAD_ACC_SMEM 1
#endif
// 8x8 source spectra in 32-byte chunks (1) or whole rows (0), q8_index; the
// FP64 spectra too (Q8_CHUNKED64)
#ifndef Q8_CHUNKED
#define Q8_CHUNKED 1
#endif
#ifndef Q8_CHUNKED64
#define Q8_CHUNKED64 1
#endif
// FP32 Hadamard: packed FP32x2 FMAs (1) or scalar FMAs (0)
#ifndef HAD_F2
#define HAD_F2 1
#endif
// FP64 operator application: output rows per block (64 or 128), FP64
// tensor-core (mma.sync) inner product
#ifndef APPLY_TM
#define APPLY_TM 64
#endif
#ifndef APPLY_MMA
#define APPLY_MMA 0
#endif
// FP64 operator application on the cp.async + mma.sync kernel
#ifndef APPLY_TC
#define APPLY_TC 1
#endif

namespace rtfmm_b200 {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };
// two complex values in one vector load
template <typename T> struct Cplx2;
template <> struct Cplx2<float> { using type = float4; };
template <> struct Cplx2<double> { using type = double4; };

// Layout of the 8x8 source spectra Q (complex, [frequency][source][slot]).
// A frequency's rows are stored in 32-byte chunks (4 slots in FP32, 2 in
// FP64): chunk 0 of every source, then chunk 1, ..., so that the Hadamard's
// lanes, which take consecutive targets and so mostly consecutive sources,
// read a chunk of their rows from consecutive sectors, and an up-pass block
// (slot pairs of one source) still writes whole sectors.
template <typename T>
__host__ __device__ __forceinline__ size_t q8_index(size_t f, int src, int slot, int nsrc) {
  constexpr int per = 32 / (2 * sizeof(T)), nch = 8 / per;  // slots per chunk, chunks per row
  if (Q8_CHUNKED && (sizeof(T) == 4 || Q8_CHUNKED64))
    return ((f * nch + slot / per) * nsrc + src) * per + slot % per;
  return (f * nsrc + src) * 8 + slot;
}

// 32-byte (one sector) vector loads, sm_100: one lane reads a whole sector.
__device__ __forceinline__ void ld_sector(const float* p, float (&v)[8]) {
  asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
               : "l"(p));
}
__device__ __forceinline__ void ld_sector(const double* p, double (&v)[4]) {
  asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}

__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// 1/sqrt(x) in FP64 by Newton-Raphson, y <- y (3/2 - x y^2 / 2), from a
// hardware seed.  The PTX FP64 approximation (rsqrt.approx.ftz.f64, one
// special-function op) is good to 9.1e-7 relative; one step gives 1.3e-12 and
// two give 3.3e-16 (maxima measured against CUDA's rsqrt over 1e-30..1e30).
// The FP32 approximation (1.5e-7, but two conversions on the same pipe as the
// seed) gives 3.2e-14 and 3.3e-16, for arguments in the normal FP32 range.
// x must be positive and normal (pairs closer than 1e-154 are not supported).
template <int NR>
__device__ __forceinline__ double rsqrt_nr(double x) {
#if RSQ_SEED64
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#else
  const float xf = (float)x;
  if (!(xf >= 1.2e-38f && xf <= 3.0e38f)) return rsqrt(x);
  double y = (double)rsqrt_approx(xf);
#endif
  const double h = 0.5 * x;
#pragma unroll
  for (int i = 0; i < NR; ++i) y = y * fma(-h * y, y, 1.5);
  return y;
}

// ---------------------------------------------------------------------------
// body preparation
// ---------------------------------------------------------------------------
__global__ void k_gather_bodies(const double* __restrict__ x_in, const double* __restrict__ q_in,
                                const int64_t* __restrict__ perm, int n, double4* __restrict__ body64) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t k = perm[i];
  body64[i] = make_double4(x_in[3 * k], x_in[3 * k + 1], x_in[3 * k + 2], q_in[k]);
}

// FP32 leaf-relative positions: (x - c_leaf, q) so that P2P differences stay
// accurate in single precision.
__global__ void k_prep32(const double4* __restrict__ body64, const int* __restrict__ body_leaf,
                         const LeafInfo* __restrict__ leaves, float4* __restrict__ body32, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 b = body64[i];
  const LeafInfo L = leaves[body_leaf[i]];
  body32[i] = make_float4((float)(b.x - L.cx), (float)(b.y - L.cy), (float)(b.z - L.cz), (float)b.w);
}

// body_leaf[b] = the leaf holding tree-order body b (block per leaf)
__global__ void k_body_leaf(const LeafInfo* __restrict__ leaves, int nleaf, int n, int* __restrict__ body_leaf) {
  const int l = blockIdx.x;
  if (l >= nleaf) return;
  const LeafInfo L = leaves[l];
  for (int b = threadIdx.x; b < L.bnum; b += blockDim.x)
    if (L.boff + b >= 0 && L.boff + b < n) body_leaf[L.boff + b] = l;
}

// ---------------------------------------------------------------------------
// P2P: one warp per work item (up to 32 targets of one leaf); sources staged
// 32 at a time in a per-warp shared-memory slot and read as broadcasts, the
// next tile's bodies and the next list entry loaded while the current tile is
// computed.  FP32 partial sums per source leaf are accumulated into FP64.
// ---------------------------------------------------------------------------
constexpr int kP2PWarps = P2P_WARPS;
constexpr int kP2PUnroll = P2P_UNROLL;
constexpr int kP2PTile = P2P_TILE;  // sources staged per tile (32 or 64)

// Lanes of group `k0` (of G groups) take the tile's sources k0, k0+G, ...
template <int G, bool MASK>
__device__ __forceinline__ void p2p32_tile(const float4* __restrict__ s, int k0, int cnt, float px, float py,
                                           float pz, float& p, float& fx, float& fy, float& fz) {
#pragma unroll kP2PUnroll
  for (int k = k0; k < cnt; k += G) {
    const float4 b = s[k];
    const float dx = px - b.x, dy = py - b.y, dz = pz - b.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float ir = rsqrt_approx(r2);
    if (MASK) ir = r2 > 0.f ? ir : 0.f;
    const float qir = b.w * ir;
    p += qir;
    const float q3 = qir * ir * ir;
    fx = fmaf(q3, dx, fx);
    fy = fmaf(q3, dy, fy);
    fz = fmaf(q3, dz, fz);
  }
}

// One source pair k of a packed tile (layout below) against this lane's target.
template <bool MASK>
__device__ __forceinline__ void p2p32_pair2(const float4* __restrict__ s, int k, float2 px, float2 py, float2 pz,
                                            float2& p, float2& fx, float2& fy, float2& fz) {
  const float4 u = s[2 * k], v = s[2 * k + 1];
  const float2 dx = __fadd2_rn(px, make_float2(u.x, u.y));
  const float2 dy = __fadd2_rn(py, make_float2(u.z, u.w));
  const float2 dz = __fadd2_rn(pz, make_float2(v.x, v.y));
  float2 r2 = __fmul2_rn(dz, dz);
  r2 = __ffma2_rn(dy, dy, r2);
  r2 = __ffma2_rn(dx, dx, r2);
  float2 ir = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
  if (MASK) {
    ir.x = r2.x > 0.f ? ir.x : 0.f;
    ir.y = r2.y > 0.f ? ir.y : 0.f;
  }
  const float2 qir = __fmul2_rn(make_float2(v.z, v.w), ir);
  p = __fadd2_rn(p, qir);
  const float2 q3 = __fmul2_rn(__fmul2_rn(qir, ir), ir);
  fx = __ffma2_rn(q3, dx, fx);
  fy = __ffma2_rn(q3, dy, fy);
  fz = __ffma2_rn(q3, dz, fz);
}

// The same over source pairs with packed FP32x2 arithmetic (sm_100
// FADD2/FMUL2/FFMA2): the tile is held as 16 pairs, pair k at s[2k] =
// (-x, -x', -y, -y') and s[2k+1] = (-z, -z', q, q'); lanes of group k0 take
// pairs k0, k0+G, ...  Per pair the arithmetic and its rounding are those of
// p2p32_tile; only the sum over sources is split into two interleaved halves.
// All 16 pairs of a tile are written (padding carries no charge and sits far
// away); running the padding too, in fixed blocks, was measured slower.
template <int G, bool MASK>
__device__ __forceinline__ void p2p32_tile2(const float4* __restrict__ s, int k0, int npair, float2 px, float2 py,
                                            float2 pz, float2& p, float2& fx, float2& fy, float2& fz) {
#pragma unroll kP2PUnroll
  for (int k = k0; k < npair; k += G) p2p32_pair2<MASK>(s, k, px, py, pz, p, fx, fy, fz);
}

// One work item: W = 32/G lanes per target group, G groups per warp.
template <int G>
__device__ __forceinline__ void p2p32_item(const float4* __restrict__ body32, const P2PItem32& it,
                                           const int* __restrict__ list_off, const P2PSrc32* __restrict__ list,
                                           float4* __restrict__ sw, int lane, double* __restrict__ phi,
                                           double* __restrict__ grad) {
  constexpr int W = 32 / G;
  const int grp = lane / W, ti = lane % W;
  const bool active = ti < it.nt;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  // tile padding: no charge, far from every target (finite 1/r)
  const float4 pad = make_float4(1e18f, 1e18f, 1e18f, 0.f);
  const float4 xt = active ? body32[it.boff + ti] : zero;
  double P = 0.0, Gx = 0.0, Gy = 0.0, Gz = 0.0;
  int e = list_off[it.leaf];
  const int e1 = list_off[it.leaf + 1];
  P2PSrc32 cur{}, nxt{};
  // this lane stages sources c0 + lane + 32 h of the tile, h < kP2PTile / 32
  constexpr int NH = kP2PTile / 32;
  float4 stage[NH];
#pragma unroll
  for (int h = 0; h < NH; ++h) stage[h] = pad;
  if (e < e1) {
    cur = list[e];
#pragma unroll
    for (int h = 0; h < NH; ++h)
      if (lane + 32 * h < cur.bnum) stage[h] = body32[cur.boff + lane + 32 * h];
  }
  if (e + 1 < e1) nxt = list[e + 1];
  int c0 = 0;
#if P2P_PACKED
  float2 p = make_float2(0.f, 0.f), fx = p, fy = p, fz = p;
  float* sf = reinterpret_cast<float*>(sw) + 8 * (lane >> 1) + (lane & 1);
#else
  static_assert(kP2PTile == 32, "the scalar P2P form stages 32 sources");
  float p = 0.f, fx = 0.f, fy = 0.f, fz = 0.f;
#endif
  while (e < e1) {
    const int cnt = min(kP2PTile, cur.bnum - c0);
    __syncwarp();
#if P2P_PACKED
#pragma unroll
    for (int h = 0; h < NH; ++h) {
      sf[128 * h + 0] = -stage[h].x;
      sf[128 * h + 2] = -stage[h].y;
      sf[128 * h + 4] = -stage[h].z;
      sf[128 * h + 6] = stage[h].w;
    }
#else
    sw[lane] = stage[0];
#endif
    __syncwarp();
    // next tile: the rest of this source leaf, else the first of the next
    const bool last = c0 + kP2PTile >= cur.bnum;
#pragma unroll
    for (int h = 0; h < NH; ++h) {
      stage[h] = pad;
      if (!last) {
        if (lane + 32 * h < cur.bnum - c0 - kP2PTile) stage[h] = body32[cur.boff + c0 + kP2PTile + lane + 32 * h];
      } else if (e + 1 < e1) {
        if (lane + 32 * h < nxt.bnum) stage[h] = body32[nxt.boff + lane + 32 * h];
      }
    }
    const float px = xt.x - cur.dx, py = xt.y - cur.dy, pz = xt.z - cur.dz;
#if P2P_PACKED
    const int npair = (cnt + 1) >> 1;
    if (cur.self)
      p2p32_tile2<G, true>(sw, grp, npair, make_float2(px, px), make_float2(py, py), make_float2(pz, pz), p, fx,
                           fy, fz);
    else
      p2p32_tile2<G, false>(sw, grp, npair, make_float2(px, px), make_float2(py, py), make_float2(pz, pz), p, fx,
                            fy, fz);
#else
    if (cur.self)
      p2p32_tile<G, true>(sw, grp, cnt, px, py, pz, p, fx, fy, fz);
    else
      p2p32_tile<G, false>(sw, grp, cnt, px, py, pz, p, fx, fy, fz);
#endif
    if (last) {
#if P2P_PACKED
      P += (double)p.x + (double)p.y;
      Gx += (double)fx.x + (double)fx.y;
      Gy += (double)fy.x + (double)fy.y;
      Gz += (double)fz.x + (double)fz.y;
      p = fx = fy = fz = make_float2(0.f, 0.f);
#else
      P += (double)p;
      Gx += (double)fx;
      Gy += (double)fy;
      Gz += (double)fz;
      p = fx = fy = fz = 0.f;
#endif
      ++e;
      c0 = 0;
      cur = nxt;
      if (e + 1 < e1) nxt = list[e + 1];
    } else {
      c0 += kP2PTile;
    }
  }
  // sum the source groups (lanes ti, ti + W, ...)
#pragma unroll
  for (int o = W; o < 32; o <<= 1) {
    P += __shfl_xor_sync(0xffffffffu, P, o);
    Gx += __shfl_xor_sync(0xffffffffu, Gx, o);
    Gy += __shfl_xor_sync(0xffffffffu, Gy, o);
    Gz += __shfl_xor_sync(0xffffffffu, Gz, o);
  }
  if (active && grp == 0) {
    const int b = it.boff + ti;
    phi[b] = P;
    grad[3 * b + 0] = -Gx;
    grad[3 * b + 1] = -Gy;
    grad[3 * b + 2] = -Gz;
  }
}

__global__ void __launch_bounds__(32 * kP2PWarps, P2P_MINB)
    k_p2p32(const float4* __restrict__ body32, const P2PItem32* __restrict__ items, int nitems,
            const int* __restrict__ list_off, const P2PSrc32* __restrict__ list, double* __restrict__ phi,
            double* __restrict__ grad) {
  __shared__ float4 sbuf[kP2PWarps][kP2PTile];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x * kP2PWarps + warp;
  if (item >= nitems) return;  // warp-uniform
  const P2PItem32 it = items[item];
  switch (it.lw) {
    case 5: p2p32_item<1>(body32, it, list_off, list, sbuf[warp], lane, phi, grad); break;
    case 4: p2p32_item<2>(body32, it, list_off, list, sbuf[warp], lane, phi, grad); break;
    case 3: p2p32_item<4>(body32, it, list_off, list, sbuf[warp], lane, phi, grad); break;
    default: p2p32_item<8>(body32, it, list_off, list, sbuf[warp], lane, phi, grad); break;
  }
}

// FP64 P2P, the same work items as the FP32 kernel (lane groups for a leaf's
// last targets, next tile and list entry loaded during the current tile);
// per pair the reference's arithmetic (dx = x_t - (x_s + offset),
// kernel.cpp:283-290) in FP64 with the Newton-refined reciprocal square root.
template <int G>
__device__ __forceinline__ void p2p64_item(const double4* __restrict__ body64, const P2PItem32& it,
                                           const int* __restrict__ list_off, const P2PSrc64* __restrict__ list,
                                           double4* __restrict__ sw, int lane, double* __restrict__ phi,
                                           double* __restrict__ grad) {
  constexpr int W = 32 / G;
  const int grp = lane / W, ti = lane % W;
  const bool active = ti < it.nt;
  const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
  const double4 xt = active ? body64[it.boff + ti] : zero;
  double P = 0.0, Gx = 0.0, Gy = 0.0, Gz = 0.0;
  int e = list_off[it.leaf];
  const int e1 = list_off[it.leaf + 1];
  P2PSrc64 cur{}, nxt{};
  double4 stage = zero;
  if (e < e1) {
    cur = list[e];
    if (lane < cur.bnum) stage = body64[cur.boff + lane];
  }
  if (e + 1 < e1) nxt = list[e + 1];
  int c0 = 0;
  while (e < e1) {
    const int cnt = min(32, cur.bnum - c0);
    __syncwarp();
    sw[lane] = stage;
    __syncwarp();
    const bool last = c0 + 32 >= cur.bnum;
    stage = zero;
    if (!last) {
      if (lane < cur.bnum - c0 - 32) stage = body64[cur.boff + c0 + 32 + lane];
    } else if (e + 1 < e1) {
      if (lane < nxt.bnum) stage = body64[nxt.boff + lane];
    }
#pragma unroll 4
    for (int k = grp; k < cnt; k += G) {
      const double4 b = sw[k];
      const double dx = xt.x - (b.x + cur.ox), dy = xt.y - (b.y + cur.oy), dz = xt.z - (b.z + cur.oz);
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double ir = r2 > 0.0 ? rsqrt_nr<2>(r2) : 0.0;
      const double qir = b.w * ir;
      P += qir;
      const double q3 = qir * ir * ir;
      Gx += q3 * dx;
      Gy += q3 * dy;
      Gz += q3 * dz;
    }
    if (last) {
      ++e;
      c0 = 0;
      cur = nxt;
      if (e + 1 < e1) nxt = list[e + 1];
    } else {
      c0 += 32;
    }
  }
#pragma unroll
  for (int o = W; o < 32; o <<= 1) {
    P += __shfl_xor_sync(0xffffffffu, P, o);
    Gx += __shfl_xor_sync(0xffffffffu, Gx, o);
    Gy += __shfl_xor_sync(0xffffffffu, Gy, o);
    Gz += __shfl_xor_sync(0xffffffffu, Gz, o);
  }
  if (active && grp == 0) {
    const int bi = it.boff + ti;
    phi[bi] = P;
    grad[3 * bi + 0] = -Gx;
    grad[3 * bi + 1] = -Gy;
    grad[3 * bi + 2] = -Gz;
  }
}

__global__ void __launch_bounds__(32 * kP2PWarps)
    k_p2p64(const double4* __restrict__ body64, const P2PItem32* __restrict__ items, int nitems,
            const int* __restrict__ list_off, const P2PSrc64* __restrict__ list, double* __restrict__ phi,
            double* __restrict__ grad) {
  __shared__ double4 sbuf[kP2PWarps][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x * kP2PWarps + warp;
  if (item >= nitems) return;  // warp-uniform
  const P2PItem32 it = items[item];
  switch (it.lw) {
    case 5: p2p64_item<1>(body64, it, list_off, list, sbuf[warp], lane, phi, grad); break;
    case 4: p2p64_item<2>(body64, it, list_off, list, sbuf[warp], lane, phi, grad); break;
    case 3: p2p64_item<4>(body64, it, list_off, list, sbuf[warp], lane, phi, grad); break;
    default: p2p64_item<8>(body64, it, list_off, list, sbuf[warp], lane, phi, grad); break;
  }
}

// ---------------------------------------------------------------------------
// Close-pair refinement of the FP32 P2P (mixed form).
//
// The FP32 positions are leaf-relative, so each coordinate carries an
// absolute rounding of about 2^-24 of the leaf size, and a pair at distance
// d gets a relative error of about (leaf size / d) 2^-24 in its terms.  The
// relative L2 error of the whole gradient is dominated by the few closest
// pairs of the input (at N = 2^20 uniform bodies they sit ~1e-4 apart, a
// leaf is ~0.05 wide).  So the pairs closer than kCloseFrac times the larger
// of their two leaves' half edges are listed once per set-up (k_close_scan,
// a count pass and an emit pass in list order), and every pass replaces
// their FP32 terms by FP64 ones (k_close_fix): it recomputes the FP32 term
// of each listed pair with the P2P kernel's exact operation sequence (same
// FP32 inputs, same roundings, same rsqrt.approx) and adds the FP64 term
// minus it.  What remains of the FP32 term is its rounding inside the FP32
// partial sum, ~2^-24 of the term.
// ---------------------------------------------------------------------------
#ifndef CLOSE_FRAC
#define CLOSE_FRAC 0.125f
#endif
constexpr float kCloseFrac = CLOSE_FRAC;

// One warp per P2P work item, one lane per target (lanes >= nt idle); the
// lanes of an item share its list, so source loads are warp broadcasts.
// EMIT = false: cnt[t] = close sources of target t.  EMIT = true: the pairs
// (source body, list entry) of target t at pairs[off[t] ...], in list order.
template <bool EMIT>
__global__ void __launch_bounds__(256)
    k_close_scan(const float4* __restrict__ body32, const P2PItem32* __restrict__ items, int nitems,
                 const int* __restrict__ list_off, const P2PSrc32* __restrict__ list,
                 const LeafInfo* __restrict__ leaves, int* __restrict__ cnt, const int* __restrict__ off,
                 int2* __restrict__ pairs) {
  const int item = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (item >= nitems) return;
  const P2PItem32 it = items[item];
  if (lane >= it.nt) return;
  const int t = it.boff + lane;
  const float4 xt = body32[t];
  const float rt = (float)leaves[it.leaf].r;
  int c = 0;
  int pos = EMIT ? off[t] : 0;
  const int pend = EMIT ? off[t + 1] : 0;  // the count pass's total for t bounds the writes
  const int e1 = list_off[it.leaf + 1];
  const unsigned mask = __activemask();
  for (int e = list_off[it.leaf]; e < e1; ++e) {
    const P2PSrc32 s = list[e];
    const float rs = (float)leaves[s.leaf].r;
    const float rc = kCloseFrac * fmaxf(rt, rs);
    const float rc2 = rc * rc;
    const float px = xt.x - s.dx, py = xt.y - s.dy, pz = xt.z - s.dz;
    // the source leaf's box (half edge rs, a little margin for the FP32
    // rounding of the positions) is farther than rc from every target of
    // this warp: no close pair in it
    const float bx = fmaxf(fabsf(px) - 1.001f * rs, 0.f), by = fmaxf(fabsf(py) - 1.001f * rs, 0.f),
                bz = fmaxf(fabsf(pz) - 1.001f * rs, 0.f);
    if (!__any_sync(mask, bx * bx + by * by + bz * bz < rc2)) continue;
    for (int k = 0; k < s.bnum; ++k) {
      const float4 b = body32[s.boff + k];
      const float dx = px - b.x, dy = py - b.y, dz = pz - b.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (r2 < rc2 && !(s.self && s.boff + k == t)) {
        if (EMIT) {
          if (pos < pend) pairs[pos++] = make_int2(s.boff + k, e);
        } else
          ++c;
      }
    }
  }
  if (!EMIT) cnt[t] = c;
}

// One thread per target body (tree order).  cycle > 0: periodic, the pair's
// FP64 difference taken at its nearest image (a close pair is far closer
// than half a period, so that is the image its list entry carries).
__global__ void k_close_fix(const double4* __restrict__ body64, const float4* __restrict__ body32,
                            const P2PSrc32* __restrict__ list, const int* __restrict__ off,
                            const int2* __restrict__ pairs, int n, double cycle, double* __restrict__ phi,
                            double* __restrict__ grad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int b0 = off[t], b1 = off[t + 1];
  if (b0 == b1) return;
  const float4 xt = body32[t];
  const double4 yt = body64[t];
  double P = 0.0, Gx = 0.0, Gy = 0.0, Gz = 0.0;
  for (int k = b0; k < b1; ++k) {
    const int2 pr = pairs[k];
    const P2PSrc32 s = list[pr.y];
    // the FP32 terms exactly as k_p2p32 formed them
    const float4 b = body32[pr.x];
    const float px = xt.x - s.dx, py = xt.y - s.dy, pz = xt.z - s.dz;
    const float dx = __fadd_rn(px, -b.x), dy = __fadd_rn(py, -b.y), dz = __fadd_rn(pz, -b.z);
    float r2 = __fmul_rn(dz, dz);
    r2 = __fmaf_rn(dy, dy, r2);
    r2 = __fmaf_rn(dx, dx, r2);
    float ir = rsqrt_approx(r2);
    if (!(r2 > 0.f)) ir = 0.f;
    const float qir = __fmul_rn(b.w, ir);
    const float q3 = __fmul_rn(__fmul_rn(qir, ir), ir);
    // the FP64 terms of the pair
    const double4 y = body64[pr.x];
    double ex = yt.x - y.x, ey = yt.y - y.y, ez = yt.z - y.z;
    if (cycle > 0.0) {
      ex -= cycle * rint(ex / cycle);
      ey -= cycle * rint(ey / cycle);
      ez -= cycle * rint(ez / cycle);
    }
    const double rr = ex * ex + ey * ey + ez * ez;
    const double jr = rr > 0.0 ? rsqrt_nr<2>(rr) : 0.0;
    const double qjr = y.w * jr;
    const double q3d = qjr * jr * jr;
    P += qjr - (double)qir;
    Gx += q3d * ex - (double)q3 * (double)dx;
    Gy += q3d * ey - (double)q3 * (double)dy;
    Gz += q3d * ez - (double)q3 * (double)dz;
  }
  phi[t] += P;
  grad[3 * t + 0] -= Gx;
  grad[3 * t + 1] -= Gy;
  grad[3 * t + 2] -= Gz;
}

// ---------------------------------------------------------------------------
// P2M: check-surface potential of each leaf's bodies (FP64).  Surface points
// are unit * (2.95 r) + centre (kernel.cpp:336).  One block per leaf, two
// surface points per thread, the block sized to the surface (160 threads for
// the 296 points of P = 8) so that few lanes idle.
// ---------------------------------------------------------------------------
constexpr int kSurfThreads = 128;
constexpr int kCheckMaxThreads = 256;
constexpr int kCheckPer = 2;

template <int NR>
__global__ void __launch_bounds__(kCheckMaxThreads)
    k_p2m_check(const double4* __restrict__ body64, const LeafInfo* __restrict__ leaves,
                const double* __restrict__ surf_unit, int ns, double* __restrict__ out) {
  __shared__ double4 sb[kCheckMaxThreads];
  const LeafInfo L = leaves[blockIdx.x];
  const double R = L.r * 2.95;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i0 = 0; i0 < ns; i0 += nt * kCheckPer) {
    double yx[kCheckPer], yy[kCheckPer], yz[kCheckPer], acc[kCheckPer];
#pragma unroll
    for (int k = 0; k < kCheckPer; ++k) {
      const int i = i0 + tid + k * nt;
      const int ii = i < ns ? i : 0;
      yx[k] = surf_unit[3 * ii + 0] * R + L.cx;
      yy[k] = surf_unit[3 * ii + 1] * R + L.cy;
      yz[k] = surf_unit[3 * ii + 2] * R + L.cz;
      acc[k] = 0.0;
    }
    for (int b0 = 0; b0 < L.bnum; b0 += nt) {
      const int cnt = min(nt, L.bnum - b0);
      __syncthreads();
      if (tid < cnt) sb[tid] = body64[L.boff + b0 + tid];
      __syncthreads();
#pragma unroll 2
      for (int j = 0; j < cnt; ++j) {
        const double4 b = sb[j];
#pragma unroll
        for (int k = 0; k < kCheckPer; ++k) {
          const double dx = yx[k] - b.x, dy = yy[k] - b.y, dz = yz[k] - b.z;
          const double r2 = dx * dx + dy * dy + dz * dz;
          const double ir = r2 > 0.0 ? rsqrt_nr<NR>(r2) : 0.0;
          acc[k] += b.w * ir;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kCheckPer; ++k) {
      const int i = i0 + tid + k * nt;
      if (i < ns) out[(size_t)blockIdx.x * ns + i] = acc[k];
    }
  }
}

// ---------------------------------------------------------------------------
// L2P: potential and gradient at each leaf's bodies from the downward
// equivalent density on the 2.95 r surface (kernel.cpp:1461, 1469-1510), FP64.
// One block per leaf.  A leaf with fewer bodies than threads splits the
// surface points among G = threads / bnum groups of bnum threads (group g
// takes points g, g+G, ...) and sums the groups in shared memory, so that a
// 34-body leaf keeps 102 of 128 threads busy instead of 34.
// ---------------------------------------------------------------------------
template <int NR>
__global__ void __launch_bounds__(kSurfThreads)
    k_l2p_eval(const double4* __restrict__ body64, const LeafInfo* __restrict__ leaves,
               const double* __restrict__ surf_unit, int ns, const double* __restrict__ q_down,
               double* __restrict__ phi, double* __restrict__ grad) {
  extern __shared__ double4 sy[];  // ns entries
  __shared__ double red[4][kSurfThreads];
  const LeafInfo L = leaves[blockIdx.x];
  const double R = L.r * 2.95;
  for (int i = threadIdx.x; i < ns; i += blockDim.x)
    sy[i] = make_double4(surf_unit[3 * i] * R + L.cx, surf_unit[3 * i + 1] * R + L.cy,
                         surf_unit[3 * i + 2] * R + L.cz, q_down[(size_t)blockIdx.x * ns + i]);
  __syncthreads();
  const int bnum = L.bnum;
  if (bnum <= 0) return;  // block-uniform
  const int B = bnum < kSurfThreads ? bnum : kSurfThreads;
  const int G = kSurfThreads / B;
  const int grp = threadIdx.x / B, tl = threadIdx.x - grp * B;
  for (int t0 = 0; t0 < bnum; t0 += B) {
    double p = 0, gx = 0, gy = 0, gz = 0;
    const int t = t0 + tl;
    if (grp < G && t < bnum) {
      const double4 x = body64[L.boff + t];
      for (int i = grp; i < ns; i += G) {
        const double4 y = sy[i];
        const double dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double ir = r2 > 0.0 ? rsqrt_nr<NR>(r2) : 0.0;
        const double qir = y.w * ir;
        p += qir;
        const double q3 = qir * ir * ir;
        gx += q3 * dx;
        gy += q3 * dy;
        gz += q3 * dz;
      }
    }
    if (G > 1) {
      red[0][threadIdx.x] = p;
      red[1][threadIdx.x] = gx;
      red[2][threadIdx.x] = gy;
      red[3][threadIdx.x] = gz;
      __syncthreads();
      if (grp == 0) {
        for (int g2 = 1; g2 < G; ++g2) {
          const int o = g2 * B + tl;
          p += red[0][o];
          gx += red[1][o];
          gy += red[2][o];
          gz += red[3][o];
        }
      }
      __syncthreads();
    }
    if (grp == 0 && t < bnum) {
      const int b = L.boff + t;
      phi[b] = p;
      grad[3 * b + 0] = -gx;
      grad[3 * b + 1] = -gy;
      grad[3 * b + 2] = -gz;
    }
  }
}

// ---------------------------------------------------------------------------
// Batched FP64 operator application:
//   C[outrow[r]][n] = beta*C + scale[r] * sum_s sum_j A[inrow[r*S+s]][j] B[g][s][j][n]
// 128x64 output tiles, 16-deep K steps, 8x4 outputs per thread; the next K
// step's A rows (gathered through inrow) and B panel are loaded into
// registers while the current step is multiplied out of shared memory.
// ---------------------------------------------------------------------------
constexpr int kTM = APPLY_TM, kTN = 64, kTK = 16;
constexpr int kRPT = kTM / 16;  // output rows per thread

__global__ void __launch_bounds__(256, 2) k_apply_f64(ApplyBatch b) {
  __shared__ double As[kTK][kTM + 1];
  __shared__ double Bs[kTK][kTN];
  const int g = blockIdx.z;
  const int rbeg = b.group_off[g], rend = b.group_off[g + 1];
  const int r0 = rbeg + blockIdx.y * kTM;
  const int c0 = blockIdx.x * kTN;
  if (r0 >= rend) return;  // block-uniform
  const int ns = b.ns, S = b.S;
  const double* Bg = b.B + (size_t)g * S * ns * ns;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int nkt = (ns + kTK - 1) / kTK, total = S * nkt;
  // this thread loads A rows ty + 16u (the rows it also writes) at k = tx,
  // and B elements tid + 256u of the 16x64 panel
  int src[kRPT];
  double ra[kRPT], rb[4];
  int s_cur = 0;
  auto load_src = [&](int s) {
#pragma unroll
    for (int u = 0; u < kRPT; ++u) {
      const int row = r0 + ty + 16 * u;
      src[u] = row < rend ? b.inrow[(size_t)row * S + s] : -1;
    }
  };
  auto fetch = [&](int kt) {
    const int s = kt / nkt, j0 = (kt - s * nkt) * kTK;
    const int j = j0 + tx;
#pragma unroll
    for (int u = 0; u < kRPT; ++u) ra[u] = (src[u] >= 0 && j < ns) ? b.A[(size_t)src[u] * ns + j] : 0.0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + 256 * u;
      const int jj = j0 + (e >> 6), n = c0 + (e & 63);
      rb[u] = (jj < ns && n < ns) ? Bg[((size_t)s * ns + jj) * ns + n] : 0.0;
    }
  };
#if APPLY_MMA
  static_assert(kTM == 64, "the tensor-core path tiles 64 rows as 2 x 4 warps");
  const int lane = tid & 31, wm = (tid >> 5) & 1, wn = tid >> 6;
  double dacc[4][2][2];
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) dacc[mt][nt][0] = dacc[mt][nt][1] = 0.0;
#else
  double acc[kRPT][4];
#pragma unroll
  for (int i = 0; i < kRPT; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
#endif
  load_src(0);
  fetch(0);
  for (int kt = 0; kt < total; ++kt) {
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kRPT; ++u) As[tx][ty + 16 * u] = ra[u];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + 256 * u;
      Bs[e >> 6][e & 63] = rb[u];
    }
    __syncthreads();
    if (kt + 1 < total) {
      const int s_next = (kt + 1) / nkt;
      if (s_next != s_cur) {
        s_cur = s_next;
        load_src(s_next);
      }
      fetch(kt + 1);
    }
#if APPLY_MMA
    // FP64 tensor-core steps: mma.sync m8n8k4 over this warp's 32x16 block
    // (4 x 2 tiles of 8x8).  Fragments: A[m][k] at m = lane/4, k = lane%4;
    // B[k][n] at k = lane%4, n = lane/4; D[m][n] at m = lane/4,
    // n = 2 (lane%4) + {0, 1}.
#pragma unroll
    for (int k4 = 0; k4 < kTK; k4 += 4) {
      double fa[4], fb[2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) fa[mt] = As[k4 + (lane & 3)][wm * 32 + mt * 8 + (lane >> 2)];
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) fb[nt] = Bs[k4 + (lane & 3)][wn * 16 + nt * 8 + (lane >> 2)];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
          asm volatile(
              "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
              : "+d"(dacc[mt][nt][0]), "+d"(dacc[mt][nt][1])
              : "d"(fa[mt]), "d"(fb[nt]));
    }
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int row = r0 + wm * 32 + mt * 8 + (lane >> 2);
    if (row >= rend) continue;
    const int o = b.outrow[row];
    const double sc = b.scale ? b.scale[row] : 1.0;
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int n = c0 + wn * 16 + nt * 8 + 2 * (lane & 3) + i;
        if (n >= ns) continue;
        double* cp = b.C + (size_t)o * ns + n;
        *cp = b.beta ? *cp + sc * dacc[mt][nt][i] : sc * dacc[mt][nt][i];
      }
  }
}
#else
#pragma unroll
    for (int k = 0; k < kTK; ++k) {
      double a[kRPT], bb[4];
#pragma unroll
      for (int i = 0; i < kRPT; ++i) a[i] = As[k][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bb[j] = Bs[k][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < kRPT; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
    }
  }
#pragma unroll
  for (int i = 0; i < kRPT; ++i) {
    const int row = r0 + ty + 16 * i;
    if (row >= rend) continue;
    const int o = b.outrow[row];
    const double sc = b.scale ? b.scale[row] : 1.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = c0 + tx + 16 * j;
      if (n >= ns) continue;
      double* cp = b.C + (size_t)o * ns + n;
      *cp = b.beta ? *cp + sc * acc[i][j] : sc * acc[i][j];
    }
  }
}
#endif

// ---------------------------------------------------------------------------
// The same batched application on the FP64 tensor path: 64x64 output tiles
// per 128-thread block (2 x 2 warps of 32x32, each 4 x 4 mma.sync m8n8k4
// f64 tiles), A rows (gathered through inrow) and the B panel moved into
// shared memory by cp.async through a three-stage ring, so that the loads of
// K step t+2 are in flight while step t is multiplied.  Products and sums
// are IEEE FP64 as in the SIMT kernel; only the summation order differs.
// Every 16-byte copy is in bounds or zero-filled (ns is even: 6(P-1)^2+2).
// ---------------------------------------------------------------------------
constexpr int kGM = 64, kGN = 64, kGK = 16, kGStages = 3, kGThreads = 128;
constexpr int kAPitch = kGK + 4;  // doubles per A row in shared memory (conflict-free fragments)
constexpr int kBPitch = kGN + 4;  // doubles per B row
constexpr int kAStage = kGM * kAPitch, kBStage = kGK * kBPitch;
[[maybe_unused]] constexpr size_t kGSmem = sizeof(double) * kGStages * (kAStage + kBStage);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int nbytes = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kGThreads) k_apply_f64_tc(ApplyBatch b) {
  extern __shared__ __align__(16) double gsm[];
  double* As = gsm;
  double* Bs = gsm + kGStages * kAStage;
  const int g = blockIdx.z;
  const int rbeg = b.group_off[g], rend = b.group_off[g + 1];
  const int r0 = rbeg + blockIdx.y * kGM;
  const int c0 = blockIdx.x * kGN;
  if (r0 >= rend) return;  // block-uniform
  const int ns = b.ns, S = b.S;
  const double* Bg = b.B + (size_t)g * S * ns * ns;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int nkt = (ns + kGK - 1) / kGK, total = S * nkt;
  // copies of this thread: A chunk e = tid + 128u -> row e/8, doubles 2(e%8)..+1;
  // B chunk e -> K row e/32, columns 2(e%32)..+1
  int srow[4];
  int s_cur = -1;
  auto issue = [&](int kt) {
    const int s = kt / nkt, j0 = (kt - s * nkt) * kGK;
    if (s != s_cur) {
      s_cur = s;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int row = r0 + ((tid + kGThreads * u) >> 3);
        srow[u] = row < rend ? b.inrow[(size_t)row * S + s] : -1;
      }
    }
    double* as = As + (kt % kGStages) * kAStage;
    double* bs = Bs + (kt % kGStages) * kBStage;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + kGThreads * u;
      const int r = e >> 3, ch = e & 7, j = j0 + 2 * ch;
      const bool ok = srow[u] >= 0 && j < ns;
      cp_async16(as + r * kAPitch + 2 * ch, ok ? b.A + (size_t)srow[u] * ns + j : b.A, ok);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + kGThreads * u;
      const int kr = e >> 5, ch = e & 31, jj = j0 + kr, n = c0 + 2 * ch;
      const bool ok = jj < ns && n < ns;
      cp_async16(bs + kr * kBPitch + 2 * ch, ok ? Bg + ((size_t)s * ns + jj) * ns + n : Bg, ok);
    }
  };
  double acc[4][4][2];
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
#pragma unroll
  for (int st = 0; st < kGStages - 1; ++st) {
    if (st < total) issue(st);
    cp_async_commit();
  }
  for (int kt = 0; kt < total; ++kt) {
    cp_async_wait<kGStages - 2>();
    __syncthreads();  // step kt is in shared memory; step kt-1's buffer is free
    if (kt + kGStages - 1 < total) issue(kt + kGStages - 1);
    cp_async_commit();
    const double* as = As + (kt % kGStages) * kAStage + (wm * 32 + (lane >> 2)) * kAPitch + (lane & 3);
    const double* bs = Bs + (kt % kGStages) * kBStage + (lane & 3) * kBPitch + wn * 32 + (lane >> 2);
#pragma unroll
    for (int k4 = 0; k4 < kGK; k4 += 4) {
      double fa[4], fb[4];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) fa[mt] = as[mt * 8 * kAPitch + k4];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) fb[nt] = bs[k4 * kBPitch + nt * 8];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma8x8x4(acc[mt][nt], fa[mt], fb[nt]);
    }
  }
  cp_async_wait<0>();
  // D fragment: row lane/4, columns 2 (lane%4) + {0, 1} of each 8x8 tile
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int row = r0 + wm * 32 + mt * 8 + (lane >> 2);
    if (row >= rend) continue;
    const int o = b.outrow[row];
    const double sc = b.scale ? b.scale[row] : 1.0;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int n = c0 + wn * 32 + nt * 8 + 2 * (lane & 3);
      if (n >= ns) continue;  // n even, ns even: n + 1 < ns as well
      double2* cp = reinterpret_cast<double2*>(b.C + (size_t)o * ns + n);
      double2 v = make_double2(sc * acc[mt][nt][0], sc * acc[mt][nt][1]);
      if (b.beta) {
        const double2 c = *cp;
        v.x += c.x;
        v.y += c.y;
      }
      *cp = v;
    }
  }
}

// Sibling sum of the per-child M2M products, in crange order
// (m2m_precompute accumulates child by child, kernel.cpp:398-403).
__global__ void k_sum_children(const int* __restrict__ list, int nparents, const double* __restrict__ Y, int ns,
                               double* __restrict__ q) {
  const int pidx = blockIdx.x;
  if (pidx >= nparents) return;
  const int par = list[3 * pidx], coff = list[3 * pidx + 1], cnum = list[3 * pidx + 2];
  for (int n = threadIdx.x; n < ns; n += blockDim.x) {
    double acc = 0.0;
    for (int c = 0; c < cnum; ++c) acc += Y[(size_t)(coff + c) * ns + n];
    q[(size_t)par * ns + n] = acc;
  }
}

// ---------------------------------------------------------------------------
// FFT-M2L.  Grids are N = 2P-1 points per edge, stored [z][y][x]; spectra are
// the r2c half-spectrum [kz][ky][kx], kx < P.  The twiddle table holds
// w^m = exp(-2 pi i m / N) for m < N.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void cmad(T& re, T& im, T ar, T ai, T br, T bi) {
  re = fma(ar, br, re);
  re = fma(-ai, bi, re);
  im = fma(ar, bi, im);
  im = fma(ai, br, im);
}

// up: one block per (source parent, group of sp child slots): scatter each
// child's equivalent density onto the [0,P)^3 corner of the grid
// (surf_conv_idx_map_up, kernel.cpp:1246-1252, 1304-1315) and take its
// forward DFT separably (x, then y, then z).  The z pass of all sp slots runs
// together so that each frequency's sp values are written contiguously into
// the frequency-major spectrum Q[f][src][slot].
// items: 10 ints per block = src, first slot, child cell per slot (-1 = none).
// PP > 0 fixes P at compile time (cheap index arithmetic); PP = 0 takes it
// from the argument.
template <typename T, int PP>
__global__ void __launch_bounds__(256)
    k_m2l_up(const double* __restrict__ q_equiv, const int* __restrict__ items,
             const int* __restrict__ surf_ijk, const double* __restrict__ twiddle, int P_, int ns, int nsrc,
             int sp, T* __restrict__ Q) {
  const int P = PP > 0 ? PP : P_;
  extern __shared__ unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int N = 2 * P - 1;
  const int P3 = P * P * P, Nf = N * N * P, PNP = P * N * P;
  T* W = sm;                       // N*N complex: W[k][n] = w^(k n mod N)
  T* cube = W + 2 * N * N;         // P^3
  T* A = cube + P3;                // P^3 complex: [z][y][kx]
  T* Bm = A + 2 * P3;              // sp * P*N*P complex: [slot][z][ky][kx]
  const int* it = items + 10 * blockIdx.x;
  const int src = it[0], slot0 = it[1];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < N * N; e += nt) {
    const int m = ((e / N) * (e % N)) % N;
    W[2 * e] = (T)twiddle[2 * m];
    W[2 * e + 1] = (T)twiddle[2 * m + 1];
  }
  for (int j = 0; j < sp; ++j) {
    const int child = it[2 + j];
    T* Bj = Bm + 2 * (size_t)j * PNP;
    if (child < 0) {
      for (int e = tid; e < 2 * PNP; e += nt) Bj[e] = T(0);
      continue;
    }
    for (int e = tid; e < P3; e += nt) cube[e] = T(0);
    __syncthreads();
    for (int i = tid; i < ns; i += nt) {
      const int x = surf_ijk[3 * i], y = surf_ijk[3 * i + 1], z = surf_ijk[3 * i + 2];
      cube[(z * P + y) * P + x] = (T)q_equiv[(size_t)child * ns + i];
    }
    __syncthreads();
    for (int e = tid; e < P3; e += nt) {
      const int z = e / (P * P), y = (e / P) % P, kx = e % P;
      T re = 0, im = 0;
      const T* row = cube + (z * P + y) * P;
      const T* wk = W + 2 * kx * N;
      for (int x = 0; x < P; ++x) {
        re = fma(row[x], wk[2 * x], re);
        im = fma(row[x], wk[2 * x + 1], im);
      }
      A[2 * e] = re;
      A[2 * e + 1] = im;
    }
    __syncthreads();
    for (int e = tid; e < PNP; e += nt) {
      const int z = e / (N * P), ky = (e / P) % N, kx = e % P;
      T re = 0, im = 0;
      const T* wk = W + 2 * ky * N;
      for (int y = 0; y < P; ++y) {
        const int a = (z * P + y) * P + kx;
        cmad(re, im, A[2 * a], A[2 * a + 1], wk[2 * y], wk[2 * y + 1]);
      }
      Bj[2 * e] = re;
      Bj[2 * e + 1] = im;
    }
    __syncthreads();
  }
  __syncthreads();
  using V2 = typename Cplx2<T>::type;  // two complex values
  for (int f = tid; f < Nf; f += nt) {
    const int kz = f / (N * P), ky = (f / P) % N, kx = f % P;
    const T* wk = W + 2 * kz * N;
    for (int j = 0; j < sp; j += 2) {
      T* out = Q + 2 * q8_index<T>(f, src, slot0 + j, nsrc);
      T re0 = 0, im0 = 0, re1 = 0, im1 = 0;
      const T* B0 = Bm + 2 * (size_t)j * PNP;
      const T* B1 = B0 + 2 * (size_t)PNP;
      for (int z = 0; z < P; ++z) {
        const int b = (z * N + ky) * P + kx;
        cmad(re0, im0, B0[2 * b], B0[2 * b + 1], wk[2 * z], wk[2 * z + 1]);
        if (j + 1 < sp) cmad(re1, im1, B1[2 * b], B1[2 * b + 1], wk[2 * z], wk[2 * z + 1]);
      }
      if (j + 1 < sp) {
        V2 v;
        v.x = re0;
        v.y = im0;
        v.z = re1;
        v.w = im1;
        *reinterpret_cast<V2*>(out) = v;
      } else {
        out[0] = re0;
        out[1] = im0;
      }
    }
  }
}

// The up and down kernels above with register blocking, for the orders P
// fixed at compile time: the sp children of a block go through each DFT pass
// together, and a thread keeps one input line of the pass (the values along
// the transformed axis) in registers and forms every output of that line, the
// twiddles read as shared-memory broadcasts.  Each output sums its terms in
// the same order as k_m2l_up / k_m2l_down, so the results are the same bit
// for bit; the shared-memory traffic per multiply-add falls from two loads
// to about one broadcast.
template <typename T, int PP>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? UP_RB_MINB : 2)
    k_m2l_up_rb(const double* __restrict__ q_equiv, const int* __restrict__ items, const int* __restrict__ surf_ijk,
                const double* __restrict__ twiddle, int ns, int nsrc, int sp, T* __restrict__ Q) {
  constexpr int P = PP, N = 2 * P - 1, P3 = P * P * P, PNP = P * N * P;
  // the last pass: a thread per (pair of slots, ky, kx, range of kz)
  constexpr int KC = (128 / (N * P)) < 1 ? 1 : ((128 / (N * P)) > N ? N : 128 / (N * P));
  constexpr int KH = (N + KC - 1) / KC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the twiddle table padded to 8 values, so that A and the cube (read as
  // 16-byte vectors) start on 16-byte boundaries
  constexpr int WSZ = (2 * N * N + 7) / 8 * 8;
  T* W = reinterpret_cast<T*>(smem_raw);  // N*N complex: W[k][n] = w^(k n mod N)
  T* A = W + WSZ;                         // sp * P^3 complex: [slot][z][y][kx]
  T* cube = A + 2 * (size_t)sp * P3;      // sp * P^3, read by the first pass only
  T* Bm = cube;                           // sp * P*N*P complex: [slot][z][ky][kx], after it
  const int* it = items + 10 * blockIdx.x;
  const int src = it[0], slot0 = it[1];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < N * N; e += nt) {
    const int m = ((e / N) * (e % N)) % N;
    W[2 * e] = (T)twiddle[2 * m];
    W[2 * e + 1] = (T)twiddle[2 * m + 1];
  }
  for (int e = tid; e < sp * P3; e += nt) cube[e] = T(0);
  __syncthreads();
  for (int e = tid; e < sp * ns; e += nt) {
    const int j = e / ns, i = e - j * ns;
    const int child = it[2 + j];
    if (child < 0) continue;  // an absent child: zero spectra
    const int x = surf_ijk[3 * i], y = surf_ijk[3 * i + 1], z = surf_ijk[3 * i + 2];
    cube[(size_t)j * P3 + (z * P + y) * P + x] = (T)q_equiv[(size_t)child * ns + i];
  }
  __syncthreads();
  // x -> kx: a thread per (slot, z, y)
  for (int e = tid; e < sp * P * P; e += nt) {
    const int j = e / (P * P), zy = e - j * P * P;
    const T* row = cube + (size_t)j * P3 + zy * P;
    T r[P];
    if constexpr (sizeof(T) == 4 && P % 4 == 0) {
#pragma unroll
      for (int x = 0; x < P; x += 4) {
        const float4 v = *reinterpret_cast<const float4*>(row + x);
        r[x] = v.x;
        r[x + 1] = v.y;
        r[x + 2] = v.z;
        r[x + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int x = 0; x < P; ++x) r[x] = row[x];
    }
    T* a = A + 2 * ((size_t)j * P3 + zy * P);
#pragma unroll
    for (int kx = 0; kx < P; ++kx) {
      const T* wk = W + 2 * kx * N;
      T re = 0, im = 0;
#pragma unroll
      for (int x = 0; x < P; ++x) {
        re = fma(r[x], wk[2 * x], re);
        im = fma(r[x], wk[2 * x + 1], im);
      }
      a[2 * kx] = re;
      a[2 * kx + 1] = im;
    }
  }
  __syncthreads();
  // y -> ky: a thread per (slot, z, kx)
  for (int e = tid; e < sp * P * P; e += nt) {
    const int j = e / (P * P), z = (e / P) % P, kx = e % P;
    T ar[P], ai[P];
#pragma unroll
    for (int y = 0; y < P; ++y) {
      const T* q = A + 2 * ((size_t)j * P3 + (z * P + y) * P + kx);
      ar[y] = q[0];
      ai[y] = q[1];
    }
    T* b = Bm + 2 * ((size_t)j * PNP + z * N * P + kx);
#pragma unroll
    for (int ky = 0; ky < N; ++ky) {
      const T* wk = W + 2 * ky * N;
      T re = 0, im = 0;
#pragma unroll
      for (int y = 0; y < P; ++y) cmad(re, im, ar[y], ai[y], wk[2 * y], wk[2 * y + 1]);
      b[2 * ky * P] = re;
      b[2 * ky * P + 1] = im;
    }
  }
  __syncthreads();
  // z -> kz: a thread per (pair of slots, ky, kx, range of kz); the two
  // slots of a pair written together as in k_m2l_up
  using V2 = typename Cplx2<T>::type;
  const int npair = (sp + 1) / 2;
  for (int e = tid; e < npair * N * P * KC; e += nt) {
    const int jp = e / (N * P * KC), c = (e / (N * P)) % KC, ky = (e / P) % N, kx = e % P;
    const int j = 2 * jp;
    const bool two = j + 1 < sp;
    T br[2][P], bi[2][P];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int z = 0; z < P; ++z) {
        if (u == 0 || two) {
          const T* q = Bm + 2 * ((size_t)(j + u) * PNP + (z * N + ky) * P + kx);
          br[u][z] = q[0];
          bi[u][z] = q[1];
        } else {
          br[u][z] = bi[u][z] = T(0);
        }
      }
    const int kz1 = (c + 1) * KH < N ? (c + 1) * KH : N;
    for (int kz = c * KH; kz < kz1; ++kz) {
      const T* wk = W + 2 * kz * N;
      const int f = (kz * N + ky) * P + kx;
      T* out = Q + 2 * q8_index<T>(f, src, slot0 + j, nsrc);
      T re0 = 0, im0 = 0, re1 = 0, im1 = 0;
#pragma unroll
      for (int z = 0; z < P; ++z) {
        cmad(re0, im0, br[0][z], bi[0][z], wk[2 * z], wk[2 * z + 1]);
        if (two) cmad(re1, im1, br[1][z], bi[1][z], wk[2 * z], wk[2 * z + 1]);
      }
      if (two) {
        V2 v;
        v.x = re0;
        v.y = im0;
        v.z = re1;
        v.w = im1;
        *reinterpret_cast<V2*>(out) = v;
      } else {
        out[0] = re0;
        out[1] = im0;
      }
    }
  }
}

template <typename T, int PP>
__global__ void __launch_bounds__(256)
    k_m2l_down_rb(const T* __restrict__ Pk, const int* __restrict__ items, const double* __restrict__ tscale,
                  const int* __restrict__ surf_ijk, const double* __restrict__ twiddle, int ns, int ntar, int sp,
                  double* __restrict__ p_check) {
  constexpr int P = PP, N = 2 * P - 1, P3 = P * P * P, PNP = P * N * P, Nf = N * N * P;
  extern __shared__ unsigned char smem_raw[];
  T* W = reinterpret_cast<T*>(smem_raw);  // P*N complex: W[o][k] = conj(w)^(k (P-1+o) mod N)
  T* Y1 = W + 2 * P * N;                  // sp * P*N*P complex: [slot][zo][ky][kx]
  T* X = Y1 + 2 * (size_t)sp * PNP;       // sp * Nf complex: [slot][f]; later Y2
  T* Y2 = X;                              // sp * P^3 complex: [slot][zo][yo][kx]
  const int* it = items + 10 * blockIdx.x;
  const int tar = it[0], slot0 = it[1];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < P * N; e += nt) {
    const int o = e / N, k = e % N;
    const int m = (k * (P - 1 + o)) % N;
    W[2 * e] = (T)twiddle[2 * m];
    W[2 * e + 1] = -(T)twiddle[2 * m + 1];
  }
  if (sp >= 2) {
    using V2 = typename Cplx2<T>::type;
    const int hp = sp / 2;
    for (int e = tid; e < Nf * hp; e += nt) {
      const int f = e / hp, j = 2 * (e % hp);
      const V2 v = *reinterpret_cast<const V2*>(Pk + (((size_t)f * ntar + tar) * 8 + slot0 + j) * 2);
      X[2 * ((size_t)j * Nf + f)] = v.x;
      X[2 * ((size_t)j * Nf + f) + 1] = v.y;
      X[2 * ((size_t)(j + 1) * Nf + f)] = v.z;
      X[2 * ((size_t)(j + 1) * Nf + f) + 1] = v.w;
    }
  } else {
    for (int f = tid; f < Nf; f += nt) {
      const T* in = Pk + (((size_t)f * ntar + tar) * 8 + slot0) * 2;
      X[2 * f] = in[0];
      X[2 * f + 1] = in[1];
    }
  }
  __syncthreads();
  // kz -> zo (zo < P only): a thread per (slot, ky, kx)
  for (int e = tid; e < sp * N * P; e += nt) {
    const int j = e / (N * P), ky = (e / P) % N, kx = e % P;
    T xr[N], xi[N];
#pragma unroll
    for (int kz = 0; kz < N; ++kz) {
      const T* q = X + 2 * ((size_t)j * Nf + (kz * N + ky) * P + kx);
      xr[kz] = q[0];
      xi[kz] = q[1];
    }
#pragma unroll
    for (int zo = 0; zo < P; ++zo) {
      const T* wo = W + 2 * zo * N;
      T re = 0, im = 0;
#pragma unroll
      for (int kz = 0; kz < N; ++kz) cmad(re, im, xr[kz], xi[kz], wo[2 * kz], wo[2 * kz + 1]);
      T* y1 = Y1 + 2 * ((size_t)j * PNP + (zo * N + ky) * P + kx);
      y1[0] = re;
      y1[1] = im;
    }
  }
  __syncthreads();  // X is read: its space becomes Y2
  // ky -> yo (yo < P): a thread per (slot, zo, kx)
  for (int e = tid; e < sp * P * P; e += nt) {
    const int j = e / (P * P), zo = (e / P) % P, kx = e % P;
    T yr[N], yi[N];
#pragma unroll
    for (int ky = 0; ky < N; ++ky) {
      const T* q = Y1 + 2 * ((size_t)j * PNP + (zo * N + ky) * P + kx);
      yr[ky] = q[0];
      yi[ky] = q[1];
    }
#pragma unroll
    for (int yo = 0; yo < P; ++yo) {
      const T* wo = W + 2 * yo * N;
      T re = 0, im = 0;
#pragma unroll
      for (int ky = 0; ky < N; ++ky) cmad(re, im, yr[ky], yi[ky], wo[2 * ky], wo[2 * ky + 1]);
      T* y2 = Y2 + 2 * ((size_t)j * P3 + (zo * P + yo) * P + kx);
      y2[0] = re;
      y2[1] = im;
    }
  }
  __syncthreads();
  // kx -> xo at the check-surface points, real part; p_check += value * scale
  const double sc = tscale[tar];
  for (int e = tid; e < sp * ns; e += nt) {
    const int j = e / ns, i = e - j * ns;
    const int child = it[2 + j];
    if (child < 0) continue;
    const int xo = surf_ijk[3 * i], yo = surf_ijk[3 * i + 1], zo = surf_ijk[3 * i + 2];
    const T* row = Y2 + 2 * ((size_t)j * P3 + (zo * P + yo) * P);
    const T* wo = W + 2 * xo * N;
    T acc = 0;
    // Re(Y * conj(w)^m) summed over kx >= 1, doubled for the missing half
    for (int kx = 1; kx < P; ++kx) {
      acc = fma(row[2 * kx], wo[2 * kx], acc);
      acc = fma(-row[2 * kx + 1], wo[2 * kx + 1], acc);
    }
    const T v = row[0] + T(2) * acc;
    p_check[(size_t)child * ns + i] += (double)v * sc;
  }
}

// Hadamard 8x8 (hadamard_8x8 + c2c_8x8x2_avx, kernel.cpp:1012-1082, c2c.h:201-296):
//   Pk[f][t][itar] = sum_d sum_isrc G[f][d][isrc][itar] * Q[f][src(t,d)][isrc]
// A block holds one frequency's 26x64 kernel coefficients in shared memory
// (every coefficient read is a broadcast) and each thread owns TT targets of
// that frequency: one coefficient read feeds TT targets, and each (target,
// direction) reads one 64-byte source row with sector loads.  L1 wavefronts
// per FMA fall as 1/(4 TT) + 1/16, which is what bounds this kernel.
// FP32 partial sums over DF directions are accumulated into FP64.
template <typename T> struct HadCfg;
template <> struct HadCfg<float> {
  static constexpr int TT = HAD_TT, DF = HAD_DF, THREADS = 256 / HAD_TT, MINB = HAD_MINB;
  static constexpr bool ACC_SMEM = HAD_ACC_SMEM;
};
template <> struct HadCfg<double> {
  static constexpr int TT = 1, DF = 1, THREADS = 256, MINB = 1;
  static constexpr bool ACC_SMEM = false;
};

template <typename T>
__device__ __forceinline__ void load_row8(const T* qrow, typename Cplx<T>::type (&q)[8]) {
  constexpr int kPer = 32 / sizeof(T);  // values per 32-byte sector
#pragma unroll
  for (int c = 0; c < 16 / kPer; ++c) {
    T v[kPer];
    ld_sector(qrow + c * kPer, v);
#pragma unroll
    for (int k = 0; k < kPer / 2; ++k) {
      q[c * kPer / 2 + k].x = v[2 * k];
      q[c * kPer / 2 + k].y = v[2 * k + 1];
    }
  }
}

template <typename T, int TT>
__device__ __forceinline__ void had_rows(const typename Cplx<T>::type* __restrict__ Qf, int nsrc, const int (&sd)[TT],
                                         typename Cplx<T>::type (&q)[TT][8]) {
#pragma unroll
  for (int u = 0; u < TT; ++u) {
    if (sd[u] >= 0) {
      if constexpr (Q8_CHUNKED && (sizeof(T) == 4 || Q8_CHUNKED64)) {
        // chunk c of this source: slots per*c .. per*c+per-1, one sector
        constexpr int per = 32 / (2 * sizeof(T)), nch = 8 / per;
#pragma unroll
        for (int c = 0; c < nch; ++c) {
          const T* qc = reinterpret_cast<const T*>(Qf) + ((size_t)c * nsrc + sd[u]) * 2 * per;
          T v[2 * per];
          ld_sector(qc, v);
#pragma unroll
          for (int k = 0; k < per; ++k) {
            q[u][per * c + k].x = v[2 * k];
            q[u][per * c + k].y = v[2 * k + 1];
          }
        }
      } else {
        load_row8<T>(reinterpret_cast<const T*>(Qf + (size_t)sd[u] * 8), q[u]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) q[u][i].x = q[u][i].y = T(0);
    }
  }
}

template <typename T, int TT>
__device__ __forceinline__ void had_index(const int* __restrict__ tsrcT, int d, int t0, int nt, int ntar,
                                          int (&sd)[TT]) {
#pragma unroll
  for (int u = 0; u < TT; ++u) {
    const int t = t0 + u * nt;
    sd[u] = t < ntar ? tsrcT[d * ntar + t] : -1;
  }
}

template <typename T, int TT>
__device__ __forceinline__ void had_mac(const typename Cplx<T>::type* __restrict__ g, const int (&sd)[TT],
                                        const typename Cplx<T>::type (&q)[TT][8], T (&pr)[TT][8], T (&pi)[TT][8]) {
  bool any = false;
#pragma unroll
  for (int u = 0; u < TT; ++u) any |= sd[u] >= 0;
  if (!any) return;
#pragma unroll
  for (int isrc = 0; isrc < 8; ++isrc)
#pragma unroll
    for (int itar = 0; itar < 8; itar += 2) {
      const typename Cplx2<T>::type gv = *reinterpret_cast<const typename Cplx2<T>::type*>(g + isrc * 8 + itar);
#pragma unroll
      for (int u = 0; u < TT; ++u) {
        cmad(pr[u][itar], pi[u][itar], gv.x, gv.y, q[u][isrc].x, q[u][isrc].y);
        cmad(pr[u][itar + 1], pi[u][itar + 1], gv.z, gv.w, q[u][isrc].x, q[u][isrc].y);
      }
    }
}

// The same product in packed FP32x2 FMAs, with the coefficients of an itar
// pair laid (gr0, gr1, gi0, gi1) in shared memory: per output the FMAs and
// their order are those of cmad, so the sums are bit for bit the scalar ones.
template <int TT>
__device__ __forceinline__ void had_mac_f2(const float4* __restrict__ g, const int (&sd)[TT], const float2 (&q)[TT][8],
                                           float (&pr)[TT][8], float (&pi)[TT][8]) {
  bool any = false;
#pragma unroll
  for (int u = 0; u < TT; ++u) any |= sd[u] >= 0;
  if (!any) return;
#pragma unroll
  for (int isrc = 0; isrc < 8; ++isrc) {
    float2 qr[TT], qi[TT], nqi[TT];
#pragma unroll
    for (int u = 0; u < TT; ++u) {
      qr[u] = make_float2(q[u][isrc].x, q[u][isrc].x);
      qi[u] = make_float2(q[u][isrc].y, q[u][isrc].y);
      nqi[u] = make_float2(-q[u][isrc].y, -q[u][isrc].y);
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const float4 gv = g[isrc * 4 + p];
      const float2 gr = make_float2(gv.x, gv.y), gi = make_float2(gv.z, gv.w);
#pragma unroll
      for (int u = 0; u < TT; ++u) {
        float2 re = make_float2(pr[u][2 * p], pr[u][2 * p + 1]);
        float2 im = make_float2(pi[u][2 * p], pi[u][2 * p + 1]);
        re = __ffma2_rn(gr, qr[u], re);
        re = __ffma2_rn(gi, nqi[u], re);
        im = __ffma2_rn(gr, qi[u], im);
        im = __ffma2_rn(gi, qr[u], im);
        pr[u][2 * p] = re.x;
        pr[u][2 * p + 1] = re.y;
        pi[u][2 * p] = im.x;
        pi[u][2 * p + 1] = im.y;
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(HadCfg<T>::THREADS, HadCfg<T>::MINB)
    k_m2l_hadamard8(const T* __restrict__ Q, const T* __restrict__ G, const int* __restrict__ tsrcT, int ntar,
                    int nsrc, int Nf, T* __restrict__ Pk) {
  using C2 = typename Cplx<T>::type;
  constexpr int TT = HadCfg<T>::TT, DF = HadCfg<T>::DF, NT = HadCfg<T>::THREADS;
  __shared__ __align__(32) C2 Gs[26 * 64];
  const int f = blockIdx.y;
  const C2* Gf = reinterpret_cast<const C2*>(G) + (size_t)f * 26 * 64;
  constexpr bool kF2 = HAD_F2 && sizeof(T) == 4;
  if constexpr (kF2) {
    // (gr, gi) of itar 2p, 2p+1 -> (gr0, gr1, gi0, gi1)
    T* gs = reinterpret_cast<T*>(Gs);
    for (int e = threadIdx.x; e < 26 * 64; e += NT) {
      const int h = e & 1, b = (e & ~1) * 2;
      const C2 v = Gf[e];
      gs[b + h] = v.x;
      gs[b + 2 + h] = v.y;
    }
  } else {
    for (int e = threadIdx.x; e < 26 * 64; e += NT) Gs[e] = Gf[e];
  }
  // targets of this thread: t0 + u * NT, u < TT (coalesced tsrcT reads)
  const int t0 = blockIdx.x * NT * TT + threadIdx.x;
  const C2* Qf = reinterpret_cast<const C2*>(Q) + (size_t)f * nsrc * 8;
  // two-stage pipeline over directions: the source rows of direction d+1
  // are in flight while direction d is multiplied, and the row indices run
  // one direction further ahead
  int ia[TT], ib[TT];
  C2 qa[TT][8], qb[TT][8];
  if (t0 < ntar) {
    had_index<T, TT>(tsrcT, 0, t0, NT, ntar, ia);
    had_rows<T, TT>(Qf, nsrc, ia, qa);
    had_index<T, TT>(tsrcT, 1, t0, NT, ntar, ib);
  }
  __syncthreads();
  if (t0 >= ntar) return;
  T pr[TT][8], pi[TT][8];
#pragma unroll
  for (int u = 0; u < TT; ++u)
#pragma unroll
    for (int i = 0; i < 8; ++i) pr[u][i] = pi[u][i] = T(0);
  // FP64 accumulators: registers, or one shared-memory column per thread
  constexpr bool kAccS = HadCfg<T>::ACC_SMEM;
  __shared__ double accs[kAccS ? TT * 16 : 1][NT];
  double ar[TT][8], ai[TT][8];
#pragma unroll
  for (int u = 0; u < TT; ++u)
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if constexpr (kAccS) {
        accs[u * 16 + 2 * i][threadIdx.x] = 0.0;
        accs[u * 16 + 2 * i + 1][threadIdx.x] = 0.0;
      } else {
        ar[u][i] = ai[u][i] = 0.0;
      }
    }
  auto flush = [&]() {
#pragma unroll
    for (int u = 0; u < TT; ++u)
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if constexpr (kAccS) {
          accs[u * 16 + 2 * i][threadIdx.x] += (double)pr[u][i];
          accs[u * 16 + 2 * i + 1][threadIdx.x] += (double)pi[u][i];
        } else {
          ar[u][i] += (double)pr[u][i];
          ai[u][i] += (double)pi[u][i];
        }
        pr[u][i] = pi[u][i] = T(0);
      }
  };
  auto MAC = [&](const C2* g, const int (&sd)[TT], const C2 (&q)[TT][8]) {
    if constexpr (kF2) {
      had_mac_f2<TT>(reinterpret_cast<const float4*>(g), sd, q, pr, pi);
    } else {
      had_mac<T, TT>(g, sd, q, pr, pi);
    }
  };
  for (int d = 0; d < 26; d += 2) {
    int ja[TT];
    had_rows<T, TT>(Qf, nsrc, ib, qb);
    if (d + 2 < 26) had_index<T, TT>(tsrcT, d + 2, t0, NT, ntar, ja);
    MAC(Gs + d * 64, ia, qa);
    if (DF == 1 || (d + 1) % DF == 0) flush();
    if (d + 2 < 26) {
#pragma unroll
      for (int u = 0; u < TT; ++u) ia[u] = ja[u];
      had_rows<T, TT>(Qf, nsrc, ia, qa);
    }
    int jb[TT];
    if (d + 3 < 26) had_index<T, TT>(tsrcT, d + 3, t0, NT, ntar, jb);
    MAC(Gs + (d + 1) * 64, ib, qb);
    if ((d + 2) % DF == 0 || d + 2 == 26) flush();
    if (d + 3 < 26) {
#pragma unroll
      for (int u = 0; u < TT; ++u) ib[u] = jb[u];
    }
  }
#pragma unroll
  for (int u = 0; u < TT; ++u) {
    const int t = t0 + u * NT;
    if (t >= ntar) break;
    C2* out = reinterpret_cast<C2*>(Pk) + ((size_t)f * ntar + t) * 8;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      C2 v;
      if constexpr (kAccS) {
        v.x = (T)accs[u * 16 + 2 * i][threadIdx.x];
        v.y = (T)accs[u * 16 + 2 * i + 1][threadIdx.x];
      } else {
        v.x = (T)ar[u][i];
        v.y = (T)ai[u][i];
      }
      out[i] = v;
    }
  }
}

// The 8x8 kernel spectra re-laid frequency-major for the Hadamard:
// G[(f * 26 + d) * 64 + pair] = cc8[(d * 64 + pair) * Nf + f] (complex), in the
// pass's precision (FP32 by round to nearest).
template <typename T>
__global__ void k_g8_layout(const double2* __restrict__ cc8, int Nf, T* __restrict__ G) {
  const size_t total = (size_t)26 * 64 * Nf;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int pr = (int)(e % 64), d = (int)((e / 64) % 26);
    const size_t f = e / (64 * 26);
    const double2 v = cc8[((size_t)d * 64 + pr) * Nf + f];
    G[2 * e] = (T)v.x;
    G[2 * e + 1] = (T)v.y;
  }
}

// Hadamard 1x27 (hadamard_1x27 + c2c_1x27x1_AVX, kernel.cpp:1084-1138) for the
// image levels, FP64; the 27 image spectra of a direction are pre-summed.
__global__ void k_m2l_hadamard27(const double* __restrict__ Q, const double* __restrict__ G27,
                                 const int* __restrict__ tsrc, int ntar, int nsrc, int Nf,
                                 double* __restrict__ Pk) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.y;
  if (f >= Nf || t >= ntar) return;
  double re = 0, im = 0;
  for (int d = 0; d < 26; ++d) {
    const int s = tsrc[t * 26 + d];
    if (s < 0) continue;
    const double gr = G27[((size_t)d * Nf + f) * 2], gi = G27[((size_t)d * Nf + f) * 2 + 1];
    const size_t qo = 2 * q8_index<double>(f, s, 0, nsrc);  // the up pass's layout, slot 0
    cmad(re, im, gr, gi, Q[qo], Q[qo + 1]);
  }
  const size_t po = (((size_t)f * ntar + t) * 8 + 0) * 2;
  Pk[po] = re;
  Pk[po + 1] = im;
}

// down: one block per (target parent, group of sp child slots): read the sp
// spectra of each frequency as one contiguous run of the frequency-major
// Pk[f][tar][slot], then for each child the inverse DFT evaluated only at its
// check-surface points, which sit at [P-1, 2P-2]^3 of the grid
// (surf_conv_idx_map_down, kernel.cpp:1253-1259), and
// p_check[child] += value * scale / N^3 (kernel.cpp:1369-1382).
// items: 10 ints per block = tar, first slot, child cell per slot (-1 = none).
template <typename T, int PP>
__global__ void __launch_bounds__(256)
    k_m2l_down(const T* __restrict__ Pk, const int* __restrict__ items, const double* __restrict__ tscale,
               const int* __restrict__ surf_ijk, const double* __restrict__ twiddle, int P_, int ns, int ntar,
               int sp, double* __restrict__ p_check) {
  const int P = PP > 0 ? PP : P_;
  extern __shared__ unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int N = 2 * P - 1;
  const int P3 = P * P * P, Nf = N * N * P;
  T* W = sm;                        // P*N complex: W[o][k] = conj(w)^(k (P-1+o) mod N)
  T* Y1 = W + 2 * P * N;            // P*N*P complex: [zo][ky][kx]
  T* Y2 = Y1 + 2 * P * N * P;       // P^3 complex: [zo][yo][kx]
  T* X = Y2 + 2 * P3;               // sp * Nf complex: [slot][f]
  const int* it = items + 10 * blockIdx.x;
  const int tar = it[0], slot0 = it[1];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < P * N; e += nt) {
    const int o = e / N, k = e % N;
    const int m = (k * (P - 1 + o)) % N;
    W[2 * e] = (T)twiddle[2 * m];
    W[2 * e + 1] = -(T)twiddle[2 * m + 1];
  }
  if (sp >= 2) {
    using V2 = typename Cplx2<T>::type;
    const int hp = sp / 2;
    for (int e = tid; e < Nf * hp; e += nt) {
      const int f = e / hp, j = 2 * (e % hp);
      const V2 v = *reinterpret_cast<const V2*>(Pk + (((size_t)f * ntar + tar) * 8 + slot0 + j) * 2);
      X[2 * ((size_t)j * Nf + f)] = v.x;
      X[2 * ((size_t)j * Nf + f) + 1] = v.y;
      X[2 * ((size_t)(j + 1) * Nf + f)] = v.z;
      X[2 * ((size_t)(j + 1) * Nf + f) + 1] = v.w;
    }
  } else {
    for (int f = tid; f < Nf; f += nt) {
      const T* in = Pk + (((size_t)f * ntar + tar) * 8 + slot0) * 2;
      X[2 * f] = in[0];
      X[2 * f + 1] = in[1];
    }
  }
  __syncthreads();
  const double sc = tscale[tar];
  for (int j = 0; j < sp; ++j) {
    const int child = it[2 + j];
    if (child < 0) continue;  // block-uniform
    for (int e = tid; e < P * N * P; e += nt) {
      const int zo = e / (N * P), ky = (e / P) % N, kx = e % P;
      const T* wo = W + 2 * zo * N;
      T re = 0, im = 0;
      const T* Xj = X + 2 * (size_t)j * Nf;
      for (int kz = 0; kz < N; ++kz) {
        const int a = (kz * N + ky) * P + kx;
        cmad(re, im, Xj[2 * a], Xj[2 * a + 1], wo[2 * kz], wo[2 * kz + 1]);
      }
      Y1[2 * e] = re;
      Y1[2 * e + 1] = im;
    }
    __syncthreads();
    for (int e = tid; e < P3; e += nt) {
      const int zo = e / (P * P), yo = (e / P) % P, kx = e % P;
      const T* wo = W + 2 * yo * N;
      T re = 0, im = 0;
      for (int ky = 0; ky < N; ++ky) {
        const int a = (zo * N + ky) * P + kx;
        cmad(re, im, Y1[2 * a], Y1[2 * a + 1], wo[2 * ky], wo[2 * ky + 1]);
      }
      Y2[2 * e] = re;
      Y2[2 * e + 1] = im;
    }
    __syncthreads();
    for (int i = tid; i < ns; i += nt) {
      const int xo = surf_ijk[3 * i], yo = surf_ijk[3 * i + 1], zo = surf_ijk[3 * i + 2];
      const T* row = Y2 + 2 * ((zo * P + yo) * P);
      const T* wo = W + 2 * xo * N;
      T acc = 0;
      // Re(Y * conj(w)^m) summed over kx >= 1, doubled for the missing half
      for (int kx = 1; kx < P; ++kx) {
        acc = fma(row[2 * kx], wo[2 * kx], acc);
        acc = fma(-row[2 * kx + 1], wo[2 * kx + 1], acc);
      }
      const T v = row[0] + T(2) * acc;
      p_check[(size_t)child * ns + i] += (double)v * sc;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// post: far + near, dipole correction (kernel.cpp:1580-1596), 1/(4 pi)
// (body.cpp:88-96), and the scatter back to input order (body.cpp:177-190).
// ---------------------------------------------------------------------------
constexpr int kDipBlocks = kDipoleBlocks;

__global__ void k_dipole_partial(const double4* __restrict__ body64, int n, double* __restrict__ partial) {
  // per block: sum of q x, q y, q z and q
  __shared__ double s[4][256];
  double ax = 0, ay = 0, az = 0, aq = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double4 b = body64[i];
    ax += b.x * b.w;
    ay += b.y * b.w;
    az += b.z * b.w;
    aq += b.w;
  }
  s[0][threadIdx.x] = ax;
  s[1][threadIdx.x] = ay;
  s[2][threadIdx.x] = az;
  s[3][threadIdx.x] = aq;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int k = 0; k < 4; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) partial[blockIdx.x * 4 + k] = s[k][0];
}

__global__ void k_dipole_final(double* __restrict__ partial) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double d[4] = {0, 0, 0, 0};
  for (int b = 0; b < kDipBlocks; ++b)
    for (int k = 0; k < 4; ++k) d[k] += partial[b * 4 + k];
  for (int k = 0; k < 4; ++k) partial[4 * kDipBlocks + k] = d[k];
}

// Adjoint support.  k_swap_charges puts the weights w (input order) into the
// tree-order bodies and keeps their charges; k_restore_charges puts them
// back; k_adj_combine forms dL/dx_k = w_k grad(phi_q)_k + q_k grad(psi_w)_k
// in input order (k = perm[i]).
__global__ void k_swap_charges(double4* __restrict__ body64, const double* __restrict__ w,
                               const int64_t* __restrict__ perm, int n, double* __restrict__ qsave) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  qsave[i] = body64[i].w;
  body64[i].w = w[perm[i]];
}

// New charges (input order) for bodies whose positions are already on the
// device in tree order.
__global__ void k_set_charges(double4* __restrict__ body64, const double* __restrict__ q,
                              const int64_t* __restrict__ perm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  body64[i].w = q[perm[i]];
}

__global__ void k_restore_charges(double4* __restrict__ body64, const double* __restrict__ qsave, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  body64[i].w = qsave[i];
}

__global__ void k_adj_combine(const int64_t* __restrict__ perm, const double* __restrict__ w,
                              const double* __restrict__ qsave, const double* __restrict__ grad_q,
                              const double* __restrict__ grad_w, int n, double* __restrict__ dLdx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t k = perm[i];
  const double wk = w[k], qk = qsave[i];
#pragma unroll
  for (int c = 0; c < 3; ++c) dLdx[3 * k + c] = wk * grad_q[3 * k + c] + qk * grad_w[3 * k + c];
}

__global__ void k_post(const double* __restrict__ phi_far, const double* __restrict__ grad_far,
                       const double* __restrict__ phi_near, const double* __restrict__ grad_near,
                       const double4* __restrict__ body64, const int64_t* __restrict__ perm, int n,
                       const double* __restrict__ dip, double coef, int dipole, double cx, double cy, double cz,
                       double out_scale, double* __restrict__ out_phi, double* __restrict__ out_grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p = 0, g0 = 0, g1 = 0, g2 = 0;
  if (phi_far) {
    p += phi_far[i];
    g0 += grad_far[3 * i];
    g1 += grad_far[3 * i + 1];
    g2 += grad_far[3 * i + 2];
  }
  if (phi_near) {
    p += phi_near[i];
    g0 += grad_near[3 * i];
    g1 += grad_near[3 * i + 1];
    g2 += grad_near[3 * i + 2];
  }
  if (dipole) {
    // mu = sum q (x - centre): the reference's dipole, whose box is centred
    // at the origin (argument.cpp:61-62)
    const double Q = dip[3];
    const double dx = dip[0] - Q * cx, dy = dip[1] - Q * cy, dz = dip[2] - Q * cz;
    if (dipole == 1) {
      // the reference's per-body form coef |mu|^2 / (N q_i) (kernel.cpp:1593)
      const double dnorm = dx * dx + dy * dy + dz * dz;
      p -= coef * dnorm / n / body64[i].w;
    } else {
      // the potential of the surface term: coef mu . (x_i - centre)
      const double4 b = body64[i];
      p -= coef * (dx * (b.x - cx) + dy * (b.y - cy) + dz * (b.z - cz));
    }
    g0 -= coef * dx;
    g1 -= coef * dy;
    g2 -= coef * dz;
  }
  const int64_t o = perm[i];
  out_phi[o] = p * out_scale;
  out_grad[3 * o + 0] = g0 * out_scale;
  out_grad[3 * o + 1] = g1 * out_scale;
  out_grad[3 * o + 2] = g2 * out_scale;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline int cdiv(int64_t a, int b) { return (int)((a + b - 1) / b); }

cudaError_t launch_gather_bodies(const double* x_in, const double* q_in, const int64_t* perm, int n,
                                 double4* body64, cudaStream_t st) {
  if (n > 0) k_gather_bodies<<<cdiv(n, 256), 256, 0, st>>>(x_in, q_in, perm, n, body64);
  return cudaGetLastError();
}

cudaError_t launch_prep32(const double4* body64, const int* body_leaf, const LeafInfo* leaves,
                          float4* body32, int n, cudaStream_t st) {
  if (n > 0) k_prep32<<<cdiv(n, 256), 256, 0, st>>>(body64, body_leaf, leaves, body32, n);
  return cudaGetLastError();
}

cudaError_t launch_p2p32(const float4* body32, const P2PItem32* items, int nitems, const int* list_off,
                         const P2PSrc32* list, double* phi, double* grad, cudaStream_t st) {
  if (nitems > 0)
    k_p2p32<<<cdiv(nitems, kP2PWarps), 32 * kP2PWarps, 0, st>>>(body32, items, nitems, list_off, list, phi,
                                                               grad);
  return cudaGetLastError();
}

cudaError_t launch_p2p64(const double4* body64, const P2PItem32* items, int nitems, const int* list_off,
                         const P2PSrc64* list, double* phi, double* grad, cudaStream_t st) {
  if (nitems > 0)
    k_p2p64<<<cdiv(nitems, kP2PWarps), 32 * kP2PWarps, 0, st>>>(body64, items, nitems, list_off, list, phi,
                                                               grad);
  return cudaGetLastError();
}

cudaError_t launch_close_count(const float4* body32, const P2PItem32* items, int nitems, const int* list_off,
                               const P2PSrc32* list, const LeafInfo* leaves, int* cnt, cudaStream_t st) {
  if (nitems > 0)
    k_close_scan<false><<<cdiv(nitems, 8), 256, 0, st>>>(body32, items, nitems, list_off, list, leaves, cnt,
                                                         nullptr, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_close_emit(const float4* body32, const P2PItem32* items, int nitems, const int* list_off,
                              const P2PSrc32* list, const LeafInfo* leaves, const int* off, int2* pairs,
                              cudaStream_t st) {
  if (nitems > 0)
    k_close_scan<true><<<cdiv(nitems, 8), 256, 0, st>>>(body32, items, nitems, list_off, list, leaves, nullptr,
                                                        off, pairs);
  return cudaGetLastError();
}

cudaError_t launch_close_fix(const double4* body64, const float4* body32, const P2PSrc32* list, const int* off,
                             const int2* pairs, int n, double cycle, double* phi, double* grad, cudaStream_t st) {
  if (n > 0) k_close_fix<<<cdiv(n, 256), 256, 0, st>>>(body64, body32, list, off, pairs, n, cycle, phi, grad);
  return cudaGetLastError();
}

cudaError_t launch_count_scan(const int* cnt, int* off, int n, void* tmp, size_t* tmp_bytes, cudaStream_t st) {
  return cub::DeviceScan::ExclusiveSum(tmp, *tmp_bytes, cnt, off, n, st);
}

cudaError_t launch_p2m_check(const double4* body64, const LeafInfo* leaves, int nleaf,
                             const double* surf_unit, int ns, double* out, cudaStream_t st, int newton) {
  if (nleaf > 0) {
    const int per = cdiv(ns, kCheckPer);
    const int nt = per >= kCheckMaxThreads ? kCheckMaxThreads : cdiv(per, 32) * 32;
    if (newton == 1)
      k_p2m_check<1><<<nleaf, nt, 0, st>>>(body64, leaves, surf_unit, ns, out);
    else
      k_p2m_check<2><<<nleaf, nt, 0, st>>>(body64, leaves, surf_unit, ns, out);
  }
  return cudaGetLastError();
}

template <int NR>
static cudaError_t l2p_nr(const double4* body64, const LeafInfo* leaves, int nleaf, const double* surf_unit, int ns,
                          const double* q_down, double* phi, double* grad, cudaStream_t st) {
  const size_t sm = sizeof(double4) * ns;
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_l2p_eval<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
  }
  k_l2p_eval<NR><<<nleaf, kSurfThreads, sm, st>>>(body64, leaves, surf_unit, ns, q_down, phi, grad);
  return cudaGetLastError();
}

cudaError_t launch_l2p_eval(const double4* body64, const LeafInfo* leaves, int nleaf,
                            const double* surf_unit, int ns, const double* q_down, double* phi,
                            double* grad, cudaStream_t st, int newton) {
  if (nleaf <= 0) return cudaGetLastError();
  return newton == 1 ? l2p_nr<1>(body64, leaves, nleaf, surf_unit, ns, q_down, phi, grad, st)
                     : l2p_nr<2>(body64, leaves, nleaf, surf_unit, ns, q_down, phi, grad, st);
}

cudaError_t launch_apply(const ApplyBatch& b, cudaStream_t st) {
  if (b.max_rows > 0 && b.groups > 0) {
#if APPLY_TC
    if (b.ns % 2 != 0) return cudaErrorInvalidValue;  // 16-byte copies need an even ns
    // the shared-memory opt-in is per function and device; set once per
    // device, safely when several host threads make their first call at once
    static std::atomic<bool> attr_set[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !attr_set[dev].load(std::memory_order_acquire)) {
      e = cudaFuncSetAttribute(k_apply_f64_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGSmem);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) attr_set[dev].store(true, std::memory_order_release);
    }
    dim3 grid(cdiv(b.ns, kGN), cdiv(b.max_rows, kGM), b.groups);
    k_apply_f64_tc<<<grid, kGThreads, kGSmem, st>>>(b);
#else
    dim3 grid(cdiv(b.ns, kTN), cdiv(b.max_rows, kTM), b.groups);
    k_apply_f64<<<grid, 256, 0, st>>>(b);
#endif
  }
  return cudaGetLastError();
}

cudaError_t launch_sum_children(const int* list, int nparents, const double* Y, int ns, double* q,
                                cudaStream_t st) {
  if (nparents > 0) k_sum_children<<<nparents, 128, 0, st>>>(list, nparents, Y, ns, q);
  return cudaGetLastError();
}

// orders with a compile-time instance (the register-blocked kernels)
static bool fixed_p(int P) { return (P >= 4 && P <= 8) || P == 10; }
template <typename T>
static size_t up_smem(int P, int sp) {
  const size_t N = 2 * P - 1, P3 = (size_t)P * P * P;
  if (fixed_p(P))
    return sizeof(T) * ((2 * N * N + 7) / 8 * 8 + 2 * (size_t)sp * P3 + std::max((size_t)sp * P3, 2 * (size_t)sp * P * N * P));
  return sizeof(T) * (2 * N * N + 3 * P3 + 2 * (size_t)sp * P * N * P);
}
template <typename T>
static size_t down_smem(int P, int sp) {
  const size_t N = 2 * P - 1, P3 = (size_t)P * P * P;
  if (fixed_p(P)) return sizeof(T) * (2 * (size_t)P * N + 2 * (size_t)sp * P * N * P + 2 * (size_t)sp * N * N * P);
  return sizeof(T) * (2 * (size_t)P * N + 2 * (size_t)P * N * P + 2 * P3 + 2 * (size_t)sp * N * N * P);
}

// Largest slot group (8, 4, 2, 1) whose working set fits in shared memory.
static const size_t kSmemMax = 220 * 1024;
// Capped at one 32-byte sector of spectrum per frequency (4 FP32 or 2 FP64
// complex values), which keeps enough blocks in flight.
template <typename T>
int m2l_up_slots(int P) {
  for (int sp = (int)(32 / (2 * sizeof(T))); sp > 1; sp /= 2)
    if (up_smem<T>(P, sp) <= kSmemMax) return sp;
  return 1;
}
template <typename T>
int m2l_down_slots(int P) {
  for (int sp = (int)(32 / (2 * sizeof(T))); sp > 1; sp /= 2)
    if (down_smem<T>(P, sp) <= kSmemMax) return sp;
  return 1;
}
template int m2l_up_slots<float>(int);
template int m2l_up_slots<double>(int);
template int m2l_down_slots<float>(int);
template int m2l_down_slots<double>(int);

template <typename T, int PP>
static cudaError_t up_p(const double* q_equiv, const int* items, int nitems, const int* surf_ijk,
                        const double* twiddle, int P, int ns, int nsrc, int sp, T* Q, cudaStream_t st) {
  const size_t sm = up_smem<T>(P, sp);
  if constexpr (PP > 0) {
    cudaError_t e = cudaFuncSetAttribute(k_m2l_up_rb<T, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_m2l_up_rb<T, PP><<<nitems, 256, sm, st>>>(q_equiv, items, surf_ijk, twiddle, ns, nsrc, sp, Q);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_m2l_up<T, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_m2l_up<T, PP><<<nitems, 256, sm, st>>>(q_equiv, items, surf_ijk, twiddle, P, ns, nsrc, sp, Q);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_m2l_up(const double* q_equiv, const int* items, int nitems, const int* surf_ijk,
                          const double* twiddle, int P, int ns, int nsrc, int sp, T* Q, cudaStream_t st) {
  if (nitems <= 0) return cudaGetLastError();
  switch (P) {
    case 4: return up_p<T, 4>(q_equiv, items, nitems, surf_ijk, twiddle, P, ns, nsrc, sp, Q, st);
    case 5: return up_p<T, 5>(q_equiv, items, nitems, surf_ijk, twiddle, P, ns, nsrc, sp, Q, st);
    case 6: return up_p<T, 6>(q_equiv, items, nitems, surf_ijk, twiddle, P, ns, nsrc, sp, Q, st);
    case 7: return up_p<T, 7>(q_equiv, items, nitems, surf_ijk, twiddle, P, ns, nsrc, sp, Q, st);
    case 8: return up_p<T, 8>(q_equiv, items, nitems, surf_ijk, twiddle, P, ns, nsrc, sp, Q, st);
    case 10: return up_p<T, 10>(q_equiv, items, nitems, surf_ijk, twiddle, P, ns, nsrc, sp, Q, st);
    default: return up_p<T, 0>(q_equiv, items, nitems, surf_ijk, twiddle, P, ns, nsrc, sp, Q, st);
  }
}

template <typename T>
cudaError_t launch_m2l_hadamard8(const T* Q, const T* G, const int* tsrcT, int ntar, int nsrc, int Nf, T* Pk,
                                 cudaStream_t st) {
  if (ntar > 0) {
    constexpr int NT = HadCfg<T>::THREADS, TT = HadCfg<T>::TT;
    dim3 grid(cdiv(ntar, NT * TT), Nf);
    k_m2l_hadamard8<T><<<grid, NT, 0, st>>>(Q, G, tsrcT, ntar, nsrc, Nf, Pk);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_g8_layout(const double* cc8, int Nf, T* G, cudaStream_t st) {
  const size_t total = (size_t)26 * 64 * Nf;
  if (total > 0)
    k_g8_layout<T><<<(int)std::min<size_t>((total + 255) / 256, 148 * 16), 256, 0, st>>>(
        reinterpret_cast<const double2*>(cc8), Nf, G);
  return cudaGetLastError();
}
template cudaError_t launch_g8_layout<float>(const double*, int, float*, cudaStream_t);
template cudaError_t launch_g8_layout<double>(const double*, int, double*, cudaStream_t);

cudaError_t launch_body_leaf(const LeafInfo* leaves, int nleaf, int n, int* body_leaf, cudaStream_t st) {
  if (nleaf > 0) k_body_leaf<<<nleaf, 128, 0, st>>>(leaves, nleaf, n, body_leaf);
  return cudaGetLastError();
}

cudaError_t launch_m2l_hadamard27(const double* Q, const double* G27, const int* tsrc, int ntar, int nsrc,
                                  int Nf, double* Pk, cudaStream_t st) {
  if (ntar > 0) {
    dim3 grid(cdiv(Nf, 128), ntar);
    k_m2l_hadamard27<<<grid, 128, 0, st>>>(Q, G27, tsrc, ntar, nsrc, Nf, Pk);
  }
  return cudaGetLastError();
}

template <typename T, int PP>
static cudaError_t down_p(const T* Pk, const int* items, const double* tscale, int nitems, const int* surf_ijk,
                          const double* twiddle, int P, int ns, int ntar, int sp, double* p_check,
                          cudaStream_t st) {
  const size_t sm = down_smem<T>(P, sp);
  if constexpr (PP > 0) {
    cudaError_t e =
        cudaFuncSetAttribute(k_m2l_down_rb<T, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_m2l_down_rb<T, PP><<<nitems, 256, sm, st>>>(Pk, items, tscale, surf_ijk, twiddle, ns, ntar, sp, p_check);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_m2l_down<T, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_m2l_down<T, PP><<<nitems, 256, sm, st>>>(Pk, items, tscale, surf_ijk, twiddle, P, ns, ntar, sp, p_check);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_m2l_down(const T* Pk, const int* items, const double* tscale, int nitems,
                            const int* surf_ijk, const double* twiddle, int P, int ns, int ntar, int sp,
                            double* p_check, cudaStream_t st) {
  if (nitems <= 0) return cudaGetLastError();
  switch (P) {
    case 4: return down_p<T, 4>(Pk, items, tscale, nitems, surf_ijk, twiddle, P, ns, ntar, sp, p_check, st);
    case 5: return down_p<T, 5>(Pk, items, tscale, nitems, surf_ijk, twiddle, P, ns, ntar, sp, p_check, st);
    case 6: return down_p<T, 6>(Pk, items, tscale, nitems, surf_ijk, twiddle, P, ns, ntar, sp, p_check, st);
    case 7: return down_p<T, 7>(Pk, items, tscale, nitems, surf_ijk, twiddle, P, ns, ntar, sp, p_check, st);
    case 8: return down_p<T, 8>(Pk, items, tscale, nitems, surf_ijk, twiddle, P, ns, ntar, sp, p_check, st);
    case 10: return down_p<T, 10>(Pk, items, tscale, nitems, surf_ijk, twiddle, P, ns, ntar, sp, p_check, st);
    default: return down_p<T, 0>(Pk, items, tscale, nitems, surf_ijk, twiddle, P, ns, ntar, sp, p_check, st);
  }
}

cudaError_t launch_dipole(const double4* body64, int n, double* partial, cudaStream_t st) {
  k_dipole_partial<<<kDipBlocks, 256, 0, st>>>(body64, n, partial);
  k_dipole_final<<<1, 32, 0, st>>>(partial);
  return cudaGetLastError();
}

cudaError_t launch_swap_charges(double4* body64, const double* w, const int64_t* perm, int n, double* qsave,
                                cudaStream_t st) {
  if (n > 0) k_swap_charges<<<cdiv(n, 256), 256, 0, st>>>(body64, w, perm, n, qsave);
  return cudaGetLastError();
}

cudaError_t launch_set_charges(double4* body64, const double* q, const int64_t* perm, int n, cudaStream_t st) {
  if (n > 0) k_set_charges<<<cdiv(n, 256), 256, 0, st>>>(body64, q, perm, n);
  return cudaGetLastError();
}

cudaError_t launch_restore_charges(double4* body64, const double* qsave, int n, cudaStream_t st) {
  if (n > 0) k_restore_charges<<<cdiv(n, 256), 256, 0, st>>>(body64, qsave, n);
  return cudaGetLastError();
}

cudaError_t launch_adj_combine(const int64_t* perm, const double* w, const double* qsave, const double* grad_q,
                               const double* grad_w, int n, double* dLdx, cudaStream_t st) {
  if (n > 0) k_adj_combine<<<cdiv(n, 256), 256, 0, st>>>(perm, w, qsave, grad_q, grad_w, n, dLdx);
  return cudaGetLastError();
}

// Leaf rows of the cell vectors <-> a leaf-ordered buffer (the exchange of
// a sharded pass): gather writes buf[l] = own[l] ? v[cell[l]] : 0 (own null:
// every row), scatter writes v[cell[l]] = buf[l].
__global__ void k_leaf_rows(double* __restrict__ v, int nrow, const int* __restrict__ cells,
                            const char* __restrict__ own, int nleaf, int ns, double* __restrict__ buf, int scatter) {
  const int l = blockIdx.x;
  if (l >= nleaf) return;
  const int c = cells[l];
  if (c < 0 || c >= nrow) return;  // not a row of v
  double* row = v + (size_t)c * ns;
  double* b = buf + (size_t)l * ns;
  if (scatter) {
    for (int i = threadIdx.x; i < ns; i += blockDim.x) row[i] = b[i];
  } else {
    const bool keep = own == nullptr || own[l];
    for (int i = threadIdx.x; i < ns; i += blockDim.x) b[i] = keep ? row[i] : 0.0;
  }
}

cudaError_t launch_leaf_rows(double* v, int nrow, const int* cells, const char* own, int nleaf, int ns,
                             double* buf, bool scatter, cudaStream_t st) {
  if (nleaf > 0 && (!v || !cells || !buf)) return cudaErrorInvalidValue;
  if (nleaf > 0) k_leaf_rows<<<nleaf, 128, 0, st>>>(v, nrow, cells, own, nleaf, ns, buf, scatter ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_post(const double* phi_far, const double* grad_far, const double* phi_near,
                        const double* grad_near, const double4* body64, const int64_t* perm, int n,
                        const double* dipole_partial, double coef, int dipole, const double* centre,
                        double out_scale, double* out_phi, double* out_grad, cudaStream_t st) {
  if (n > 0)
    k_post<<<cdiv(n, 256), 256, 0, st>>>(phi_far, grad_far, phi_near, grad_near, body64, perm, n,
                                          dipole_partial + 4 * kDipBlocks, coef, dipole, centre[0], centre[1],
                                          centre[2], out_scale, out_phi, out_grad);
  return cudaGetLastError();
}

template cudaError_t launch_m2l_up<float>(const double*, const int*, int, const int*, const double*, int, int,
                                          int, int, float*, cudaStream_t);
template cudaError_t launch_m2l_up<double>(const double*, const int*, int, const int*, const double*, int, int,
                                           int, int, double*, cudaStream_t);
template cudaError_t launch_m2l_hadamard8<float>(const float*, const float*, const int*, int, int, int, float*,
                                                 cudaStream_t);
template cudaError_t launch_m2l_hadamard8<double>(const double*, const double*, const int*, int, int, int,
                                                  double*, cudaStream_t);
template cudaError_t launch_m2l_down<float>(const float*, const int*, const double*, int, const int*,
                                            const double*, int, int, int, int, double*, cudaStream_t);
template cudaError_t launch_m2l_down<double>(const double*, const int*, const double*, int, const int*,
                                             const double*, int, int, int, int, double*, cudaStream_t);

}  // namespace rtfmm_b200
