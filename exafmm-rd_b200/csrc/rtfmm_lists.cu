// The P2P lists of the dual-tree walk, built on the GPU.
//
// Traverser::horizontal_origin (3dpp/src/traverser.cpp:70-176) is a
// recursion over frames (target, source, their parents) under each periodic
// offset; every frame either emits one P2P pair, divides into child frames,
// or ends.  The lists are the emitted pairs in the order the recursion
// (depth first, children in order, walks in offset order) emits them.
//
// Here the frames are expanded breadth first, one round per level of the
// frame tree, by walk_step (rtfmm_walk.h, the same function the host walk
// runs).  Each frame carries its path from the root (the walk index, then
// the child index taken at every division), so the depth-first emission
// order of the pairs is the lexicographic order of their paths: no two
// emitting frames are one another's ancestors, so two paths always differ
// at a digit both have.  The pairs are sorted by path, then stably by target
// cell, and each target's run becomes its list.
//
// Paths hold 19 digits in a first 64-bit word (after 5 bits of walk index)
// and 21 in a second: walks up to 40 divisions deep.  Deeper walks, and
// trees of 2^25 cells or more, are left to the host walk.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "rtfmm_tree.h"
#include "rtfmm_walk.h"

namespace rtfmm_b200 {
namespace {

constexpr int kHiDigits = 19;
constexpr int kLoDigits = 21;
constexpr int kMaxDivisions = kHiDigits + kLoDigits;
constexpr int kWalkShift = 57;
constexpr int kCellBits = 25;

struct DevCells {
  const double* __restrict__ cx;
  const double* __restrict__ cr;
  const int* __restrict__ cdepth;
  const int* __restrict__ ccnum;
  const int* __restrict__ ccoff;
  __device__ double x(int i, int k) const { return cx[3 * i + k]; }
  __device__ double r(int i) const { return cr[i]; }
  __device__ int depth(int i) const { return cdepth[i]; }
  __device__ int cnum(int i) const { return ccnum[i]; }
  __device__ int coff(int i) const { return ccoff[i]; }
};

__device__ __forceinline__ void put_digit(unsigned long long& hi, unsigned long long& lo, int pos, int digit) {
  if (pos < kHiDigits)
    hi |= (unsigned long long)digit << (3 * (kHiDigits - 1 - pos));
  else
    lo |= (unsigned long long)digit << (3 * (kLoDigits - 1 - (pos - kHiDigits)));
}

// Outcome counts of one round's frames.
__global__ void k_walk_count(DevCells C, const int4* __restrict__ fr, const unsigned long long* __restrict__ khi,
                             int nf, const double* __restrict__ offs, int* __restrict__ nkid,
                             int* __restrict__ nhit) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const int4 v = fr[i];
  const WalkFrame f{v.x, v.y, v.z, v.w};
  const int walk = (int)(khi[i] >> kWalkShift);
  int hit = -1;
  WalkFrame kids[8];
  const int r = walk_step(C, f, offs + 3 * walk, &hit, kids);
  nkid[i] = r < 0 ? -r : 0;
  nhit[i] = r == 1;
}

// The round's child frames and emitted pairs at their scanned offsets.
__global__ void k_walk_emit(DevCells C, const int4* __restrict__ fr, const unsigned long long* __restrict__ khi,
                            const unsigned long long* __restrict__ klo, int nf, const double* __restrict__ offs,
                            const int* __restrict__ kid_off, const int* __restrict__ hit_off, int round,
                            int4* __restrict__ nfr, unsigned long long* __restrict__ nkhi,
                            unsigned long long* __restrict__ nklo, unsigned long long* __restrict__ hhi,
                            unsigned long long* __restrict__ hlo, unsigned long long* __restrict__ hval, int hbase,
                            int* __restrict__ overflow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const int4 v = fr[i];
  const WalkFrame f{v.x, v.y, v.z, v.w};
  const unsigned long long hi = khi[i], lo = klo[i];
  const int walk = (int)(hi >> kWalkShift);
  int hit = -1;
  WalkFrame kids[8];
  const int r = walk_step(C, f, offs + 3 * walk, &hit, kids);
  if (r == 1) {
    const int j = hbase + hit_off[i];
    hhi[j] = hi;
    hlo[j] = lo;
    hval[j] = ((unsigned long long)f.tc << (kCellBits + 5)) | ((unsigned long long)hit << 5) | (unsigned)walk;
  } else if (r < 0) {
    if (round >= kMaxDivisions) {
      atomicExch(overflow, 1);
      return;
    }
    const int base = kid_off[i];
    for (int c = 0; c < -r; ++c) {
      unsigned long long h2 = hi, l2 = lo;
      put_digit(h2, l2, round, c);
      nfr[base + c] = make_int4(kids[c].tc, kids[c].sc, kids[c].tcp, kids[c].scp);
      nkhi[base + c] = h2;
      nklo[base + c] = l2;
    }
  }
}

__global__ void k_iota(int n, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = i;
}

template <typename T>
__global__ void k_gather(const T* __restrict__ in, const int* __restrict__ idx, int n, T* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[idx[i]];
}

int cdiv(int64_t a, int b) { return (int)((a + b - 1) / b); }

struct Scratch {
  const TreeScratchFn& fn;
  int base;
  template <typename T>
  cudaError_t get(int slot, T** out, size_t count) {
    *out = (T*)fn(base + slot, std::max<size_t>(1, count) * sizeof(T));
    return *out ? cudaSuccess : cudaErrorMemoryAllocation;
  }
};

}  // namespace

#define LCK(call)                                               \
  do {                                                          \
    cudaError_t e_ = (call);                                    \
    if (e_ != cudaSuccess) {                                    \
      msg = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return kTreeError;                                        \
    }                                                           \
  } while (0)

int device_p2p_walk(Plan& plan, const std::vector<WalkRoot>& roots, cudaStream_t st, const TreeScratchFn& scratch,
                    int slot_base, std::string& msg) {
  const int nc = (int)plan.cells.size();
  if (nc >= (1 << kCellBits) || roots.size() > 31) return kTreeTooDeep;
  Scratch S{scratch, slot_base};
  enum {
    S_CX, S_CR, S_CD, S_CN, S_CO, S_OFF,
    S_FR0, S_HI0, S_LO0, S_FR1, S_HI1, S_LO1,
    S_NKID, S_NHIT, S_KOFF, S_HOFF, S_FLAG, S_TMP,
    S_HHI0, S_HLO0, S_HVAL0, S_HHI1, S_HLO1, S_HVAL1,
    S_IDX0, S_IDX1, S_G0, S_G1
  };
  // cells, structure of arrays
  std::vector<double> hx(3 * (size_t)nc), hr(nc);
  std::vector<int> hd(nc), hn(nc), ho(nc);
  for (int c = 0; c < nc; ++c) {
    const Cell& cl = plan.cells[c];
    for (int k = 0; k < 3; ++k) hx[3 * (size_t)c + k] = cl.x[k];
    hr[c] = cl.r;
    hd[c] = cl.depth;
    hn[c] = cl.cnum;
    ho[c] = cl.coff;
  }
  const int nw = (int)roots.size();
  std::vector<double> hoff(3 * nw);
  for (int w = 0; w < nw; ++w)
    for (int k = 0; k < 3; ++k) hoff[3 * w + k] = roots[w].off[k];
  DevCells C;
  double *dcx, *dcr, *doff;
  int *dcd, *dcn, *dco;
  LCK(S.get(S_CX, &dcx, hx.size()));
  LCK(S.get(S_CR, &dcr, nc));
  LCK(S.get(S_CD, &dcd, nc));
  LCK(S.get(S_CN, &dcn, nc));
  LCK(S.get(S_CO, &dco, nc));
  LCK(S.get(S_OFF, &doff, hoff.size()));
  LCK(cudaMemcpyAsync(dcx, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice, st));
  LCK(cudaMemcpyAsync(dcr, hr.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, st));
  LCK(cudaMemcpyAsync(dcd, hd.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
  LCK(cudaMemcpyAsync(dcn, hn.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
  LCK(cudaMemcpyAsync(dco, ho.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
  LCK(cudaMemcpyAsync(doff, hoff.data(), sizeof(double) * hoff.size(), cudaMemcpyHostToDevice, st));
  C.cx = dcx;
  C.cr = dcr;
  C.cdepth = dcd;
  C.ccnum = dcn;
  C.ccoff = dco;

  // round 0: the root frames, path = walk index
  std::vector<int4> hfr(nw);
  std::vector<unsigned long long> hhi(nw), hlo(nw, 0);
  for (int w = 0; w < nw; ++w) {
    hfr[w] = make_int4(roots[w].tc, roots[w].sc, roots[w].tcp, roots[w].scp);
    hhi[w] = (unsigned long long)w << kWalkShift;
  }
  int4* fr[2];
  unsigned long long *khi[2], *klo[2];
  LCK(S.get(S_FR0, &fr[0], nw));
  LCK(S.get(S_HI0, &khi[0], nw));
  LCK(S.get(S_LO0, &klo[0], nw));
  LCK(cudaMemcpyAsync(fr[0], hfr.data(), sizeof(int4) * nw, cudaMemcpyHostToDevice, st));
  LCK(cudaMemcpyAsync(khi[0], hhi.data(), sizeof(unsigned long long) * nw, cudaMemcpyHostToDevice, st));
  LCK(cudaMemcpyAsync(klo[0], hlo.data(), sizeof(unsigned long long) * nw, cudaMemcpyHostToDevice, st));
  int* flag;
  LCK(S.get(S_FLAG, &flag, 1));
  LCK(cudaMemsetAsync(flag, 0, sizeof(int), st));

  // emitted pairs, grown with a copy when a round needs more room
  int hcap = 0, hcount = 0, hset = 0;
  unsigned long long *hh[2] = {nullptr, nullptr}, *hl[2] = {nullptr, nullptr}, *hv[2] = {nullptr, nullptr};
  auto grow_hits = [&](int need) -> int {
    if (need <= hcap) return kTreeOk;
    const int cap = std::max(need, hcap * 2);
    const int o = hset ^ 1;
    LCK(S.get(S_HHI0 + 3 * o, &hh[o], cap));
    LCK(S.get(S_HLO0 + 3 * o, &hl[o], cap));
    LCK(S.get(S_HVAL0 + 3 * o, &hv[o], cap));
    if (hcount > 0) {
      LCK(cudaMemcpyAsync(hh[o], hh[hset], sizeof(unsigned long long) * hcount, cudaMemcpyDeviceToDevice, st));
      LCK(cudaMemcpyAsync(hl[o], hl[hset], sizeof(unsigned long long) * hcount, cudaMemcpyDeviceToDevice, st));
      LCK(cudaMemcpyAsync(hv[o], hv[hset], sizeof(unsigned long long) * hcount, cudaMemcpyDeviceToDevice, st));
    }
    hset = o;
    hcap = cap;
    return kTreeOk;
  };
  int rc = grow_hits(1 << 16);
  if (rc) return rc;

  void* tmp = nullptr;
  size_t tmp_cap = 0;
  auto need_tmp = [&](size_t bytes) -> int {
    if (bytes <= tmp_cap) return kTreeOk;
    char* t = nullptr;
    LCK(S.get(S_TMP, &t, bytes));
    tmp = t;
    tmp_cap = bytes;
    return kTreeOk;
  };

  int cur = 0, nf = nw, round = 0, lo_used = 0;
  while (nf > 0) {
    int *nkid, *nhit, *koff, *hoff_d;
    LCK(S.get(S_NKID, &nkid, nf));
    LCK(S.get(S_NHIT, &nhit, nf));
    LCK(S.get(S_KOFF, &koff, nf));
    LCK(S.get(S_HOFF, &hoff_d, nf));
    k_walk_count<<<cdiv(nf, 128), 128, 0, st>>>(C, fr[cur], khi[cur], nf, doff, nkid, nhit);
    LCK(cudaGetLastError());
    size_t tb = 0;
    LCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, nkid, koff, nf, st));
    if ((rc = need_tmp(tb))) return rc;
    LCK(cub::DeviceScan::ExclusiveSum(tmp, tb, nkid, koff, nf, st));
    LCK(cub::DeviceScan::ExclusiveSum(tmp, tb, nhit, hoff_d, nf, st));
    int last[4];
    LCK(cudaMemcpyAsync(&last[0], koff + nf - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    LCK(cudaMemcpyAsync(&last[1], nkid + nf - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    LCK(cudaMemcpyAsync(&last[2], hoff_d + nf - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    LCK(cudaMemcpyAsync(&last[3], nhit + nf - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    LCK(cudaStreamSynchronize(st));
    const int64_t nkids = (int64_t)last[0] + last[1], nhits = (int64_t)last[2] + last[3];
    if (nkids > (1 << 30) || hcount + nhits > (1 << 30)) return kTreeTooDeep;
    if (nkids > 0 && round >= kMaxDivisions) return kTreeTooDeep;  // paths would not fit
    if ((rc = grow_hits(hcount + (int)nhits))) return rc;
    const int nx = cur ^ 1;
    LCK(S.get(S_FR0 + 3 * nx, &fr[nx], nkids));
    LCK(S.get(S_HI0 + 3 * nx, &khi[nx], nkids));
    LCK(S.get(S_LO0 + 3 * nx, &klo[nx], nkids));
    k_walk_emit<<<cdiv(nf, 128), 128, 0, st>>>(C, fr[cur], khi[cur], klo[cur], nf, doff, koff, hoff_d, round,
                                              fr[nx], khi[nx], klo[nx], hh[hset], hl[hset], hv[hset], hcount,
                                              flag);
    LCK(cudaGetLastError());
    if (nkids > 0 && round >= kHiDigits) lo_used = 1;
    hcount += (int)nhits;
    nf = (int)nkids;
    cur = nx;
    ++round;
  }
  int hflag = 0;
  LCK(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  LCK(cudaStreamSynchronize(st));
  if (hflag) return kTreeTooDeep;

  // depth-first order, then stably by target cell
  const int H = hcount;
  std::vector<unsigned long long> out(H);
  if (H > 0) {
    int *idx0, *idx1;
    unsigned long long *g0, *g1;
    LCK(S.get(S_IDX0, &idx0, H));
    LCK(S.get(S_IDX1, &idx1, H));
    LCK(S.get(S_G0, &g0, H));
    LCK(S.get(S_G1, &g1, H));
    size_t tb = 0, t2 = 0;
    LCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, hl[hset], g0, idx0, idx1, H, 0, 64, st));
    LCK(cub::DeviceRadixSort::SortKeys(nullptr, t2, g0, g1, H, 0, 64, st));
    if ((rc = need_tmp(std::max(tb, t2)))) return rc;
    k_iota<<<cdiv(H, 256), 256, 0, st>>>(H, idx0);
    LCK(cudaGetLastError());
    if (lo_used) {
      LCK(cub::DeviceRadixSort::SortPairs(tmp, tb, hl[hset], g0, idx0, idx1, H, 0, 64, st));
      k_gather<<<cdiv(H, 256), 256, 0, st>>>(hh[hset], idx1, H, g1);
      LCK(cudaGetLastError());
      LCK(cub::DeviceRadixSort::SortPairs(tmp, tb, g1, g0, idx1, idx0, H, 0, 64, st));
    } else {
      LCK(cub::DeviceRadixSort::SortPairs(tmp, tb, hh[hset], g0, idx0, idx1, H, 0, 64, st));
      std::swap(idx0, idx1);
    }
    // idx0: pair indices in depth-first order
    k_gather<<<cdiv(H, 256), 256, 0, st>>>(hv[hset], idx0, H, g0);
    LCK(cudaGetLastError());
    LCK(cub::DeviceRadixSort::SortKeys(tmp, tb, g0, g1, H, kCellBits + 5, 2 * kCellBits + 5, st));
    LCK(cudaMemcpyAsync(out.data(), g1, sizeof(unsigned long long) * H, cudaMemcpyDeviceToHost, st));
    LCK(cudaStreamSynchronize(st));
  }

  // each target's run becomes its list
  std::vector<int> run_start;
  for (int i = 0; i < H; ++i)
    if (i == 0 || (out[i] >> (kCellBits + 5)) != (out[i - 1] >> (kCellBits + 5))) run_start.push_back(i);
  run_start.push_back(H);
  plan.p2p.v.assign(nc, {});
  const unsigned long long cmask = (1ull << kCellBits) - 1;
#pragma omp parallel for schedule(dynamic, 64)
  for (int r = 0; r < (int)run_start.size() - 1; ++r) {
    const int a = run_start[r], b = run_start[r + 1];
    const int tc = (int)(out[a] >> (kCellBits + 5));
    std::vector<P2PEntry>& L = plan.p2p.v[tc];
    L.resize(b - a);
    for (int i = a; i < b; ++i) {
      const int sc = (int)((out[i] >> 5) & cmask);
      const int w = (int)(out[i] & 31);
      L[i - a] = P2PEntry{sc, roots[w].off};
    }
  }
  return kTreeOk;
}

#undef LCK

}  // namespace rtfmm_b200
