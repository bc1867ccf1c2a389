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

namespace {
// plan.p2p from the sorted pairs: each target's run becomes its list
void pairs_to_lists(const std::vector<unsigned long long>& out, const std::vector<V3>& offs, int nc, Plan& plan) {
  const int H = (int)out.size();
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
      L[i - a] = P2PEntry{sc, offs[w]};
    }
  }
}
}  // namespace

int device_walk_host_lists(const DeviceWalk& dw, Plan& plan, cudaStream_t st, std::string& msg) {
  std::vector<unsigned long long> out(dw.npairs);
  if (dw.npairs > 0) {
    LCK(cudaMemcpyAsync(out.data(), dw.pairs, sizeof(unsigned long long) * dw.npairs, cudaMemcpyDeviceToHost, st));
    LCK(cudaStreamSynchronize(st));
  }
  pairs_to_lists(out, dw.host_offs, dw.ncell, plan);
  return kTreeOk;
}

int device_p2p_walk(Plan& plan, const std::vector<WalkRoot>& roots, cudaStream_t st, const TreeScratchFn& scratch,
                    int slot_base, DeviceWalk* dw, std::string& msg, bool host_lists) {
  const int nc = (int)plan.cells.size();
  if (nc >= (1 << kCellBits) || roots.size() > 31) return kTreeTooDeep;
  Scratch S{scratch, slot_base};
  enum {
    S_CX, S_CR, S_CD, S_CN, S_CO, S_OFF,
    S_FR0, S_HI0, S_LO0, S_FR1, S_HI1, S_LO1,
    S_NKID, S_NHIT, S_KOFF, S_HOFF, S_FLAG, S_TMP,
    S_HHI0, S_HLO0, S_HVAL0, S_HHI1, S_HLO1, S_HVAL1,
    S_IDX0, S_IDX1, S_G0, S_G1, S_CB, S_CM
  };
  // cells, structure of arrays
  std::vector<double> hx(3 * (size_t)nc), hr(nc);
  std::vector<int> hd(nc), hn(nc), ho(nc), hb(nc), hm(nc);
  for (int c = 0; c < nc; ++c) {
    const Cell& cl = plan.cells[c];
    for (int k = 0; k < 3; ++k) hx[3 * (size_t)c + k] = cl.x[k];
    hr[c] = cl.r;
    hd[c] = cl.depth;
    hn[c] = cl.cnum;
    ho[c] = cl.coff;
    hb[c] = cl.boff;
    hm[c] = cl.bnum;
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
  int *dcb, *dcm;
  LCK(S.get(S_CB, &dcb, nc));
  LCK(S.get(S_CM, &dcm, nc));
  LCK(cudaMemcpyAsync(dcb, hb.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
  LCK(cudaMemcpyAsync(dcm, hm.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
  C.cx = dcx;
  C.cr = dcr;
  C.cdepth = dcd;
  C.ccnum = dcn;
  C.ccoff = dco;

  // the first frontier: the root frames, path = walk index
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
    if (host_lists || !dw) {
      LCK(cudaMemcpyAsync(out.data(), g1, sizeof(unsigned long long) * H, cudaMemcpyDeviceToHost, st));
      LCK(cudaStreamSynchronize(st));
    }
    if (dw) {
      dw->pairs = g1;
      dw->npairs = H;
    }
  }
  std::vector<V3> offs(nw);
  for (int w = 0; w < nw; ++w) offs[w] = roots[w].off;
  if (dw) {
    dw->offs = doff;
    dw->nwalk = nw;
    dw->ncell = nc;
    dw->cboff = dcb;
    dw->cbnum = dcm;
    dw->host_offs = offs;
    if (H == 0) dw->npairs = 0;
  }
  if (host_lists || !dw)
    pairs_to_lists(out, offs, nc, plan);
  else
    plan.p2p.v.assign(nc, {});
  return kTreeOk;
}


namespace {

struct LeafTables {
  const LeafInfo* __restrict__ leaves;
  int nlf;
  const int* __restrict__ parent;
  const int* __restrict__ cboff;
  const int* __restrict__ cbnum;
  const int* __restrict__ body_leaf;
  const int* __restrict__ dfs;
  const int* __restrict__ dfs_pos;
  const int* __restrict__ cstart;
  const int* __restrict__ cend;
  const unsigned long long* __restrict__ pairs;
  const double* __restrict__ offs;
};

constexpr int kMaxPathLen = 48;

__global__ void k_pair_bounds(const unsigned long long* __restrict__ pairs, int H, int* __restrict__ cstart,
                              int* __restrict__ cend) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= H) return;
  const unsigned long long t = pairs[i] >> (kCellBits + 5);
  if (i == 0 || (pairs[i - 1] >> (kCellBits + 5)) != t) cstart[t] = i;
  if (i == H - 1 || (pairs[i + 1] >> (kCellBits + 5)) != t) cend[t] = i + 1;
}

// Cells from the root down to c that have pairs (ascending index).
__device__ int leaf_path(const LeafTables& T, int c, int* path) {
  int k = 0;
  for (int a = c; a >= 0 && k < kMaxPathLen; a = T.parent[a])
    if (T.cend[a] > T.cstart[a]) path[k++] = a;
  for (int i = 0; i < k / 2; ++i) {
    const int t = path[i];
    path[i] = path[k - 1 - i];
    path[k - 1 - i] = t;
  }
  return k;
}

// The leaves under cell c: a run of the leaves in first-body order.
__device__ __forceinline__ void leaf_run(const LeafTables& T, int c, int* lo, int* hi) {
  const int b0 = T.cboff[c], nb = T.cbnum[c];
  *lo = T.dfs_pos[T.body_leaf[b0]];
  *hi = T.dfs_pos[T.body_leaf[b0 + nb - 1]] + 1;
}

__global__ void k_leaf_list_count(LeafTables T, int* __restrict__ cnt, int* __restrict__ icnt) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= T.nlf) return;
  int path[kMaxPathLen];
  const int np = leaf_path(T, T.leaves[l].cell, path);
  int c = 0;
  for (int i = 0; i < np; ++i)
    for (int e = T.cstart[path[i]]; e < T.cend[path[i]]; ++e) {
      const int sc = (int)((T.pairs[e] >> 5) & ((1ull << kCellBits) - 1));
      int lo, hi;
      leaf_run(T, sc, &lo, &hi);
      c += hi - lo;
    }
  cnt[l] = c;
  icnt[l] = (T.leaves[l].bnum + 31) / 32;
}

__global__ void k_leaf_list_fill(LeafTables T, const int* __restrict__ off, const int* __restrict__ ioff, int mixed,
                                 P2PSrc32* __restrict__ l32, P2PSrc64* __restrict__ l64,
                                 P2PItem32* __restrict__ items, unsigned long long* __restrict__ pair_total) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= T.nlf) return;
  const LeafInfo Tl = T.leaves[l];
  int path[kMaxPathLen];
  const int np = leaf_path(T, Tl.cell, path);
  int k = off[l];
  unsigned long long pairs = 0;
  for (int i = 0; i < np; ++i)
    for (int e = T.cstart[path[i]]; e < T.cend[path[i]]; ++e) {
      const unsigned long long v = T.pairs[e];
      const int sc = (int)((v >> 5) & ((1ull << kCellBits) - 1));
      const double* o = T.offs + 3 * (int)(v & 31);
      int lo, hi;
      leaf_run(T, sc, &lo, &hi);
      for (int r = lo; r < hi; ++r) {
        const int sl = T.dfs[r];
        const LeafInfo Sl = T.leaves[sl];
        const int self = (Sl.cell == Tl.cell && o[0] == 0 && o[1] == 0 && o[2] == 0) ? 1 : 0;
        if (mixed) {
          P2PSrc32 a;
          // the host build's expression: (c_src + offset) - c_tar in FP64, then FP32
          a.dx = (float)(Sl.cx + o[0] - Tl.cx);
          a.dy = (float)(Sl.cy + o[1] - Tl.cy);
          a.dz = (float)(Sl.cz + o[2] - Tl.cz);
          a.leaf = sl;
          a.self = self;
          a.boff = Sl.boff;
          a.bnum = Sl.bnum;
          a.pad = 0;
          l32[k] = a;
        } else {
          P2PSrc64 b;
          b.ox = o[0];
          b.oy = o[1];
          b.oz = o[2];
          b.leaf = sl;
          b.self = self;
          b.boff = Sl.boff;
          b.bnum = Sl.bnum;
          l64[k] = b;
        }
        pairs += (unsigned long long)Tl.bnum * (unsigned long long)Sl.bnum;
        ++k;
      }
    }
  atomicAdd(pair_total, pairs);
  // work items: 32 targets each; the last <= 16 targets of a leaf take a
  // narrower lane group (16, 8 or 4 lanes)
  int j = ioff[l];
  for (int t0 = 0; t0 < Tl.bnum; t0 += 32, ++j) {
    const int rem = min(32, Tl.bnum - t0);
    int lw = 5;
    while (lw > 2 && rem <= (1 << (lw - 1))) --lw;
    items[j] = P2PItem32{l, Tl.boff + t0, rem, lw};
  }
}

}  // namespace

int device_p2p_tables(const DeviceWalk& w, const DeviceLeafInput& in, bool mixed, cudaStream_t st,
                      const TreeScratchFn& scratch, int slot_base, const P2PTableAlloc& alloc, P2PTablesOut* out,
                      std::string& msg) {
  Scratch S{scratch, slot_base};
  const int nlf = in.nlf;
  int *cstart, *cend, *cnt, *icnt, *off, *ioff;
  unsigned long long* total;
  LCK(S.get(0, &cstart, w.ncell));
  LCK(S.get(1, &cend, w.ncell));
  LCK(S.get(2, &cnt, nlf + 1));
  LCK(S.get(3, &icnt, nlf + 1));
  LCK(S.get(4, &ioff, nlf + 1));
  LCK(S.get(5, &total, 1));
  LCK(cudaMemsetAsync(cstart, 0, sizeof(int) * w.ncell, st));
  LCK(cudaMemsetAsync(cend, 0, sizeof(int) * w.ncell, st));
  LCK(cudaMemsetAsync(cnt + nlf, 0, sizeof(int), st));
  LCK(cudaMemsetAsync(icnt + nlf, 0, sizeof(int), st));
  LCK(cudaMemsetAsync(total, 0, sizeof(unsigned long long), st));
  if (w.npairs > 0) {
    k_pair_bounds<<<cdiv(w.npairs, 256), 256, 0, st>>>(w.pairs, w.npairs, cstart, cend);
    LCK(cudaGetLastError());
  }
  LeafTables T{in.leaves, nlf, in.parent, w.cboff, w.cbnum, in.body_leaf, in.dfs, in.dfs_pos, cstart, cend,
               w.pairs, w.offs};
  k_leaf_list_count<<<cdiv(nlf, 128), 128, 0, st>>>(T, cnt, icnt);
  LCK(cudaGetLastError());
  off = alloc.list_off(nlf + 1);
  if (!off) {
    msg = "device allocation of the P2P list offsets failed";
    return kTreeError;
  }
  size_t tb = 0;
  LCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, nlf + 1, st));
  char* tmp = nullptr;
  LCK(S.get(6, &tmp, tb));
  LCK(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, nlf + 1, st));
  LCK(cub::DeviceScan::ExclusiveSum(tmp, tb, icnt, ioff, nlf + 1, st));
  int tot[2];
  LCK(cudaMemcpyAsync(&tot[0], off + nlf, sizeof(int), cudaMemcpyDeviceToHost, st));
  LCK(cudaMemcpyAsync(&tot[1], ioff + nlf, sizeof(int), cudaMemcpyDeviceToHost, st));
  LCK(cudaStreamSynchronize(st));
  P2PSrc32* l32 = nullptr;
  P2PSrc64* l64 = nullptr;
  if (mixed)
    l32 = alloc.list32(tot[0]);
  else
    l64 = alloc.list64(tot[0]);
  P2PItem32* items = alloc.items(tot[1]);
  if ((mixed && !l32) || (!mixed && !l64) || !items) {
    msg = "device allocation of the P2P lists failed";
    return kTreeError;
  }
  k_leaf_list_fill<<<cdiv(nlf, 128), 128, 0, st>>>(T, off, ioff, mixed ? 1 : 0, l32, l64, items, total);
  LCK(cudaGetLastError());
  unsigned long long pairs = 0;
  LCK(cudaMemcpyAsync(&pairs, total, sizeof(pairs), cudaMemcpyDeviceToHost, st));
  LCK(cudaStreamSynchronize(st));
  out->nlist = tot[0];
  out->nitems = tot[1];
  out->pairs = (int64_t)pairs;
  return kTreeOk;
}

#undef LCK

}  // namespace rtfmm_b200
