// The octree of device-resident bodies, built on the GPU.
//
// Tree::build_nonuniform_octree (3dpp/src/tree.cpp:102-188) splits every
// cell holding more than ncrit bodies into its non-empty octants, breadth
// first, with a stable partition of the cell's bodies.  Its result is fixed
// by each body's path of octant digits from the root, so it is built here as:
//
//   1. per body, the digits of levels 1..21, each from the comparison the
//      host split makes (4(x>cx)+2(y>cy)+(z>cz) against the centre of the
//      body's cell one level up, centres halving as Tree::get_child_cell_x,
//      tree.cpp:198-209), packed 3 bits a level into a 64-bit key;
//   2. a stable radix sort of (key, body index): every cell is a contiguous
//      run of the sorted bodies;
//   3. level by level, the cells of a level that hold more than ncrit bodies
//      find their children's runs by binary search on the next digit; child
//      slots are assigned by a prefix sum in (parent, octant) order, which is
//      the breadth-first order of the host build;
//   4. inside each leaf the bodies are put back in input order (the host's
//      repeated stable partitions keep them so), by a second radix sort on
//      (leaf start, body index).
//
// The cells and the permutation are the host builder's, bit for bit: the
// centres are recomputed on the host from the parents exactly as the host
// build does, and only the octants, counts and order come from the device.
// The permutation stays on the device.  A tree that needs more than 21
// levels is left to the host builder.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "rtfmm_tree.h"

namespace rtfmm_b200 {
namespace {

constexpr int kKeyLevels = 21;

__global__ void k_path_keys(const double* __restrict__ x, const double* __restrict__ q, int n, double cx, double cy,
                            double cz, double r0, unsigned long long* __restrict__ key, int* __restrict__ idx,
                            int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
  if (!isfinite(px) || !isfinite(py) || !isfinite(pz) || !isfinite(q[i])) atomicExch(bad, 1);
  double c0 = cx, c1 = cy, c2 = cz, r = r0;
  unsigned long long k = 0;
  for (int l = 0; l < kKeyLevels; ++l) {
    const int o = ((px > c0) << 2) | ((py > c1) << 1) | (pz > c2);
    k = (k << 3) | (unsigned long long)o;
    const double h = r / 2;
    c0 = c0 + ((o & 4) ? h : -h);
    c1 = c1 + ((o & 2) ? h : -h);
    c2 = c2 + ((o & 1) ? h : -h);
    r = h;
  }
  key[i] = k;
  idx[i] = i;
}

// First position in [lo, hi) whose digit (key >> shift & 7) is >= o; the
// digits are non-decreasing there (sorted keys sharing the cell's prefix).
__device__ __forceinline__ int digit_lower_bound(const unsigned long long* key, int lo, int hi, int shift, int o) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((int)((key[mid] >> shift) & 7ull) < o)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Children of one level's cells: nchild[k] (0 for cells kept as leaves) and,
// with `emit`, the child runs written at child_off[k] in octant order.
__global__ void k_split_level(const unsigned long long* __restrict__ key, const int* __restrict__ boff,
                              const int* __restrict__ bnum, int nl, int ncrit, int depth, int* __restrict__ nchild,
                              const int* __restrict__ child_off, int emit, int* __restrict__ nboff,
                              int* __restrict__ nbnum, int* __restrict__ noct, int* __restrict__ npar,
                              int* __restrict__ too_deep) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nl) return;
  const int b0 = boff[k], nb = bnum[k];
  if (nb <= ncrit) {
    if (!emit) nchild[k] = 0;
    return;
  }
  if (depth >= kKeyLevels) {
    atomicExch(too_deep, 1);
    if (!emit) nchild[k] = 0;
    return;
  }
  const int shift = 3 * (kKeyLevels - 1 - depth);
  int start[9];
  for (int o = 0; o < 8; ++o) start[o] = digit_lower_bound(key, b0, b0 + nb, shift, o);
  start[8] = b0 + nb;
  if (!emit) {
    int c = 0;
    for (int o = 0; o < 8; ++o) c += start[o + 1] > start[o];
    nchild[k] = c;
    return;
  }
  int j = child_off[k];
  for (int o = 0; o < 8; ++o) {
    const int cnt = start[o + 1] - start[o];
    if (cnt == 0) continue;
    nboff[j] = start[o];
    nbnum[j] = cnt;
    noct[j] = o;
    npar[j] = k;
    ++j;
  }
}

// (leaf start << 32) | body index for every body of every leaf.
__global__ void k_leaf_keys(const int* __restrict__ lboff, const int* __restrict__ lbnum, int nleaf,
                            const int* __restrict__ idx, unsigned long long* __restrict__ key2) {
  for (int l = blockIdx.x; l < nleaf; l += gridDim.x) {
    const int b0 = lboff[l], nb = lbnum[l];
    for (int t = threadIdx.x; t < nb; t += blockDim.x)
      key2[b0 + t] = ((unsigned long long)(unsigned)b0 << 32) | (unsigned)idx[b0 + t];
  }
}

__global__ void k_perm_out(const unsigned long long* __restrict__ key2, int n, int64_t* __restrict__ perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[i] = (int64_t)(key2[i] & 0xffffffffull);
}

// Scratch buffers by slot from the caller's allocator.
struct Scratch {
  const TreeScratchFn& fn;
  int next = 0;
  template <typename T>
  cudaError_t get(T** out, size_t count) {
    *out = (T*)fn(next++, std::max<size_t>(1, count) * sizeof(T));
    return *out ? cudaSuccess : cudaErrorMemoryAllocation;
  }
};

int cdiv(int64_t a, int b) { return (int)((a + b - 1) / b); }

}  // namespace

#define TCK(call)                                              \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) {                                   \
      msg = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return kTreeError;                                       \
    }                                                          \
  } while (0)

int device_build_tree(const double* x_dev, const double* q_dev, int64_t n64, cudaStream_t st, Plan& plan,
                      int64_t* d_perm, const TreeScratchFn& scratch, std::string& msg) {
  const Args& a = plan.args;
  const int n = (int)n64;
  plan.n = n64;
  plan.r0 = a.cycle / 2;
  plan.cells.clear();
  Cell root;
  root.octant = 13;
  root.depth = 0;
  root.r = plan.r0;
  root.x = a.x;
  root.coff = 0;
  root.cnum = 0;
  root.boff = 0;
  root.bnum = n;
  plan.cells.push_back(root);
  plan.perm.clear();
  if (n == 0) {
    plan.ntree = 1;
    return kTreeOk;
  }
  Scratch B{scratch};
  unsigned long long *key = nullptr, *key_alt = nullptr;
  int *idx = nullptr, *idx_alt = nullptr, *flags = nullptr;
  TCK(B.get(&key, n));
  TCK(B.get(&key_alt, n));
  TCK(B.get(&idx, n));
  TCK(B.get(&idx_alt, n));
  TCK(B.get(&flags, 2));
  TCK(cudaMemsetAsync(flags, 0, 2 * sizeof(int), st));
  k_path_keys<<<cdiv(n, 256), 256, 0, st>>>(x_dev, q_dev, n, a.x[0], a.x[1], a.x[2], plan.r0, key, idx, flags);
  TCK(cudaGetLastError());

  // stable sort by the 63 key bits
  size_t tmp_bytes = 0, t2 = 0;
  TCK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key_alt, idx, idx_alt, n, 0, 3 * kKeyLevels, st));
  TCK(cub::DeviceRadixSort::SortKeys(nullptr, t2, key, key_alt, n, 0, 64, st));
  tmp_bytes = std::max(tmp_bytes, t2);
  int* scan_probe = nullptr;
  TCK(cub::DeviceScan::ExclusiveSum(nullptr, t2, scan_probe, scan_probe, n, st));
  tmp_bytes = std::max(tmp_bytes, t2);
  void* tmp = nullptr;
  TCK(B.get((char**)&tmp, tmp_bytes));
  TCK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key_alt, idx, idx_alt, n, 0, 3 * kKeyLevels, st));
  // sorted keys in key_alt, indices in idx_alt

  // level arrays (a level has at most n cells)
  int *lboff[2], *lbnum[2], *noct = nullptr, *npar = nullptr, *nchild = nullptr, *coff = nullptr;
  for (int s = 0; s < 2; ++s) {
    TCK(B.get(&lboff[s], n));
    TCK(B.get(&lbnum[s], n));
  }
  TCK(B.get(&noct, n));
  TCK(B.get(&npar, n));
  TCK(B.get(&nchild, n));
  TCK(B.get(&coff, n));
  int zero = 0;
  TCK(cudaMemcpyAsync(lboff[0], &zero, sizeof(int), cudaMemcpyHostToDevice, st));
  TCK(cudaMemcpyAsync(lbnum[0], &n, sizeof(int), cudaMemcpyHostToDevice, st));

  size_t lev0 = 0, lev1 = 1;
  int cur = 0, depth = 0;
  std::vector<int> h_nchild, h_coff, h_boff, h_bnum, h_oct, h_par;
  while (true) {
    const int nl = (int)(lev1 - lev0);
    k_split_level<<<cdiv(nl, 128), 128, 0, st>>>(key_alt, lboff[cur], lbnum[cur], nl, a.ncrit, depth, nchild,
                                                nullptr, 0, nullptr, nullptr, nullptr, nullptr, flags + 1);
    TCK(cudaGetLastError());
    TCK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, nchild, coff, nl, st));
    h_nchild.resize(nl);
    h_coff.resize(nl);
    int h_flags[2] = {0, 0};
    TCK(cudaMemcpyAsync(h_nchild.data(), nchild, sizeof(int) * nl, cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(h_coff.data(), coff, sizeof(int) * nl, cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(h_flags, flags, sizeof(h_flags), cudaMemcpyDeviceToHost, st));
    TCK(cudaStreamSynchronize(st));
    if (h_flags[0]) {
      msg = "non-finite body position or charge";
      return kTreeError;
    }
    if (h_flags[1]) return kTreeTooDeep;
    const int total = h_coff[nl - 1] + h_nchild[nl - 1];
    if (total == 0) break;
    k_split_level<<<cdiv(nl, 128), 128, 0, st>>>(key_alt, lboff[cur], lbnum[cur], nl, a.ncrit, depth, nchild,
                                                coff, 1, lboff[cur ^ 1], lbnum[cur ^ 1], noct, npar, flags + 1);
    TCK(cudaGetLastError());
    h_boff.resize(total);
    h_bnum.resize(total);
    h_oct.resize(total);
    h_par.resize(total);
    TCK(cudaMemcpyAsync(h_boff.data(), lboff[cur ^ 1], sizeof(int) * total, cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(h_bnum.data(), lbnum[cur ^ 1], sizeof(int) * total, cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(h_oct.data(), noct, sizeof(int) * total, cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(h_par.data(), npar, sizeof(int) * total, cudaMemcpyDeviceToHost, st));
    TCK(cudaStreamSynchronize(st));
    for (int k = 0; k < nl; ++k) {
      if (h_nchild[k] == 0) continue;
      plan.cells[lev0 + k].coff = (int)lev1 + h_coff[k];
      plan.cells[lev0 + k].cnum = h_nchild[k];
    }
    for (int j = 0; j < total; ++j) {
      const Cell P = plan.cells[lev0 + h_par[j]];  // a copy: the push below may reallocate
      Cell ch;
      ch.octant = h_oct[j];
      ch.depth = P.depth + 1;
      ch.r = P.r / 2;
      // Tree::get_child_cell_x, as the host build computes it
      ch.x[0] = P.x[0] + ((ch.octant & 4) ? P.r / 2 : -P.r / 2);
      ch.x[1] = P.x[1] + ((ch.octant & 2) ? P.r / 2 : -P.r / 2);
      ch.x[2] = P.x[2] + ((ch.octant & 1) ? P.r / 2 : -P.r / 2);
      ch.coff = 0;
      ch.cnum = 0;
      ch.boff = h_boff[j];
      ch.bnum = h_bnum[j];
      plan.cells.push_back(ch);
    }
    lev0 = lev1;
    lev1 = plan.cells.size();
    cur ^= 1;
    ++depth;
  }
  plan.ntree = (int)plan.cells.size();

  // input order inside each leaf
  std::vector<int> lb, ln;
  for (const Cell& c : plan.cells)
    if (c.cnum == 0) {
      lb.push_back(c.boff);
      ln.push_back(c.bnum);
    }
  const int nleaf = (int)lb.size();
  int *d_lb = nullptr, *d_ln = nullptr;
  TCK(B.get(&d_lb, nleaf));
  TCK(B.get(&d_ln, nleaf));
  TCK(cudaMemcpyAsync(d_lb, lb.data(), sizeof(int) * nleaf, cudaMemcpyHostToDevice, st));
  TCK(cudaMemcpyAsync(d_ln, ln.data(), sizeof(int) * nleaf, cudaMemcpyHostToDevice, st));
  k_leaf_keys<<<std::min(nleaf, 4096), 128, 0, st>>>(d_lb, d_ln, nleaf, idx_alt, key);
  TCK(cudaGetLastError());
  int bits = 1;
  while ((1ll << bits) < n64) ++bits;
  TCK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, key, key_alt, n, 0, 32 + bits, st));
  k_perm_out<<<cdiv(n, 256), 256, 0, st>>>(key_alt, n, d_perm);
  TCK(cudaGetLastError());
  return kTreeOk;
}

#undef TCK

}  // namespace rtfmm_b200
