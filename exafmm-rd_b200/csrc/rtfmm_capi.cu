// C ABI of the B200 FMM evaluation pass: handle, device buffers and the
// orchestration of one pass across two CUDA streams.
//
//   stream s0 (far field):  P2M -> M2M levels -> FFT-M2L (up, Hadamard, down)
//                           -> L2L levels -> L2P            ... then post
//   stream s1 (near field): P2P, concurrently with the far field
//
// This is LaplaceFMM::solve (3dpp/src/fmm.cpp:13-81) split at its hot block.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <functional>
#include <mutex>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/rtfmm_b200.h"
#include "rtfmm_kernels.cuh"
#include "rtfmm_plan.h"
#include "rtfmm_precompute.h"
#include "rtfmm_tree.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

using namespace rtfmm_b200;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(e_ == cudaErrorMemoryAllocation ? RTFMM_ENOMEM : RTFMM_ECUDA,               \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

enum Stage { ST_PREP = 0, ST_P2M, ST_M2M, ST_UP, ST_HAD, ST_DOWN, ST_L2L, ST_L2P, ST_P2P, ST_POST, ST_N };

// Vector buffers an operator application reads or writes (row stride ns).
enum BufId { BUF_QEQ = 0, BUF_PCHK, BUF_LEAF, BUF_LEAF2, BUF_Y, BUF_NUM };

struct ApplyCall {
  int groups, S, rows_max;
  size_t inrow_off, outrow_off, scale_off, goff_off;  // offsets into the index / scale pools
  int bsel;        // which operator stack
  int abuf, cbuf;  // BufId of A and C
  int beta;
  bool has_scale;
  size_t sum_off = 0;  // M2M levels: (parent, coff, cnum) triplets summed after the apply
  int nsum = 0;
};

// Operator stacks, each in the [s][j][n] layout of k_apply_f64:
//   P2M  (p2m_precompute, kernel.cpp:369-370): y = U^T p, q = scale * V S^-1 y
//   L2P  (l2p_precompute, kernel.cpp:1465-1467): y = V^T p, q = scale * U S^-1 y
//   M2M per octant (transposed), L2L = M2M^T per octant, image sum / image 13
//   adjoint image levels: the transposes swap roles, so the upward step uses
//   M2M_img[13] (the transpose of the forward L2L_img) and the downward step
//   the transposed 27-image sum
#ifndef USE_PASS_GRAPH
#define USE_PASS_GRAPH 1
#endif
#ifndef STREAM_PRIO
#define STREAM_PRIO 1
#endif

// Largest P at which the FP32-mixed form runs the 8x8 FFT-M2L in FP32 (its
// gradient error stays below 1e-5 on uniform inputs up to P = 8; 3e-5 at 10).
#ifndef M2L32_MAXP
#define M2L32_MAXP 8
#endif
constexpr int kM2L32MaxP = M2L32_MAXP;

enum BSel { B_P2M1 = 0, B_P2M2, B_L2P1, B_L2P2, B_M2MT, B_M2M, B_IMGSUMT, B_IMG13, B_ADJ_IMG_UP, B_ADJ_IMG_DOWN,
            B_NUM };

}  // namespace

struct rtfmm_fmm {
  Args args;
  Plan plan;
  Operators ops;
  bool ops_valid = false;
  bool setup_done = false;
  bool device_ready = false;
  bool pass_done = false;
  std::vector<double> x_in;  // input-order positions of the set-up bodies
  double* h_xin = nullptr;   // pinned copy of x_in (host -> device source)
  std::vector<double> q_in;

  // host plan tables
  std::vector<LeafInfo> leaves;
  std::vector<int> body_leaf;
  std::vector<P2PItem32> items2; // P2P work items (target groups), both precisions
  std::vector<int> list_off;
  int n_items2 = 0;               // work items (host or device built)
  int64_t p2p_pairs = 0;          // body pairs of the P2P lists
  // the P2P lists, offsets and items were built on the GPU (device set-up):
  // the host vectors above are empty
  bool p2p_on_device = false;
  // plan.p2p is empty and the walk's pairs are on the device (f->dwalk)
  bool p2p_lists_on_device = false;
  std::vector<int> h_parent, h_dfs, h_dfs_pos;  // inputs of the device build
  DeviceWalk dwalk;                             // the GPU walk's device output
  std::vector<P2PSrc32> list32;
  std::vector<P2PSrc64> list64;
  std::vector<int> idx_pool;
  std::vector<double> scale_pool;
  std::vector<ApplyCall> p2m_call, m2m_calls, l2l_calls, l2p_call;
  std::vector<int> up8_slots, down8_slots, up27_slots, down27_slots;  // 8 child cells per parent (-1 = none)
  std::vector<int> up8_items, down8_items, up27_items, down27_items;  // 10 ints per block
  int sp_up8 = 8, sp_down8 = 8, sp_up27 = 8, sp_down27 = 8;
  std::vector<int> tsrc8, tsrc27;
  std::vector<double> tscale8, tscale27;
  int nS8 = 0, nT8 = 0, nS27 = 0, nT27 = 0;

  // device
  int dev = -1;
  cudaStream_t s0 = nullptr, s1 = nullptr;
  cudaEvent_t ev_start = nullptr, ev_near0 = nullptr, ev_near = nullptr, ev_stop = nullptr;
  cudaEvent_t ev_st[ST_N] = {};
  // device buffers by the handle field that holds them, kept across set-ups
  // and grown (with a quarter of headroom) only when a plan needs more, so a
  // new body set of similar size reuses them without cudaMalloc/cudaFree
  struct DevSlot {
    void* p = nullptr;
    size_t bytes = 0;
  };
  std::unordered_map<const void*, DevSlot> pool;
  // operator tables: generation built on the host / uploaded to the device
  uint64_t ops_gen = 0, ops_dev_gen = 0;
  size_t h_xin_cap = 0;  // doubles in h_xin
  // x_in, q_in, plan.x, plan.q, plan.perm and h_xin hold the set-up bodies;
  // after a device set-up they are fetched from d_xin, d_qin and d_perm on
  // first use (ensure_host_bodies)
  bool host_bodies = true;
  char tree_slots[64] = {};  // pool keys of the device tree's and walk's scratch
  double4* d_body64 = nullptr;
  float4* d_body32 = nullptr;
  int* d_body_leaf = nullptr;
  int64_t* d_perm = nullptr;
  double *d_xin = nullptr, *d_qin = nullptr;
  double *d_stage_x = nullptr, *d_stage_q = nullptr;  // rtfmm_b200_solve's host bodies on their way in
  LeafInfo* d_leaves = nullptr;
  double *d_qeq = nullptr, *d_pchk = nullptr, *d_leafvec = nullptr, *d_leafvec2 = nullptr, *d_y = nullptr;
  double *d_far_phi = nullptr, *d_far_grad = nullptr, *d_near_phi = nullptr, *d_near_grad = nullptr;
  double *d_out_phi = nullptr, *d_out_grad = nullptr;
  P2PItem32* d_items2 = nullptr;
  int* d_list_off = nullptr;
  P2PSrc32* d_list32 = nullptr;
  P2PSrc64* d_list64 = nullptr;
  double *d_surf_unit = nullptr, *d_twiddle = nullptr;
  int* d_surf_ijk = nullptr;
  double* d_B[B_NUM] = {};
  int* d_idx_pool = nullptr;
  double* d_scale_pool = nullptr;
  void *d_G8 = nullptr, *d_Q8 = nullptr, *d_Pk8 = nullptr;
  double *d_G27 = nullptr, *d_Q27 = nullptr, *d_Pk27 = nullptr;
  int *d_up8 = nullptr, *d_down8 = nullptr, *d_up27 = nullptr, *d_down27 = nullptr;
  int *d_tsrc8 = nullptr, *d_tsrc27 = nullptr;
  double *d_tscale8 = nullptr, *d_tscale27 = nullptr;
  double* d_dip = nullptr;
  void* d_flush = nullptr;
  size_t flush_bytes = 0;
  // adjoint scratch (allocated on first use): tree-order charges, the two
  // gradient fields, and the host path's staging of w, dL/dq and dL/dx
  double *d_adj_q = nullptr, *d_adj_gq = nullptr, *d_adj_gw = nullptr;
  double *d_adj_w = nullptr, *d_adj_dq = nullptr, *d_adj_dx = nullptr;
  cudaEvent_t ev_adj0 = nullptr, ev_adj1 = nullptr;
  // d_out_grad holds grad(phi) of the bodies' current charges without the
  // dipole correction (the last pass was such a forward pass)
  bool grad_q_valid = false;
  // d_body64 holds this set-up's positions (tree order); an evaluate then
  // only moves the charges
  bool pos_on_device = false;
  // set-up wall times (s): tree, lists, operators (0 when cached), host
  // tables, the setup call, and the upload of the device tables (in the call
  // that did it)
  double setup_s[12] = {};
  // the forward pass captured as a CUDA graph (launch_pass), dropped with
  // the device tables
  cudaGraphExec_t pass_graph = nullptr;
  bool graph_grad_q_valid = false;
  cudaEvent_t ev_g0 = nullptr, ev_g1 = nullptr;
  // the 8x8 FFT-M2L (up, Hadamard, down) runs in FP32: the mixed form at P <= 8
  bool m2l32 = false;
  // mixed form: the P2P pairs much closer than their leaves (tree-order
  // target t: pairs d_close_pairs[d_close_off[t] .. d_close_off[t+1]]),
  // found once per set of device positions, refined to FP64 every pass
  // sharding (rtfmm_b200_shard): this rank computes the bodies of the leaves
  // whose first body lies in its share of the tree-order body range, and the
  // cells above them; shard_n == 1 is the whole pass
  int shard_rank = 0, shard_n = 1;
  bool shard_up = false;  // the upward phase ran; the downward may follow
  std::vector<char> cell_own;       // per cell (image cells too): computed here
  std::vector<int> own_leaves;      // leaf-table indices of the leaves computed here
  std::vector<LeafInfo> leaves_own;
  LeafInfo* d_leaves_own = nullptr;  // == d_leaves without sharding
  int* d_leaf_cells = nullptr;      // cell of every leaf (leaf-table order)
  char* d_leaf_own = nullptr;
  int* d_close_cnt = nullptr;
  int* d_close_off = nullptr;
  int2* d_close_pairs = nullptr;
  void* d_close_tmp = nullptr;
  int64_t n_close = 0;
  bool close_valid = false;
  float stage_ms[ST_N] = {};
  int64_t launches = 0;
};

namespace {

// *p = the pooled buffer of slot `key` (default: the field p itself) with
// room for count elements, reallocated only when the slot is too small
// (cudaFree waits for the device, so no pending work still reads it).
template <typename T>
int dalloc(rtfmm_fmm* f, T** p, size_t count, const void* key = nullptr) {
  *p = nullptr;
  const size_t need = sizeof(T) * std::max<size_t>(count, 1);
  rtfmm_fmm::DevSlot& slot = f->pool[key ? key : (const void*)p];
  if (slot.bytes < need) {
    if (slot.p) CK(cudaFree(slot.p));
    slot.p = nullptr;
    slot.bytes = 0;
    size_t cap = need + need / 4;
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, cap);
    if (e != cudaSuccess) {
      cudaGetLastError();
      cap = need;
      e = cudaMalloc(&q, cap);
    }
    if (e != cudaSuccess)
      return fail(RTFMM_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    slot.p = q;
    slot.bytes = cap;
  }
  *p = reinterpret_cast<T*>(slot.p);
  return RTFMM_OK;
}

template <typename T>
int dupload(rtfmm_fmm* f, T** p, const std::vector<T>& h, const void* key = nullptr) {
  int rc = dalloc(f, p, h.size(), key);
  if (rc) return rc;
  if (!h.empty()) CK(cudaMemcpy(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return RTFMM_OK;
}

void drop_graph(rtfmm_fmm* f) {
  if (f->pass_graph) {
    cudaGraphExecDestroy(f->pass_graph);
    f->pass_graph = nullptr;
  }
}

// Forgets the device state of the current plan: the captured pass graph and
// the lazily sized adjoint scratch (fetched from the pool again at its next
// use).  The buffers themselves stay in the pool.
void drop_allocs(rtfmm_fmm* f) {
  drop_graph(f);
  f->close_valid = false;
  f->n_close = 0;
  f->d_adj_q = f->d_adj_gq = f->d_adj_gw = f->d_adj_w = f->d_adj_dq = f->d_adj_dx = nullptr;
  f->grad_q_valid = false;
  f->pos_on_device = false;
}

void free_device(rtfmm_fmm* f) {
  if (f->dev >= 0) cudaSetDevice(f->dev);
  if (f->h_xin) {
    cudaFreeHost(f->h_xin);
    f->h_xin = nullptr;
  }
  f->h_xin_cap = 0;
  drop_allocs(f);
  for (auto& kv : f->pool)
    if (kv.second.p) cudaFree(kv.second.p);
  f->pool.clear();
  f->ops_dev_gen = 0;
  f->d_flush = nullptr;
  f->flush_bytes = 0;
  if (f->s0) cudaStreamDestroy(f->s0);
  if (f->s1) cudaStreamDestroy(f->s1);
  f->s0 = f->s1 = nullptr;
  cudaEvent_t* evs[] = {&f->ev_start, &f->ev_near0, &f->ev_near, &f->ev_stop, &f->ev_adj0, &f->ev_adj1,
                        &f->ev_g0, &f->ev_g1};
  for (auto e : evs)
    if (*e) {
      cudaEventDestroy(*e);
      *e = nullptr;
    }
  for (int k = 0; k < ST_N; ++k)
    if (f->ev_st[k]) {
      cudaEventDestroy(f->ev_st[k]);
      f->ev_st[k] = nullptr;
    }
  f->device_ready = false;
}

double wall_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool finite_all(const double* a, int64_t n) {
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad) if (n > (1 << 16))
  for (int64_t i = 0; i < n; ++i) bad |= !std::isfinite(a[i]);
  return !bad;
}

// Longest root-to-leaf path of the octree (its depth limit is 40).
constexpr int kMaxPath = 48;

void build_pass_tables(rtfmm_fmm* f);

// Host tables for the device pass, derived from the plan.  Without
// host_p2p the P2P lists and items are left to the GPU (device_p2p_tables).
void build_tables(rtfmm_fmm* f, bool host_p2p = true) {
  Plan& p = f->plan;
  f->leaves.clear();
  for (int c = 0; c < p.ntree; ++c) {
    const Cell& cl = p.cells[c];
    if (cl.cnum != 0) continue;
    LeafInfo L;
    L.cx = cl.x[0];
    L.cy = cl.x[1];
    L.cz = cl.x[2];
    L.r = cl.r;
    L.scale = std::pow(0.5, cl.depth);
    L.cell = c;
    L.boff = cl.boff;
    L.bnum = cl.bnum;
    f->leaves.push_back(L);
  }
  // each body's leaf (a device set-up fills it on the GPU, k_body_leaf)
  if (host_p2p) {
    f->body_leaf.assign(p.n, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int l = 0; l < (int)f->leaves.size(); ++l)
      for (int b = 0; b < f->leaves[l].bnum; ++b) f->body_leaf[f->leaves[l].boff + b] = l;
  } else {
    f->body_leaf.clear();
  }

  // P2P lists in CSR by target leaf; work items of 32 / 64 targets.  The
  // reference's M2P/P2L-to-P2P conversions (traverser.cpp:75-86) can pair a
  // non-leaf cell with a leaf, evaluated over the cell's whole body range
  // (p2p_1toN_256, kernel.cpp:276-301).  Such a pair is expanded here into
  // the leaf pairs beneath it (same bodies, same sum), so that every list
  // entry is leaf to leaf and FP32 positions can stay leaf-relative.
  //
  // A target leaf's list is: for every cell on its root-to-leaf path that
  // has a P2P list (ascending cell index, the order the lists are keyed by),
  // each entry in list order, expanded into the source's leaves in
  // depth-first order.  The leaves under a cell are the ones whose bodies
  // lie in the cell's body range: a contiguous run of the leaves sorted by
  // their first body.  Each leaf's list is counted, then filled, in
  // parallel.
  const int nlf = (int)f->leaves.size();
  std::vector<int>& parent = f->h_parent;
  parent.assign(p.ntree, -1);
  for (int c = 0; c < p.ntree; ++c)
    for (int k = 0; k < p.cells[c].cnum; ++k)
      if (p.cells[c].coff + k < p.ntree) parent[p.cells[c].coff + k] = c;
  std::vector<int>& dfs = f->h_dfs;
  std::vector<int>& dfs_pos = f->h_dfs_pos;
  dfs.resize(nlf);
  dfs_pos.resize(nlf);
  {
    // leaves by first body: the tree's depth-first order (children in
    // octant order own consecutive body ranges), walked without a sort
    std::vector<int> leaf_of(p.ntree, -1);
    for (int l = 0; l < nlf; ++l) leaf_of[f->leaves[l].cell] = l;
    std::vector<int> stack;
    int k = 0;
    if (p.ntree > 0) stack.push_back(0);
    while (!stack.empty()) {
      const int c = stack.back();
      stack.pop_back();
      const Cell& cl = p.cells[c];
      if (cl.cnum == 0) {
        if (leaf_of[c] >= 0) dfs[k++] = leaf_of[c];
        continue;
      }
      for (int j = cl.cnum - 1; j >= 0; --j) stack.push_back(cl.coff + j);
    }
    for (int i = 0; i < nlf; ++i) dfs_pos[dfs[i]] = i;
  }
  // ownership: leaf l belongs to rank floor(boff * R / n); a cell is
  // computed by every rank that owns a leaf beneath it (image cells by all)
  {
    const int R = std::max(1, f->shard_n);
    f->cell_own.assign(p.cells.size(), R == 1 ? 1 : 0);
    f->own_leaves.clear();
    for (int l = 0; l < nlf; ++l) {
      const int owner = p.n > 0 ? (int)((int64_t)f->leaves[l].boff * R / p.n) : 0;
      if (R > 1 && owner != f->shard_rank) continue;
      f->own_leaves.push_back(l);
      if (R > 1)
        for (int a = f->leaves[l].cell; a >= 0 && !f->cell_own[a]; a = parent[a]) f->cell_own[a] = 1;
    }
    for (size_t c = p.ntree; c < p.cells.size(); ++c) f->cell_own[c] = 1;
    f->leaves_own.clear();
    for (int l : f->own_leaves) f->leaves_own.push_back(f->leaves[l]);
  }
  f->p2p_on_device = !host_p2p;
  if (!host_p2p) {
    f->list_off.clear();
    f->list32.clear();
    f->list64.clear();
    f->items2.clear();
    build_pass_tables(f);
    return;
  }
  auto leaf_run = [&](int c, int* lo, int* hi) {
    const Cell& cl = p.cells[c];
    if (cl.bnum == 0) {  // an empty root leaf (no bodies): itself
      *lo = 0;
      *hi = nlf;
      return;
    }
    *lo = dfs_pos[f->body_leaf[cl.boff]];
    *hi = dfs_pos[f->body_leaf[cl.boff + cl.bnum - 1]] + 1;
  };
  auto path_lists = [&](int c, int* path) {  // cells root..c with a P2P list
    int k = 0;
    for (int a = c; a >= 0; a = parent[a])
      if (!p.p2p.at(a).empty()) path[k++] = a;
    std::reverse(path, path + k);
    return k;
  };
  f->list_off.assign(nlf + 1, 0);
  std::vector<int> item_off(nlf + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int l = 0; l < nlf; ++l) {
    int path[kMaxPath];
    const int np = path_lists(f->leaves[l].cell, path);
    int64_t cnt = 0;
    for (int i = 0; i < np; ++i)
      for (const P2PEntry& e : p.p2p.at(path[i])) {
        int lo, hi;
        leaf_run(e.src, &lo, &hi);
        cnt += hi - lo;
      }
    f->list_off[l + 1] = (int)cnt;
    item_off[l + 1] = (f->leaves[l].bnum + 31) / 32;
  }
  for (int l = 0; l < nlf; ++l) {
    f->list_off[l + 1] += f->list_off[l];
    item_off[l + 1] += item_off[l];
  }
  // the list form of the handle's precision only
  const bool mixed = f->args.precision == RTFMM_FP32_MIXED;
  f->list32.assign(mixed ? f->list_off[nlf] : 0, P2PSrc32{});
  f->list64.assign(mixed ? 0 : f->list_off[nlf], P2PSrc64{});
  f->items2.assign(item_off[nlf], P2PItem32{});
  f->n_items2 = item_off[nlf];
  int64_t pairs = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : pairs)
  for (int l = 0; l < nlf; ++l) {
    const int c = f->leaves[l].cell;
    const Cell& T = p.cells[c];
    int path[kMaxPath];
    const int np = path_lists(c, path);
    int k = f->list_off[l];
    for (int i = 0; i < np; ++i)
      for (const P2PEntry& e : p.p2p.at(path[i])) {
        int lo, hi;
        leaf_run(e.src, &lo, &hi);
        for (int r = lo; r < hi; ++r) {
          const int sl = dfs[r];
          const Cell& S = p.cells[f->leaves[sl].cell];
          P2PSrc32 a;
          a.dx = (float)(S.x[0] + e.off[0] - T.x[0]);
          a.dy = (float)(S.x[1] + e.off[1] - T.x[1]);
          a.dz = (float)(S.x[2] + e.off[2] - T.x[2]);
          a.leaf = sl;
          a.self = (f->leaves[sl].cell == c && e.off[0] == 0 && e.off[1] == 0 && e.off[2] == 0) ? 1 : 0;
          a.boff = f->leaves[sl].boff;
          a.bnum = f->leaves[sl].bnum;
          a.pad = 0;
          pairs += (int64_t)f->leaves[l].bnum * a.bnum;
          if (mixed) {
            f->list32[k] = a;
          } else {
            P2PSrc64 b;
            b.ox = e.off[0];
            b.oy = e.off[1];
            b.oz = e.off[2];
            b.leaf = sl;
            b.self = a.self;
            b.boff = a.boff;
            b.bnum = a.bnum;
            f->list64[k] = b;
          }
          ++k;
        }
      }
    // FP32 items: 32 targets each; the last <= 16 targets of a leaf take a
    // narrower group (W = 16, 8 or 4 lanes) and split the sources 32/W ways
    int j = item_off[l];
    for (int t0 = 0; t0 < f->leaves[l].bnum; t0 += 32, ++j) {
      const int rem = std::min(32, f->leaves[l].bnum - t0);
      int lw = 5;
      while (lw > 2 && rem <= (1 << (lw - 1))) --lw;
      f->items2[j] = {l, f->leaves[l].boff + t0, rem, lw};
    }
  }
  f->p2p_pairs = pairs;
  if (f->shard_n > 1) {  // this rank's targets only
    std::vector<P2PItem32> mine;
    std::vector<char> own(nlf, 0);
    for (int l : f->own_leaves) own[l] = 1;
    for (const P2PItem32& it : f->items2)
      if (own[it.leaf]) mine.push_back(it);
    f->items2.swap(mine);
    f->n_items2 = (int)f->items2.size();
  }
  build_pass_tables(f);
}

// The far-field tables: batched operator applications (P2M, M2M, L2L, L2P)
// and the FFT-M2L source/target lists.
void build_pass_tables(rtfmm_fmm* f) {
  Plan& p = f->plan;
  const Operators& o = f->ops;
  const int ns = o.ns;

  // batched operator applications
  f->idx_pool.clear();
  f->scale_pool.clear();
  auto add_call = [&](std::vector<ApplyCall>& dst, int S, const std::vector<std::vector<int>>& in_by_group,
                      const std::vector<std::vector<int>>& out_by_group, const std::vector<double>* scale,
                      int bsel, int abuf, int cbuf, int beta) {
    ApplyCall ac;
    ac.groups = (int)out_by_group.size();
    ac.S = S;
    ac.rows_max = 0;
    ac.bsel = bsel;
    ac.abuf = abuf;
    ac.cbuf = cbuf;
    ac.beta = beta;
    ac.has_scale = scale != nullptr;
    ac.goff_off = f->idx_pool.size();
    int acc = 0;
    for (auto& g : out_by_group) {
      f->idx_pool.push_back(acc);
      acc += (int)g.size();
      ac.rows_max = std::max(ac.rows_max, (int)g.size());
    }
    f->idx_pool.push_back(acc);
    ac.inrow_off = f->idx_pool.size();
    for (auto& g : in_by_group) f->idx_pool.insert(f->idx_pool.end(), g.begin(), g.end());
    ac.outrow_off = f->idx_pool.size();
    for (auto& g : out_by_group) f->idx_pool.insert(f->idx_pool.end(), g.begin(), g.end());
    ac.scale_off = f->scale_pool.size();
    if (scale) f->scale_pool.insert(f->scale_pool.end(), scale->begin(), scale->end());
    if (acc > 0) dst.push_back(ac);
  };
  f->p2m_call.clear();
  f->m2m_calls.clear();
  f->l2l_calls.clear();
  f->l2p_call.clear();
  {
    // rows of the leaf vectors are this rank's leaves (all without sharding)
    std::vector<int> out;
    std::vector<double> sc;
    for (const LeafInfo& L : f->leaves_own) {
      out.push_back(L.cell);
      sc.push_back(L.scale);
    }
    std::vector<int> lid(f->leaves_own.size());
    for (int l = 0; l < (int)lid.size(); ++l) lid[l] = l;
    add_call(f->p2m_call, 1, {lid}, {lid}, nullptr, B_P2M1, BUF_LEAF, BUF_LEAF2, 0);
    add_call(f->p2m_call, 1, {lid}, {out}, &sc, B_P2M2, BUF_LEAF2, BUF_QEQ, 0);
    add_call(f->l2p_call, 1, {out}, {lid}, nullptr, B_L2P1, BUF_PCHK, BUF_LEAF, 0);
    add_call(f->l2p_call, 1, {lid}, {lid}, &sc, B_L2P2, BUF_LEAF, BUF_LEAF2, 0);
  }
  // the non-leaf cells of each depth, in cell order
  std::vector<std::vector<int>> by_depth(p.dmax - p.dmin + 1);
  for (int c = 0; c < (int)p.cells.size(); ++c)
    if (p.cells[c].cnum != 0) by_depth[p.cells[c].depth - p.dmin].push_back(c);
  // M2M bottom-up (fmm.cpp:111-150): depth = dmax .. dmin+1.  For depth >= 0
  // each child's contribution M2M[octant] q_child is one row of a batched
  // apply grouped by octant (into the Y scratch), then each parent sums its
  // children in crange order (m2m_precompute, kernel.cpp:395-404).
  for (int depth = p.dmax; depth > p.dmin; --depth) {
    std::vector<std::vector<int>> in(8), out(8);
    std::vector<int> in1, out1, sums;
    for (int c : by_depth[depth - p.dmin]) {
      const Cell& cl = p.cells[c];
      if (depth >= 0) {
        for (int k = 0; k < cl.cnum; ++k) {
          const int ch = cl.coff + k;
          in[p.cells[ch].octant].push_back(ch);
          out[p.cells[ch].octant].push_back(ch);
        }
        sums.push_back(c);
        sums.push_back(cl.coff);
        sums.push_back(cl.cnum);
      } else {
        in1.push_back(cl.coff);
        out1.push_back(c);
      }
    }
    if (depth >= 0 && !sums.empty()) {
      add_call(f->m2m_calls, 1, in, out, nullptr, B_M2MT, BUF_QEQ, BUF_Y, 0);
      f->m2m_calls.back().sum_off = f->idx_pool.size();
      f->m2m_calls.back().nsum = (int)sums.size() / 3;
      f->idx_pool.insert(f->idx_pool.end(), sums.begin(), sums.end());
    } else if (depth < 0 && !out1.empty()) {
      add_call(f->m2m_calls, 1, {in1}, {out1}, nullptr, B_IMGSUMT, BUF_QEQ, BUF_QEQ, 0);
    }
  }
  // L2L top-down (fmm.cpp:195-229): depth = dmin .. dmax-1
  for (int depth = p.dmin; depth < p.dmax; ++depth) {
    std::vector<std::vector<int>> in(8), out(8);
    std::vector<int> in1, out1;
    for (int c : by_depth[depth - p.dmin]) {
      const Cell& cl = p.cells[c];
      if (!f->cell_own[c]) continue;
      if (depth >= 0) {
        for (int k = 0; k < cl.cnum; ++k) {
          const int ch = cl.coff + k;
          in[p.cells[ch].octant].push_back(c);
          out[p.cells[ch].octant].push_back(ch);
        }
      } else {
        in1.push_back(c);
        out1.push_back(cl.coff);
      }
    }
    if (depth >= 0) {
      bool any = false;
      for (auto& g : out) any |= !g.empty();
      if (any) add_call(f->l2l_calls, 1, in, out, nullptr, B_M2M, BUF_PCHK, BUF_PCHK, 1);
    } else if (!out1.empty()) {
      add_call(f->l2l_calls, 1, {in1}, {out1}, nullptr, B_IMG13, BUF_PCHK, BUF_PCHK, 1);
    }
  }

  // FFT-M2L lists (m2l_fft_precompute_t, kernel.cpp:1153-1245).  Source
  // and target parents of the 8x8 products are numbered level by level in
  // row-major order of their lattice coordinates (x fastest): a warp of the
  // Hadamard takes consecutive targets, and the sources of consecutive
  // targets in one direction are then mostly consecutive rows of the
  // spectra.  The 1x27 image-level ones in ascending cell index (s8/s27:
  // cell -> number, -1 for none).
  const int ncell = (int)p.cells.size();
  std::vector<int> s8(ncell, -1), s27(ncell, -1);
  std::vector<int> t8cells, t27cells;
  for (const auto& kv : p.m2l) {
    if (!f->cell_own[kv.first]) continue;  // another rank's targets
    bool single = false, normal = false;
    for (const M2LEntry& e : kv.second) (e.single ? single : normal) = true;
    if (normal) t8cells.push_back(kv.first);
    if (single) t27cells.push_back(kv.first);
    for (const M2LEntry& e : kv.second) (e.single ? s27 : s8)[e.src] = 0;
  }
  {
    const V3 lo{p.args.x[0] - p.r0, p.args.x[1] - p.r0, p.args.x[2] - p.r0};
    auto lattice_key = [&](int c) {
      const Cell& cl = p.cells[c];
      int64_t m[3];
      for (int k = 0; k < 3; ++k) m[k] = (int64_t)std::llround((cl.x[k] - lo[k]) / (2 * cl.r) - 0.5);
      const int64_t side = c < p.ntree && cl.depth >= 0 ? (int64_t)1 << cl.depth : 1;
      const int64_t lin = c < p.ntree ? (m[2] * side + m[1]) * side + m[0] : c;
      return std::make_pair((int64_t)cl.depth + (c < p.ntree ? 0 : 1000), lin);
    };
    std::vector<std::pair<std::pair<int64_t, int64_t>, int>> key8;
    for (int c = 0; c < ncell; ++c)
      if (s8[c] >= 0) key8.push_back({lattice_key(c), c});
    std::sort(key8.begin(), key8.end());
    for (int k = 0; k < (int)key8.size(); ++k) s8[key8[k].second] = k;
    std::vector<std::pair<std::pair<int64_t, int64_t>, int>> keyt;
    for (int c : t8cells) keyt.push_back({lattice_key(c), c});
    std::sort(keyt.begin(), keyt.end());
    for (int k = 0; k < (int)keyt.size(); ++k) t8cells[k] = keyt[k].second;
  }
  int k8 = 0, k27 = 0;
  for (int c = 0; c < ncell; ++c) {
    if (s8[c] >= 0) ++k8;
    if (s27[c] >= 0) s27[c] = k27++;
  }
  f->nS8 = k8;
  f->nS27 = k27;
  f->nT8 = (int)t8cells.size();
  f->nT27 = (int)t27cells.size();
  auto child_slot = [&](int ch) { return p.cells[ch].octant == 13 ? 0 : p.cells[ch].octant; };
  f->up8_slots.assign((size_t)f->nS8 * 8, -1);
  f->up27_slots.assign((size_t)f->nS27 * 8, -1);
  for (int c0 = 0; c0 < ncell; ++c0) {
    const Cell& cl = p.cells[c0];
    if (s8[c0] >= 0)
      for (int c = 0; c < cl.cnum; ++c) f->up8_slots[(size_t)s8[c0] * 8 + child_slot(cl.coff + c)] = cl.coff + c;
    if (s27[c0] >= 0) f->up27_slots[(size_t)s27[c0] * 8] = cl.coff;
  }
  auto direction = [&](int t, const M2LEntry& e) {
    const Cell& T = p.cells[t];
    const Cell& S = p.cells[e.src];
    int v[3];
    for (int q = 0; q < 3; ++q) v[q] = (int)std::lround((S.x[q] + e.off[q] - T.x[q]) / (T.r * 2));
    int d = (v[2] + 1) * 9 + (v[1] + 1) * 3 + (v[0] + 1);
    return d > 13 ? d - 1 : d;
  };
  const double N3 = (double)o.N * o.N * o.N;
  auto fill_targets = [&](const std::vector<int>& tcells, bool single, const std::vector<int>& smap,
                          std::vector<int>& tsrc, std::vector<double>& tscale, std::vector<int>& down) {
    tsrc.assign(tcells.size() * 26, -1);
    tscale.assign(tcells.size(), 0.0);
    down.assign(tcells.size() * 8, -1);
#pragma omp parallel for schedule(static)
    for (int ti = 0; ti < (int)tcells.size(); ++ti) {
      const int t = tcells[ti];
      for (const M2LEntry& e : p.m2l.at(t)) {
        if ((e.single != 0) != single) continue;
        tsrc[(size_t)ti * 26 + direction(t, e)] = smap[e.src];
      }
      const Cell& T = p.cells[t];
      tscale[ti] = std::pow(T.depth >= -1 ? 2.0 : 3.0, T.depth + 1) / N3;
      for (int c = 0; c < T.cnum; ++c) down[(size_t)ti * 8 + child_slot(T.coff + c)] = T.coff + c;
    }
  };
  fill_targets(t8cells, false, s8, f->tsrc8, f->tscale8, f->down8_slots);
  fill_targets(t27cells, true, s27, f->tsrc27, f->tscale27, f->down27_slots);
  (void)ns;
}

int ensure_device(rtfmm_fmm* f) {
  if (f->dev != f->args.device || !f->s0) {
    free_device(f);
    CK(cudaSetDevice(f->args.device));
    f->dev = f->args.device;
    // the far field (a chain of dependent kernels, s0) at the highest
    // priority, P2P (one large independent kernel, s1) at the lowest, so that
    // pending P2P blocks fill the SMs the far-field chain leaves idle
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
#if STREAM_PRIO
    CK(cudaStreamCreateWithPriority(&f->s0, cudaStreamNonBlocking, prio_hi));
    CK(cudaStreamCreateWithPriority(&f->s1, cudaStreamNonBlocking, prio_lo));
#else
    CK(cudaStreamCreateWithFlags(&f->s0, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&f->s1, cudaStreamNonBlocking));
#endif
    CK(cudaEventCreate(&f->ev_start));
    CK(cudaEventCreate(&f->ev_near0));
    CK(cudaEventCreate(&f->ev_near));
    CK(cudaEventCreate(&f->ev_stop));
    CK(cudaEventCreate(&f->ev_adj0));
    CK(cudaEventCreate(&f->ev_adj1));
    CK(cudaEventCreate(&f->ev_g0));
    CK(cudaEventCreate(&f->ev_g1));
    for (int k = 0; k < ST_N; ++k) CK(cudaEventCreate(&f->ev_st[k]));
  } else {
    CK(cudaSetDevice(f->dev));
  }
  return RTFMM_OK;
}

// The operator tables of f->ops on the device (surfaces, DFT twiddles, the
// FP64 operator stacks, the M2L kernel spectra): once per set of operators.
int upload_operators(rtfmm_fmm* f) {
  const Operators& o = f->ops;
  const int ns = o.ns, Nf = o.Nf;
#define RC(x)          \
  do {                 \
    int r_ = (x);      \
    if (r_) return r_; \
  } while (0)
  RC(dupload(f, &f->d_surf_unit, o.surf_unit));
  RC(dupload(f, &f->d_surf_ijk, o.surf_ijk));
  std::vector<double> tw(2 * o.N);
  for (int m = 0; m < o.N; ++m) {
    tw[2 * m] = std::cos(2.0 * M_PI * m / o.N);
    tw[2 * m + 1] = -std::sin(2.0 * M_PI * m / o.N);
  }
  RC(dupload(f, &f->d_twiddle, tw));
  // operator stacks in the [s][j][n] layout of k_apply_f64
  const size_t nn = (size_t)ns * ns;
  std::vector<double> b;
  b = o.U;  // y[n] = sum_j U^T[n][j] p[j]
  RC(dupload(f, &f->d_B[B_P2M1], b));
  b.assign(nn, 0.0);
  for (int j = 0; j < ns; ++j)
    for (int i = 0; i < ns; ++i) b[(size_t)j * ns + i] = o.V[(size_t)i * ns + j] * o.sinv[j];
  RC(dupload(f, &f->d_B[B_P2M2], b));
  b = o.V;  // y[n] = sum_j V^T[n][j] p[j]
  RC(dupload(f, &f->d_B[B_L2P1], b));
  b.assign(nn, 0.0);
  for (int j = 0; j < ns; ++j)
    for (int i = 0; i < ns; ++i) b[(size_t)j * ns + i] = o.U[(size_t)i * ns + j] * o.sinv[j];
  RC(dupload(f, &f->d_B[B_L2P2], b));
  b.assign(8 * nn, 0.0);
  for (int oc = 0; oc < 8; ++oc)
    for (int j = 0; j < ns; ++j)
      for (int i = 0; i < ns; ++i) b[oc * nn + (size_t)j * ns + i] = o.m2m[oc][(size_t)i * ns + j];
  RC(dupload(f, &f->d_B[B_M2MT], b));
  b.assign(8 * nn, 0.0);
  for (int oc = 0; oc < 8; ++oc) std::memcpy(&b[oc * nn], o.m2m[oc].data(), sizeof(double) * nn);
  RC(dupload(f, &f->d_B[B_M2M], b));
  b.assign(nn, 0.0);
  for (int j = 0; j < ns; ++j)
    for (int i = 0; i < ns; ++i) b[(size_t)j * ns + i] = o.m2m_img_sum[(size_t)i * ns + j];
  RC(dupload(f, &f->d_B[B_IMGSUMT], b));
  b.assign(nn, 0.0);
  for (int j = 0; j < ns; ++j)
    for (int i = 0; i < ns; ++i) b[(size_t)j * ns + i] = o.l2l_img[(size_t)i * ns + j];
  RC(dupload(f, &f->d_B[B_IMG13], b));
  // adjoint: upward y = M2M_img[13] x (B[j][n] = L2L_img[j][n]); downward
  // y = (sum of M2M_img)^T x (B[j][n] = sum[j][n])
  RC(dupload(f, &f->d_B[B_ADJ_IMG_UP], o.l2l_img));
  RC(dupload(f, &f->d_B[B_ADJ_IMG_DOWN], o.m2m_img_sum));
  // M2L: kernel spectra re-laid frequency-major, G[f][d][pair], on the GPU
  // from a staging copy of cc8
  {
    double* stage = nullptr;
    CK(cudaMalloc(&stage, sizeof(double) * std::max<size_t>(1, o.cc8.size())));
    cudaError_t e = cudaMemcpy(stage, o.cc8.data(), sizeof(double) * o.cc8.size(), cudaMemcpyHostToDevice);
    if (f->m2l32) {
      float* gp = nullptr;
      int rc = dalloc(f, &gp, o.cc8.size(), &f->d_G8);
      if (rc) {
        cudaFree(stage);
        return rc;
      }
      f->d_G8 = gp;
      if (e == cudaSuccess) e = launch_g8_layout<float>(stage, Nf, gp, f->s0);
    } else {
      double* gp = nullptr;
      int rc = dalloc(f, &gp, o.cc8.size(), &f->d_G8);
      if (rc) {
        cudaFree(stage);
        return rc;
      }
      f->d_G8 = gp;
      if (e == cudaSuccess) e = launch_g8_layout<double>(stage, Nf, gp, f->s0);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(f->s0);
    cudaFree(stage);
    CK(e);
  }
  RC(dupload(f, &f->d_G27, o.cc27sum));
#undef RC
  (void)ns;
  return RTFMM_OK;
}

// Upload the plan (everything but the per-pass body values) to the device.
int upload_plan(rtfmm_fmm* f) {
  const double t0 = wall_s();
  int rc = ensure_device(f);
  if (rc) return rc;
  // a previous plan's buffers are reused (grown if needed); nothing of it
  // may still run
  CK(cudaDeviceSynchronize());
  drop_allocs(f);
  Plan& p = f->plan;
  const Operators& o = f->ops;
  const int64_t n = p.n;
  const int ns = o.ns, Nf = o.Nf;
  const size_t ncell = p.cells.size(), nleaf = f->leaves.size();
  const bool mixed = f->args.precision == RTFMM_FP32_MIXED;
#define RC(x)          \
  do {                 \
    int r_ = (x);      \
    if (r_) return r_; \
  } while (0)
  RC(dalloc(f, &f->d_body64, n));
  RC(dalloc(f, &f->d_body32, n));
  if (f->body_leaf.empty() && n > 0) {
    RC(dalloc(f, &f->d_body_leaf, n));  // filled below from the leaf table
  } else {
    RC(dupload(f, &f->d_body_leaf, f->body_leaf));
  }
  if (f->host_bodies)
    RC(dupload(f, &f->d_perm, p.perm));
  else
    RC(dalloc(f, &f->d_perm, n));  // written by the device tree
  RC(dalloc(f, &f->d_xin, 3 * n));
  RC(dalloc(f, &f->d_qin, n));
  RC(dupload(f, &f->d_leaves, f->leaves));
  if (f->body_leaf.empty() && n > 0) CK(launch_body_leaf(f->d_leaves, (int)nleaf, (int)n, f->d_body_leaf, f->s0));
  {
    // the exchange of a two-phase pass: every leaf's cell, and which leaves
    // this rank computes
    std::vector<int> lc(nleaf);
    std::vector<char> lo(nleaf, 0);
    for (size_t l = 0; l < nleaf; ++l) lc[l] = f->leaves[l].cell;
    for (int l : f->own_leaves) lo[l] = 1;
    RC(dupload(f, &f->d_leaf_cells, lc));
    RC(dupload(f, &f->d_leaf_own, lo));
  }
  if (f->shard_n > 1)
    RC(dupload(f, &f->d_leaves_own, f->leaves_own));
  else
    f->d_leaves_own = f->d_leaves;
  RC(dalloc(f, &f->d_qeq, ncell * ns));
  RC(dalloc(f, &f->d_pchk, ncell * ns));
  RC(dalloc(f, &f->d_leafvec, nleaf * ns));
  RC(dalloc(f, &f->d_leafvec2, nleaf * ns));
  RC(dalloc(f, &f->d_y, ncell * ns));
  RC(dalloc(f, &f->d_far_phi, n));
  RC(dalloc(f, &f->d_far_grad, 3 * n));
  RC(dalloc(f, &f->d_near_phi, n));
  RC(dalloc(f, &f->d_near_grad, 3 * n));
  RC(dalloc(f, &f->d_out_phi, n));
  RC(dalloc(f, &f->d_out_grad, 3 * n));
  if (!f->p2p_on_device) {  // else device_p2p_tables writes them
    RC(dupload(f, &f->d_items2, f->items2));
    RC(dupload(f, &f->d_list_off, f->list_off));
    if (mixed)
      RC(dupload(f, &f->d_list32, f->list32));
    else
      RC(dupload(f, &f->d_list64, f->list64));
  }
  RC(dupload(f, &f->d_idx_pool, f->idx_pool));
  RC(dupload(f, &f->d_scale_pool, f->scale_pool));
  std::vector<int> tsrcT(f->tsrc8.size());
  for (int t = 0; t < f->nT8; ++t)
    for (int d = 0; d < 26; ++d) tsrcT[(size_t)d * f->nT8 + t] = f->tsrc8[(size_t)t * 26 + d];
  RC(dupload(f, &f->d_tsrc8, tsrcT));
  f->m2l32 = mixed && o.P <= kM2L32MaxP;
  if (f->ops_dev_gen != f->ops_gen) {
    RC(upload_operators(f));
    f->ops_dev_gen = f->ops_gen;
  }
  {
    // M2L spectra of the sources and targets, FP32 or FP64
    const size_t e = f->m2l32 ? sizeof(float) : sizeof(double);
    char *qp = nullptr, *pp = nullptr;
    RC(dalloc(f, &qp, (size_t)f->nS8 * 8 * Nf * 2 * e, &f->d_Q8));
    RC(dalloc(f, &pp, (size_t)f->nT8 * 8 * Nf * 2 * e, &f->d_Pk8));
    f->d_Q8 = qp;
    f->d_Pk8 = pp;
  }
  RC(dalloc(f, &f->d_Q27, (size_t)f->nS27 * 8 * Nf * 2));
  RC(dalloc(f, &f->d_Pk27, (size_t)f->nT27 * 8 * Nf * 2));
  // M2L up/down blocks: groups of sp child slots (sized to shared memory)
  f->sp_up8 = f->m2l32 ? m2l_up_slots<float>(o.P) : m2l_up_slots<double>(o.P);
  f->sp_down8 = f->m2l32 ? m2l_down_slots<float>(o.P) : m2l_down_slots<double>(o.P);
  f->sp_up27 = m2l_up_slots<double>(o.P);
  f->sp_down27 = m2l_down_slots<double>(o.P);
  auto group = [](const std::vector<int>& slots, int sp, bool keep_empty, std::vector<int>& items) {
    items.clear();
    const size_t np = slots.size() / 8;
    for (size_t pidx = 0; pidx < np; ++pidx)
      for (int g0 = 0; g0 < 8; g0 += sp) {
        bool any = false;
        for (int j = 0; j < sp; ++j) any |= slots[pidx * 8 + g0 + j] >= 0;
        if (!any && !keep_empty) continue;
        items.push_back((int)pidx);
        items.push_back(g0);
        for (int j = 0; j < 8; ++j) items.push_back(j < sp ? slots[pidx * 8 + g0 + j] : -1);
      }
  };
  group(f->up8_slots, f->sp_up8, true, f->up8_items);
  group(f->down8_slots, f->sp_down8, false, f->down8_items);
  group(f->up27_slots, f->sp_up27, true, f->up27_items);
  group(f->down27_slots, f->sp_down27, false, f->down27_items);
  RC(dupload(f, &f->d_up8, f->up8_items));
  RC(dupload(f, &f->d_down8, f->down8_items));
  RC(dupload(f, &f->d_up27, f->up27_items));
  RC(dupload(f, &f->d_down27, f->down27_items));
  RC(dupload(f, &f->d_tsrc27, f->tsrc27));
  RC(dupload(f, &f->d_tscale8, f->tscale8));
  RC(dupload(f, &f->d_tscale27, f->tscale27));
  RC(dalloc(f, &f->d_dip, kDipoleScratch));
#undef RC
  if (f->h_xin_cap < (size_t)std::max<int64_t>(1, 3 * n)) {
    if (f->h_xin) cudaFreeHost(f->h_xin);
    f->h_xin = nullptr;
    f->h_xin_cap = 0;
    const size_t cap = (size_t)std::max<int64_t>(1, 3 * n + 3 * n / 4);
    CK(cudaMallocHost(&f->h_xin, sizeof(double) * cap));
    f->h_xin_cap = cap;
  }
  if (n > 0 && f->host_bodies) std::memcpy(f->h_xin, f->x_in.data(), sizeof(double) * 3 * n);
  f->device_ready = true;
  f->setup_s[5] = wall_s() - t0;
  return RTFMM_OK;
}

int run_apply(rtfmm_fmm* f, const ApplyCall& c, bool adjoint = false) {
  ApplyBatch b;
  double* bufs[BUF_NUM] = {f->d_qeq, f->d_pchk, f->d_leafvec, f->d_leafvec2, f->d_y};
  b.A = bufs[c.abuf];
  b.C = bufs[c.cbuf];
  b.inrow = f->d_idx_pool + c.inrow_off;
  b.outrow = f->d_idx_pool + c.outrow_off;
  b.group_off = f->d_idx_pool + c.goff_off;
  b.scale = c.has_scale ? f->d_scale_pool + c.scale_off : nullptr;
  int bsel = c.bsel;
  if (adjoint && bsel == B_IMGSUMT) bsel = B_ADJ_IMG_UP;
  if (adjoint && bsel == B_IMG13) bsel = B_ADJ_IMG_DOWN;
  b.B = f->d_B[bsel];
  b.groups = c.groups;
  b.S = c.S;
  b.ns = f->ops.ns;
  b.beta = c.beta;
  b.max_rows = c.rows_max;
  CK(launch_apply(b, f->s0));
  f->launches++;
  if (c.nsum > 0) {
    CK(launch_sum_children(f->d_idx_pool + c.sum_off, c.nsum, f->d_y, f->ops.ns, f->d_qeq, f->s0));
    f->launches++;
  }
  return RTFMM_OK;
}

// One evaluation pass on the device-resident bodies (d_body64).  With
// `adjoint` the pass applies the transposed operator chain to the body
// charges (which then hold the weights w): P2P, M2L and the tree-level
// M2M/L2L and P2M/L2P pairs are their own transposes on the symmetric lists,
// only the image-level operators swap; no dipole correction.
//
// phase 0 is the whole pass.  A sharded pass runs in two phases around the
// caller's exchange: phase 1 (upward) runs P2P and P2M for this rank's
// leaves and gathers every leaf's q_equiv row into xbuf (rows of other
// ranks' leaves zero); phase 2 (downward) takes xbuf summed over the ranks
// back into the leaf rows and runs M2M on the whole tree, then M2L, L2L and
// L2P for this rank's cells and the post-processing.
int enqueue_pass(rtfmm_fmm* f, bool adjoint = false, bool no_dipole = false, int phase = 0,
                 double* xbuf = nullptr) {
  const Plan& p = f->plan;
  const Operators& o = f->ops;
  const int n = (int)p.n, ns = o.ns, Nf = o.Nf, P = o.P;
  const int nleaf = (int)f->leaves_own.size();  // the leaves whose P2M / L2P run here
  const bool mixed = f->args.precision == RTFMM_FP32_MIXED;
  const unsigned stages = f->args.stages;
  const bool near = stages & RTFMM_STAGE_NEAR, far = stages & RTFMM_STAGE_FAR;
  const bool serial = stages & RTFMM_STAGE_SERIAL;
  cudaStream_t s0 = f->s0, s1 = serial ? f->s0 : f->s1;
  const bool up = phase != 2, down = phase != 1;
  f->launches = 0;
  if (phase == 1) {
    // the bodies of other ranks' leaves get no P2P or L2P here: zero outputs
    // (before ev_start, which the P2P stream waits for)
    CK(cudaMemsetAsync(f->d_near_phi, 0, sizeof(double) * n, s0));
    CK(cudaMemsetAsync(f->d_near_grad, 0, sizeof(double) * 3 * n, s0));
    CK(cudaMemsetAsync(f->d_far_phi, 0, sizeof(double) * n, s0));
    CK(cudaMemsetAsync(f->d_far_grad, 0, sizeof(double) * 3 * n, s0));
  }
  if (up) CK(cudaEventRecord(f->ev_start, s0));
  auto near_field = [&]() -> int {
    if (!serial) CK(cudaStreamWaitEvent(s1, f->ev_start, 0));
    if (mixed) {
      CK(launch_prep32(f->d_body64, f->d_body_leaf, f->d_leaves, f->d_body32, n, s1));
      f->launches++;
    }
    CK(cudaEventRecord(f->ev_near0, s1));
    if (mixed) {
      CK(launch_p2p32(f->d_body32, f->d_items2, f->n_items2, f->d_list_off, f->d_list32,
                      f->d_near_phi, f->d_near_grad, s1));
      f->launches += 1;
      if (f->n_close > 0) {
        CK(launch_close_fix(f->d_body64, f->d_body32, f->d_list32, f->d_close_off, f->d_close_pairs, n,
                            f->args.images > 0 ? f->args.cycle : 0.0, f->d_near_phi, f->d_near_grad, s1));
        f->launches += 1;
      }
    } else {
      CK(launch_p2p64(f->d_body64, f->d_items2, f->n_items2, f->d_list_off, f->d_list64,
                      f->d_near_phi, f->d_near_grad, s1));
      f->launches += 1;
    }
    CK(cudaEventRecord(f->ev_near, s1));
    return RTFMM_OK;
  };
  if (near && !serial && up) {
    int rc = near_field();
    if (rc) return rc;
  }
  if (up) CK(cudaEventRecord(f->ev_st[ST_PREP], s0));
  if (far && phase == 0) CK(cudaMemsetAsync(f->d_pchk, 0, sizeof(double) * p.cells.size() * ns, s0));
  if (far && up) {
    CK(launch_p2m_check(f->d_body64, f->d_leaves_own, nleaf, f->d_surf_unit, ns, f->d_leafvec, s0,
                        mixed ? 1 : 2));
    f->launches++;
    for (auto& c : f->p2m_call) {
      int rc = run_apply(f, c);
      if (rc) return rc;
    }
    CK(cudaEventRecord(f->ev_st[ST_P2M], s0));
  }
  if (phase == 1) {
    // every leaf's q_equiv row into the exchange buffer (others' rows zero)
    if (far) {
      CK(launch_leaf_rows(f->d_qeq, (int)p.cells.size(), f->d_leaf_cells, f->d_leaf_own, (int)f->leaves.size(), ns,
                            xbuf, false, s0));
      f->launches++;
    }
    return RTFMM_OK;
  }
  if (phase == 2 && far) {
    CK(launch_leaf_rows(f->d_qeq, (int)p.cells.size(), f->d_leaf_cells, nullptr, (int)f->leaves.size(), ns, xbuf,
                            true, s0));
    f->launches++;
  }
  if (far && down) {
    if (phase == 2) CK(cudaMemsetAsync(f->d_pchk, 0, sizeof(double) * p.cells.size() * ns, s0));
    for (auto& c : f->m2m_calls) {
      int rc = run_apply(f, c, adjoint);
      if (rc) return rc;
    }
    CK(cudaEventRecord(f->ev_st[ST_M2M], s0));
    const int nup8 = (int)f->up8_items.size() / 10, nup27 = (int)f->up27_items.size() / 10;
    const int ndn8 = (int)f->down8_items.size() / 10, ndn27 = (int)f->down27_items.size() / 10;
    if (f->m2l32) {
      CK(launch_m2l_up<float>(f->d_qeq, f->d_up8, nup8, f->d_surf_ijk, f->d_twiddle, P, ns, f->nS8, f->sp_up8,
                              (float*)f->d_Q8, s0));
    } else {
      CK(launch_m2l_up<double>(f->d_qeq, f->d_up8, nup8, f->d_surf_ijk, f->d_twiddle, P, ns, f->nS8, f->sp_up8,
                               (double*)f->d_Q8, s0));
    }
    CK(launch_m2l_up<double>(f->d_qeq, f->d_up27, nup27, f->d_surf_ijk, f->d_twiddle, P, ns, f->nS27,
                             f->sp_up27, f->d_Q27, s0));
    f->launches += (nup8 > 0) + (nup27 > 0);
    CK(cudaEventRecord(f->ev_st[ST_UP], s0));
    if (f->m2l32) {
      CK(launch_m2l_hadamard8<float>((const float*)f->d_Q8, (const float*)f->d_G8, f->d_tsrc8, f->nT8, f->nS8,
                                     Nf, (float*)f->d_Pk8, s0));
    } else {
      CK(launch_m2l_hadamard8<double>((const double*)f->d_Q8, (const double*)f->d_G8, f->d_tsrc8, f->nT8,
                                      f->nS8, Nf, (double*)f->d_Pk8, s0));
    }
    CK(launch_m2l_hadamard27(f->d_Q27, f->d_G27, f->d_tsrc27, f->nT27, f->nS27, Nf, f->d_Pk27, s0));
    f->launches += (f->nT8 > 0) + (f->nT27 > 0);
    CK(cudaEventRecord(f->ev_st[ST_HAD], s0));
    if (f->m2l32) {
      CK(launch_m2l_down<float>((const float*)f->d_Pk8, f->d_down8, f->d_tscale8, ndn8, f->d_surf_ijk,
                                f->d_twiddle, P, ns, f->nT8, f->sp_down8, f->d_pchk, s0));
    } else {
      CK(launch_m2l_down<double>((const double*)f->d_Pk8, f->d_down8, f->d_tscale8, ndn8, f->d_surf_ijk,
                                 f->d_twiddle, P, ns, f->nT8, f->sp_down8, f->d_pchk, s0));
    }
    CK(launch_m2l_down<double>(f->d_Pk27, f->d_down27, f->d_tscale27, ndn27, f->d_surf_ijk, f->d_twiddle, P, ns,
                               f->nT27, f->sp_down27, f->d_pchk, s0));
    f->launches += (ndn8 > 0) + (ndn27 > 0);
    CK(cudaEventRecord(f->ev_st[ST_DOWN], s0));
    for (auto& c : f->l2l_calls) {
      int rc = run_apply(f, c, adjoint);
      if (rc) return rc;
    }
    CK(cudaEventRecord(f->ev_st[ST_L2L], s0));
    for (auto& c : f->l2p_call) {
      int rc = run_apply(f, c);
      if (rc) return rc;
    }
    CK(launch_l2p_eval(f->d_body64, f->d_leaves_own, nleaf, f->d_surf_unit, ns, f->d_leafvec2, f->d_far_phi,
                       f->d_far_grad, s0, mixed ? 1 : 2));
    f->launches++;
    CK(cudaEventRecord(f->ev_st[ST_L2P], s0));
  } else {
    for (int k = ST_P2M; k <= ST_L2P; ++k) CK(cudaEventRecord(f->ev_st[k], s0));
  }
  if (near && serial) {
    int rc = near_field();
    if (rc) return rc;
  }
  if (near && !serial) CK(cudaStreamWaitEvent(s0, f->ev_near, 0));
  CK(cudaEventRecord(f->ev_st[ST_P2P], s0));
  const Args& a = f->args;
  const int dipole = (adjoint || no_dipole) ? 0 : a.dipole_correction;
  if (dipole) {
    CK(launch_dipole(f->d_body64, n, f->d_dip, s0));
    f->launches += 2;
  }
  const double coef = 4 * M_PI / (3 * a.cycle * a.cycle * a.cycle);
  CK(launch_post(far ? f->d_far_phi : nullptr, f->d_far_grad, near ? f->d_near_phi : nullptr, f->d_near_grad,
                 f->d_body64, f->d_perm, n, f->d_dip, coef, dipole, a.x.data(),
                 a.divide_4pi ? 1.0 / (4 * M_PI) : 1.0, f->d_out_phi, f->d_out_grad, s0));
  f->launches++;
  CK(cudaEventRecord(f->ev_st[ST_POST], s0));
  CK(cudaEventRecord(f->ev_stop, s0));
  f->grad_q_valid = !adjoint && dipole == 0 && near && far;
  return RTFMM_OK;
}

// The mixed form's close-pair list for the positions now in d_body64 (once
// per set of device positions, before a pass is enqueued or captured):
// FP32 positions, per-target counts, their prefix sum, then the pairs.
int ensure_close_pairs(rtfmm_fmm* f) {
  if (f->args.precision != RTFMM_FP32_MIXED || f->close_valid || !(f->args.stages & RTFMM_STAGE_NEAR))
    return RTFMM_OK;
  const int n = (int)f->plan.n;
  cudaStream_t s0 = f->s0;
  f->n_close = 0;
  if (n > 0 && f->n_items2 > 0) {
    int rc = 0;
    if ((rc = dalloc(f, &f->d_close_cnt, (size_t)n + 1)) || (rc = dalloc(f, &f->d_close_off, (size_t)n + 1)))
      return rc;
    CK(launch_prep32(f->d_body64, f->d_body_leaf, f->d_leaves, f->d_body32, n, s0));
    CK(cudaMemsetAsync(f->d_close_cnt, 0, sizeof(int) * ((size_t)n + 1), s0));
    CK(launch_close_count(f->d_body32, f->d_items2, f->n_items2, f->d_list_off, f->d_list32, f->d_leaves,
                          f->d_close_cnt, s0));
    size_t tmp_bytes = 0;
    CK(launch_count_scan(f->d_close_cnt, f->d_close_off, n + 1, nullptr, &tmp_bytes, s0));
    char* tmp = nullptr;
    if ((rc = dalloc(f, &tmp, tmp_bytes, &f->d_close_tmp))) return rc;
    f->d_close_tmp = tmp;
    CK(launch_count_scan(f->d_close_cnt, f->d_close_off, n + 1, tmp, &tmp_bytes, s0));
    int total = 0;
    CK(cudaMemcpyAsync(&total, f->d_close_off + n, sizeof(int), cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    if (total > 0) {
      if ((rc = dalloc(f, &f->d_close_pairs, (size_t)total))) return rc;
      CK(launch_close_emit(f->d_body32, f->d_items2, f->n_items2, f->d_list_off, f->d_list32, f->d_leaves,
                           f->d_close_off, f->d_close_pairs, s0));
      CK(cudaStreamSynchronize(s0));
    }
    f->n_close = total;
  }
  f->close_valid = true;
  return RTFMM_OK;
}

int collect_times(rtfmm_fmm* f, float* total) {
  CK(cudaEventSynchronize(f->ev_stop));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, f->ev_start, f->ev_stop));
  if (total) *total = ms;
  cudaEvent_t prev = f->ev_start;
  for (int k = 0; k < ST_N; ++k) {
    float t = 0;
    if (k == ST_P2P) {
      if (f->args.stages & RTFMM_STAGE_NEAR) CK(cudaEventElapsedTime(&t, f->ev_near0, f->ev_near));
      f->stage_ms[k] = t;
      prev = f->ev_st[k];
      continue;
    }
    CK(cudaEventElapsedTime(&t, prev, f->ev_st[k]));
    f->stage_ms[k] = t;
    prev = f->ev_st[k];
  }
  return RTFMM_OK;
}

// The forward pass as a CUDA graph: captured on first use per set of device
// tables (the launches, their arguments and the two-stream fork/join are
// fixed by the plan; charges, positions and outputs live in the handle's
// buffers), then replayed with one launch.  Kernel nodes keep the priority
// of the stream they were captured from, so the far-field chain still
// preempts P2P.  Per-stage events are not recorded in a replay: the stage
// timing and serial diagnostics (RTFMM_STAGE_TIMED, RTFMM_STAGE_SERIAL)
// issue the launches directly.
bool use_graph(const rtfmm_fmm* f) {
  return USE_PASS_GRAPH && !(f->args.stages & (RTFMM_STAGE_SERIAL | RTFMM_STAGE_TIMED));
}

// Enqueues one forward pass on s0 (graph replay or direct launches).
int launch_pass(rtfmm_fmm* f) {
  int rc0 = ensure_close_pairs(f);
  if (rc0) return rc0;
  if (!use_graph(f)) return enqueue_pass(f);
  if (!f->pass_graph) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(f->s0, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_pass(f);
    cudaError_t e = cudaStreamEndCapture(f->s0, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(RTFMM_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiateWithFlags(&f->pass_graph, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      f->pass_graph = nullptr;
      return fail(RTFMM_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    f->graph_grad_q_valid = f->grad_q_valid;
  }
  CK(cudaEventRecord(f->ev_g0, f->s0));
  CK(cudaGraphLaunch(f->pass_graph, f->s0));
  CK(cudaEventRecord(f->ev_g1, f->s0));
  f->grad_q_valid = f->graph_grad_q_valid;
  return RTFMM_OK;
}

// Waits for the pass launched by launch_pass; *total = its device time.
int pass_times(rtfmm_fmm* f, float* total) {
  if (!use_graph(f)) return collect_times(f, total);
  CK(cudaEventSynchronize(f->ev_g1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, f->ev_g0, f->ev_g1));
  if (total) *total = ms;
  for (int k = 0; k < ST_N; ++k) f->stage_ms[k] = 0;
  return RTFMM_OK;
}

}  // namespace

namespace rtfmm_b200 {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace rtfmm_b200

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

void rtfmm_b200_default_args(rtfmm_args* a) {
  if (!a) return;
  a->P = 4;
  a->ncrit = 16;
  a->images = 0;
  a->cycle = 2 * M_PI;
  a->x[0] = a->x[1] = a->x[2] = 0.0;
  a->dipole_correction = 1;
  a->divide_4pi = 0;
  a->precision = RTFMM_FP64;
  a->stages = RTFMM_STAGE_ALL;
  a->device = 0;
}

int rtfmm_b200_create(const rtfmm_args* a, rtfmm_fmm** out) {
  if (!a || !out) return fail(RTFMM_EINVAL, "null argument");
  *out = nullptr;
  if (a->P < 2 || a->P > 16) return fail(RTFMM_EINVAL, "P must be in [2, 16]");
  if (a->ncrit < 1) return fail(RTFMM_EINVAL, "ncrit must be >= 1");
  if (a->images < 0 || a->images > 20) return fail(RTFMM_EINVAL, "images must be in [0, 20]");
  if (!(a->cycle > 0) || !std::isfinite(a->cycle)) return fail(RTFMM_EINVAL, "cycle must be positive and finite");
  if (a->precision != RTFMM_FP64 && a->precision != RTFMM_FP32_MIXED)
    return fail(RTFMM_EINVAL, "unknown precision");
  if (a->dipole_correction < 0 || a->dipole_correction > 2) return fail(RTFMM_EINVAL, "dipole_correction must be 0, 1 or 2");
  if (a->stages & ~(RTFMM_STAGE_ALL | RTFMM_STAGE_SERIAL | RTFMM_STAGE_TIMED))
    return fail(RTFMM_EINVAL, "unknown stage bits");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(a->x[k])) return fail(RTFMM_EINVAL, "centre must be finite");
  rtfmm_fmm* f = new (std::nothrow) rtfmm_fmm();
  if (!f) return fail(RTFMM_ENOMEM, "host allocation failed");
  f->args.P = a->P;
  f->args.ncrit = a->ncrit;
  f->args.images = a->images;
  f->args.cycle = a->cycle;
  f->args.x = {a->x[0], a->x[1], a->x[2]};
  f->args.dipole_correction = a->dipole_correction;
  f->args.divide_4pi = a->divide_4pi;
  f->args.precision = a->precision;
  f->args.stages = (a->stages & RTFMM_STAGE_ALL) ? a->stages : (a->stages | RTFMM_STAGE_ALL);
  f->args.device = a->device;
  *out = f;
  return RTFMM_OK;
}

int rtfmm_b200_destroy(rtfmm_fmm* f) {
  if (!f) return RTFMM_OK;
  free_device(f);
  delete f;
  return RTFMM_OK;
}

}  // extern "C"

namespace {

// After a device set-up: the input-order bodies and the permutation from
// the device into x_in, q_in, plan.perm, plus (with tree_order) plan.x,
// plan.q and the pinned staging copy.  Called before anything overwrites
// d_xin or d_qin.
int ensure_host_bodies(rtfmm_fmm* f, bool tree_order = true) {
  if (f->host_bodies) return RTFMM_OK;
  Plan& p = f->plan;
  const int64_t n = p.n;
  f->x_in.resize(3 * n);
  f->q_in.resize(n);
  if (n > 0) {
    CK(cudaSetDevice(f->dev));
    CK(cudaMemcpyAsync(f->x_in.data(), f->d_xin, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, f->s0));
    CK(cudaMemcpyAsync(f->q_in.data(), f->d_qin, sizeof(double) * n, cudaMemcpyDeviceToHost, f->s0));
    if (tree_order) {
      p.perm.resize(n);
      CK(cudaMemcpyAsync(p.perm.data(), f->d_perm, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, f->s0));
    }
    CK(cudaStreamSynchronize(f->s0));
  }
  if (!tree_order) return RTFMM_OK;
  p.x.resize(3 * n);
  p.q.resize(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t k = p.perm[i];
    p.x[3 * i + 0] = f->x_in[3 * k + 0];
    p.x[3 * i + 1] = f->x_in[3 * k + 1];
    p.x[3 * i + 2] = f->x_in[3 * k + 2];
    p.q[i] = f->q_in[k];
  }
  if (f->h_xin && f->h_xin_cap >= (size_t)(3 * n) && n > 0)
    std::memcpy(f->h_xin, f->x_in.data(), sizeof(double) * 3 * n);
  f->host_bodies = true;
  return RTFMM_OK;
}

// Operator tables by (P, images, root radius), shared by the handles of the
// process: they depend on nothing else, so a handle whose tables are already
// here copies them instead of building them (0.2 s at P = 8, 0.4-0.6 s at
// P = 10).  The most recent kOpsCacheMax sets are kept.
constexpr size_t kOpsCacheMax = 4;
std::mutex g_ops_mu;
std::vector<std::shared_ptr<const Operators>> g_ops_cache;

std::shared_ptr<const Operators> ops_lookup(int P, int images, double r0) {
  std::lock_guard<std::mutex> lock(g_ops_mu);
  for (const auto& o : g_ops_cache)
    if (o->P == P && o->images == images && o->r0 == r0) return o;
  return nullptr;
}

void ops_store(const Operators& o) {
  auto c = std::make_shared<const Operators>(o);
  std::lock_guard<std::mutex> lock(g_ops_mu);
  g_ops_cache.push_back(std::move(c));
  if (g_ops_cache.size() > kOpsCacheMax) g_ops_cache.erase(g_ops_cache.begin());
}

// Scratch slots: the device tree 0..15, the walk 16..47, the P2P tables
// 48..63.
constexpr int kWalkSlots = 16;
constexpr int kTableSlots = 48;

// Lists (the P2P walk on the GPU with `gpu` scratch), operators (unless
// cached for this P, images and radius) and host tables of the plan whose
// tree is built; st[1..3] get their wall times.
void finish_setup(rtfmm_fmm* f, const TreeScratchFn* gpu = nullptr) {
  double* st = f->setup_s;
  double t = wall_s();
  bool device_tables = false;
  if (gpu) {
    // the P2P walk on the GPU (the host walk when it is too deep for it)
    const std::vector<WalkRoot> roots = traverse_begin(f->plan);
    std::string msg;
    f->dwalk = DeviceWalk();
    // the lists stay on the device when the GPU builds the P2P tables from
    // them (the host copy is fetched only on request, rtfmm_b200_get_p2p)
    const int rc = device_p2p_walk(f->plan, roots, f->s0, *gpu, kWalkSlots, &f->dwalk, msg, false);
    if (rc == kTreeError) throw std::runtime_error(msg);
    if (rc == kTreeTooDeep) {
      f->plan.p2p.clear();
      traverse_p2p(f->plan, roots);
    }
    device_tables = rc == kTreeOk && f->plan.n > 0 && f->dwalk.npairs > 0;
    if (rc == kTreeOk && !device_tables && device_walk_host_lists(f->dwalk, f->plan, f->s0, msg) != kTreeOk)
      throw std::runtime_error(msg);
    f->p2p_lists_on_device = device_tables;
    traverse_finish(f->plan);
    if (device_tables) f->plan.n_p2p = f->dwalk.npairs;
  } else {
    f->p2p_lists_on_device = false;
    traverse(f->plan);
  }
  st[1] = wall_s() - t;
  if (!f->ops_valid || f->ops.P != f->args.P || f->ops.images != f->args.images || f->ops.r0 != f->plan.r0) {
    t = wall_s();
    if (std::shared_ptr<const Operators> c = ops_lookup(f->args.P, f->args.images, f->plan.r0)) {
      f->ops = *c;
    } else {
      // with a device set-up, the SVD sweeps, the M2M products and the kernel
      // spectra run on the GPU (the same tables, bit for bit)
      const DenseBackend be = gpu_dense_backend(f->s0);
      build_operators(f->ops, f->args.P, f->plan.r0, f->args.images, gpu ? &be : nullptr);
      for (int k = 0; k < 6; ++k) st[6 + k] = f->ops.build_s[k];
      ops_store(f->ops);
    }
    f->ops_valid = true;
    f->ops_gen++;
    st[2] = wall_s() - t;
  }
  t = wall_s();
  build_tables(f, !device_tables);
  st[3] = wall_s() - t;
}

// The P2P lists, offsets and work items on the GPU from the walk's pairs,
// into the handle's device buffers (after upload_plan).
int device_tables(rtfmm_fmm* f, const TreeScratchFn& scratch) {
  const int nlf = (int)f->leaves.size();
  const int slots[3] = {kTableSlots + 8, kTableSlots + 9, kTableSlots + 10};
  const std::vector<int>* src[3] = {&f->h_parent, &f->h_dfs, &f->h_dfs_pos};
  int* dev[3];
  for (int k = 0; k < 3; ++k) {
    dev[k] = (int*)scratch(slots[k], sizeof(int) * std::max<size_t>(1, src[k]->size()));
    if (!dev[k]) return fail(RTFMM_ENOMEM, "device allocation failed");
    if (!src[k]->empty())
      CK(cudaMemcpyAsync(dev[k], src[k]->data(), sizeof(int) * src[k]->size(), cudaMemcpyHostToDevice, f->s0));
  }
  DeviceLeafInput in{f->d_leaves, nlf, dev[0], f->d_body_leaf, dev[1], dev[2]};
  P2PTableAlloc alloc;
  alloc.list_off = [f](int n) { return dalloc(f, &f->d_list_off, n) ? nullptr : f->d_list_off; };
  alloc.list32 = [f](int n) { return dalloc(f, &f->d_list32, n) ? nullptr : f->d_list32; };
  alloc.list64 = [f](int n) { return dalloc(f, &f->d_list64, n) ? nullptr : f->d_list64; };
  alloc.items = [f](int n) { return dalloc(f, &f->d_items2, n) ? nullptr : f->d_items2; };
  P2PTablesOut out;
  std::string msg;
  const bool mixed = f->args.precision == RTFMM_FP32_MIXED;
  if (device_p2p_tables(f->dwalk, in, mixed, f->s0, scratch, kTableSlots, alloc, &out, msg) != kTreeOk)
    return fail(RTFMM_ECUDA, msg);
  f->n_items2 = out.nitems;
  f->p2p_pairs = out.pairs;
  return RTFMM_OK;
}

void begin_setup(rtfmm_fmm* f, int64_t n) {
  f->setup_done = false;
  f->pass_done = false;
  f->plan = Plan();
  f->plan.args = f->args;
  f->plan.n = n;
  for (int k = 0; k < 12; ++k) f->setup_s[k] = 0;
}

void end_setup(rtfmm_fmm* f, double t0) {
  f->setup_s[4] = wall_s() - t0;
  f->setup_done = true;
  f->device_ready = false;
  f->grad_q_valid = false;
  f->pos_on_device = false;
}

}  // namespace

extern "C" {

int rtfmm_b200_setup(rtfmm_fmm* f, int64_t n, const double* x, const double* q) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (n < 0 || n > (int64_t)1 << 30) return fail(RTFMM_EINVAL, "n out of range");
  if (n > 0 && (!x || !q)) return fail(RTFMM_EINVAL, "null body arrays");
  const double t0 = wall_s();
  if (!finite_all(x, 3 * n) || !finite_all(q, n)) return fail(RTFMM_EINVAL, "non-finite body position or charge");
  try {
    begin_setup(f, n);
    f->host_bodies = true;
    f->x_in.assign(x, x + 3 * n);
    f->q_in.assign(q, q + n);
    double t = wall_s();
    std::string err = build_tree(f->plan, x, q);
    if (!err.empty()) return fail(RTFMM_EINVAL, err);
    f->setup_s[0] = wall_s() - t;
    finish_setup(f);
  } catch (const std::bad_alloc&) {
    return fail(RTFMM_ENOMEM, "host allocation failed during set-up");
  } catch (const std::exception& e) {
    return fail(RTFMM_EINVAL, std::string("set-up failed: ") + e.what());
  }
  end_setup(f, t0);
  return RTFMM_OK;
}

int rtfmm_b200_setup_device(rtfmm_fmm* f, int64_t n, const double* x_dev, const double* q_dev) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (f->shard_n > 1) return fail(RTFMM_ENOTSUP, "sharded handles are set up from host bodies (rtfmm_b200_setup)");
  if (n < 0 || n > (int64_t)1 << 30) return fail(RTFMM_EINVAL, "n out of range");
  if (n > 0 && (!x_dev || !q_dev)) return fail(RTFMM_EINVAL, "null body arrays");
  const double t0 = wall_s();
  int rc = ensure_device(f);
  if (rc) return rc;
  // nothing of a previous plan may still read the buffers reused below
  CK(cudaDeviceSynchronize());
  const TreeScratchFn scratch = [f](int slot, size_t bytes) -> void* {
    if (slot < 0 || slot >= (int)sizeof(f->tree_slots)) return nullptr;
    char* q = nullptr;
    return dalloc(f, &q, bytes, &f->tree_slots[slot]) ? nullptr : (void*)q;
  };
  try {
    begin_setup(f, n);
    double t = wall_s();
    // the bodies in input order (d_xin, d_qin) and the permutation (d_perm)
    // stay on the device; the host copies follow on first use
    double *dx = nullptr, *dq = nullptr;
    int64_t* dp = nullptr;
    if ((rc = dalloc(f, &dx, 3 * n, &f->d_xin)) || (rc = dalloc(f, &dq, n, &f->d_qin)) ||
        (rc = dalloc(f, &dp, n, &f->d_perm)))
      return rc;
    f->d_xin = dx;
    f->d_qin = dq;
    f->d_perm = dp;
    std::string msg;
    const int tr = device_build_tree(x_dev, q_dev, n, f->s0, f->plan, dp, scratch, msg);
    if (tr == kTreeError) {
      f->plan = Plan();
      const bool bad = msg == "non-finite body position or charge";
      return fail(bad ? RTFMM_EINVAL : RTFMM_ECUDA, msg);
    }
    if (n > 0) {
      CK(cudaMemcpyAsync(dx, x_dev, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, f->s0));
      CK(cudaMemcpyAsync(dq, q_dev, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->s0));
    }
    f->host_bodies = false;
    if (tr == kTreeTooDeep) {
      rc = ensure_host_bodies(f, false);
      if (rc) return rc;
      std::string err = build_tree(f->plan, f->x_in.data(), f->q_in.data());
      if (!err.empty()) return fail(RTFMM_EINVAL, err);
      f->host_bodies = true;
    }
    f->setup_s[0] = wall_s() - t;
    finish_setup(f, &scratch);
  } catch (const std::bad_alloc&) {
    return fail(RTFMM_ENOMEM, "host allocation failed during set-up");
  } catch (const std::exception& e) {
    return fail(RTFMM_EINVAL, std::string("set-up failed: ") + e.what());
  }
  end_setup(f, t0);
  // device tables (the P2P ones built on the GPU), then the bodies gathered
  // into tree order on the device
  rc = upload_plan(f);
  if (rc) return rc;
  if (f->p2p_on_device) {
    const double t = wall_s();
    rc = device_tables(f, scratch);
    if (rc) return rc;
    f->setup_s[3] += wall_s() - t;
  }
  if (n > 0) {
    CK(launch_gather_bodies(f->d_xin, f->d_qin, f->d_perm, (int)n, f->d_body64, f->s0));
    CK(cudaStreamSynchronize(f->s0));
  }
  f->pos_on_device = true;
  f->setup_s[4] = wall_s() - t0;
  return RTFMM_OK;
}

int rtfmm_b200_upload(rtfmm_fmm* f) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  if (!f->device_ready) {
    int rc = upload_plan(f);
    if (rc) return rc;
  }
  CK(cudaSetDevice(f->dev));
  int rc = ensure_host_bodies(f);
  if (rc) return rc;
  const int64_t n = f->plan.n;
  if (n > 0) {
    // input order up (positions from the pinned copy), tree order on the device
    CK(cudaMemcpyAsync(f->d_xin, f->h_xin, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, f->s0));
    CK(cudaMemcpyAsync(f->d_qin, f->q_in.data(), sizeof(double) * n, cudaMemcpyHostToDevice, f->s0));
    CK(launch_gather_bodies(f->d_xin, f->d_qin, f->d_perm, (int)n, f->d_body64, f->s0));
    CK(cudaStreamSynchronize(f->s0));
  }
  f->grad_q_valid = false;
  f->pos_on_device = true;
  return RTFMM_OK;
}

int rtfmm_b200_evaluate_device(rtfmm_fmm* f, float* ms) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (f->shard_n > 1) return fail(RTFMM_ESTATE, "sharded handle: run the pass with rtfmm_b200_shard_upward/_downward");
  if (!f->setup_done || !f->device_ready) return fail(RTFMM_ESTATE, "upload has not run");
  CK(cudaSetDevice(f->dev));
  if (f->plan.n == 0) {
    if (ms) *ms = 0;
    return RTFMM_OK;
  }
  int rc = launch_pass(f);
  if (rc) return rc;
  float t = 0;
  rc = pass_times(f, &t);
  if (rc) return rc;
  CK(cudaGetLastError());
  if (ms) *ms = t;
  f->pass_done = true;
  return RTFMM_OK;
}

int rtfmm_b200_forward_device(rtfmm_fmm* f, const double* q_dev, double* phi_dev, double* grad_dev, float* ms) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (f->shard_n > 1) return fail(RTFMM_ESTATE, "sharded handle: run the pass with rtfmm_b200_shard_upward/_downward");
  if (!f->setup_done || !f->device_ready || !f->pos_on_device)
    return fail(RTFMM_ESTATE, "upload (or an evaluate) has not run");
  if (ms) *ms = 0;
  const int64_t n = f->plan.n;
  if (n == 0) return RTFMM_OK;
  CK(cudaSetDevice(f->dev));
  if (q_dev) CK(launch_set_charges(f->d_body64, q_dev, f->d_perm, (int)n, f->s0));
  int rc = launch_pass(f);
  if (rc) return rc;
  if (phi_dev) CK(cudaMemcpyAsync(phi_dev, f->d_out_phi, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->s0));
  if (grad_dev)
    CK(cudaMemcpyAsync(grad_dev, f->d_out_grad, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, f->s0));
  float t = 0;
  rc = pass_times(f, &t);
  if (rc) return rc;
  CK(cudaStreamSynchronize(f->s0));
  CK(cudaGetLastError());
  if (ms) *ms = t;
  f->pass_done = true;
  return RTFMM_OK;
}

int rtfmm_b200_download(rtfmm_fmm* f, double* phi, double* grad) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (!f->pass_done) return fail(RTFMM_ESTATE, "no pass has run");
  if (f->plan.n == 0) return RTFMM_OK;
  CK(cudaSetDevice(f->dev));
  if (phi) CK(cudaMemcpyAsync(phi, f->d_out_phi, sizeof(double) * f->plan.n, cudaMemcpyDeviceToHost, f->s0));
  if (grad) CK(cudaMemcpyAsync(grad, f->d_out_grad, sizeof(double) * 3 * f->plan.n, cudaMemcpyDeviceToHost, f->s0));
  CK(cudaStreamSynchronize(f->s0));
  return RTFMM_OK;
}

int rtfmm_b200_evaluate(rtfmm_fmm* f, const double* q, double* phi, double* grad) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (f->shard_n > 1) return fail(RTFMM_ESTATE, "sharded handle: run the pass with rtfmm_b200_shard_upward/_downward");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  const int64_t n = f->plan.n;
  if (n == 0) return RTFMM_OK;
  if (!f->device_ready) {
    int rc = upload_plan(f);
    if (rc) return rc;
  }
  CK(cudaSetDevice(f->dev));
  // New charges for positions already on the device go through a staging
  // buffer, so d_qin keeps the set-up charges (which a later host-buffer
  // call may fetch); otherwise the set-up charges or the first move of the
  // positions need the host copies of the set-up bodies (fetched here after
  // a device set-up, before d_qin is overwritten).
  const bool staged = q && f->pos_on_device;
  if (!staged) {
    int rc0 = ensure_host_bodies(f);
    if (rc0) return rc0;
  } else {
    int rc0 = dalloc(f, &f->d_stage_q, (size_t)n);
    if (rc0) return rc0;
  }
  // host -> device (input order), then into tree order on the device; the
  // positions move only on the first call after set-up.  The charges are
  // checked on the host while they are copied; nothing reads them before the
  // check passes.
  double* qdst = staged ? f->d_stage_q : f->d_qin;
  CK(cudaMemcpyAsync(qdst, q ? q : f->q_in.data(), sizeof(double) * n, cudaMemcpyHostToDevice, f->s0));
  if (q && !finite_all(q, n)) {
    CK(cudaStreamSynchronize(f->s0));
    return fail(RTFMM_EINVAL, "non-finite charge");
  }
  if (f->pos_on_device) {
    CK(launch_set_charges(f->d_body64, qdst, f->d_perm, (int)n, f->s0));
  } else {
    CK(cudaMemcpyAsync(f->d_xin, f->h_xin, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, f->s0));
    CK(launch_gather_bodies(f->d_xin, f->d_qin, f->d_perm, (int)n, f->d_body64, f->s0));
    f->pos_on_device = true;
  }
  int rc = launch_pass(f);
  if (rc) return rc;
  f->launches++;
  if (phi) CK(cudaMemcpyAsync(phi, f->d_out_phi, sizeof(double) * n, cudaMemcpyDeviceToHost, f->s0));
  if (grad) CK(cudaMemcpyAsync(grad, f->d_out_grad, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, f->s0));
  CK(cudaStreamSynchronize(f->s0));
  CK(cudaGetLastError());
  rc = pass_times(f, nullptr);
  if (rc) return rc;
  f->pass_done = true;
  return RTFMM_OK;
}

// Bodies from which rtfmm_b200_solve builds the tree, lists and P2P tables on
// the GPU (rtfmm_b200_setup_device, the same plan bit for bit); below it the
// host set-up is quicker than the copies and launches.
constexpr int64_t kSolveDeviceSetupMin = 1 << 16;

int rtfmm_b200_solve(rtfmm_fmm* f, int64_t n, const double* x, const double* q, double* phi, double* grad) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (n >= kSolveDeviceSetupMin && f->shard_n == 1 && x && q) {
    int rc = ensure_device(f);
    if (rc) return rc;
    // the input bodies through pooled staging buffers to the device set-up
    if ((rc = dalloc(f, &f->d_stage_x, 3 * (size_t)n)) || (rc = dalloc(f, &f->d_stage_q, (size_t)n))) return rc;
    CK(cudaMemcpyAsync(f->d_stage_x, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, f->s0));
    CK(cudaMemcpyAsync(f->d_stage_q, q, sizeof(double) * n, cudaMemcpyHostToDevice, f->s0));
    CK(cudaStreamSynchronize(f->s0));
    rc = rtfmm_b200_setup_device(f, n, f->d_stage_x, f->d_stage_q);
    if (rc) return rc;
  } else {
    int rc = rtfmm_b200_setup(f, n, x, q);
    if (rc) return rc;
  }
  return rtfmm_b200_evaluate(f, q, phi, grad);
}

namespace {

int ensure_adj_scratch(rtfmm_fmm* f) {
  if (f->d_adj_q) return RTFMM_OK;
  const int64_t n = f->plan.n;
  int rc = 0;
  if ((rc = dalloc(f, &f->d_adj_q, n)) || (rc = dalloc(f, &f->d_adj_gq, 3 * n)) ||
      (rc = dalloc(f, &f->d_adj_gw, 3 * n)) || (rc = dalloc(f, &f->d_adj_w, n)) ||
      (rc = dalloc(f, &f->d_adj_dq, n)) || (rc = dalloc(f, &f->d_adj_dx, 3 * n)))
    return rc;
  return RTFMM_OK;
}

// The adjoint on device-resident data, all on s0: for L = sum_k w_k phi_k,
//   dL/dq = K^T w                    (the transposed pass on the weights)
//   dL/dx = w grad(phi_q) + q grad(psi_w)
// where psi_w is the field of the weights.  grad(phi_q) is taken from the
// last forward pass when it is still valid (same charges, no dipole
// correction), else recomputed.  w, dq, dx are in input order; the bodies
// keep their charges.
int adjoint_core(rtfmm_fmm* f, const double* w, double* dq, double* dx) {
  const int n = (int)f->plan.n;
  int rc = ensure_adj_scratch(f);
  if (rc) return rc;
  rc = ensure_close_pairs(f);
  if (rc) return rc;
  cudaStream_t s0 = f->s0;
  const bool have_gq = f->grad_q_valid;
  if (have_gq) CK(cudaMemcpyAsync(f->d_adj_gq, f->d_out_grad, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s0));
  CK(launch_swap_charges(f->d_body64, w, f->d_perm, n, f->d_adj_q, s0));
  rc = enqueue_pass(f, true);
  if (rc) return rc;
  if (dq) CK(cudaMemcpyAsync(dq, f->d_out_phi, sizeof(double) * n, cudaMemcpyDeviceToDevice, s0));
  CK(launch_restore_charges(f->d_body64, f->d_adj_q, n, s0));
  const double* gq = f->d_adj_gq;
  const double* gw = f->d_out_grad;
  if (!have_gq) {
    CK(cudaMemcpyAsync(f->d_adj_gw, f->d_out_grad, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s0));
    rc = enqueue_pass(f, false, true);
    if (rc) return rc;
    gq = f->d_out_grad;
    gw = f->d_adj_gw;
  }
  if (dx) CK(launch_adj_combine(f->d_perm, w, f->d_adj_q, gq, gw, n, dx, s0));
  return RTFMM_OK;
}

}  // namespace

int rtfmm_b200_adjoint(rtfmm_fmm* f, const double* w, double* dLdq, double* dLdx) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (f->shard_n > 1) return fail(RTFMM_ESTATE, "sharded handle: run the pass with rtfmm_b200_shard_upward/_downward");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  const int64_t n = f->plan.n;
  if (n == 0) return RTFMM_OK;
  if (!w) return fail(RTFMM_EINVAL, "null weights");
  if (!finite_all(w, n)) return fail(RTFMM_EINVAL, "non-finite weight");
  if (!f->device_ready) {
    int rc = upload_plan(f);
    if (rc) return rc;
  }
  CK(cudaSetDevice(f->dev));
  int rc = ensure_adj_scratch(f);
  if (rc) return rc;
  rc = ensure_host_bodies(f);
  if (rc) return rc;
  // the bodies with the set-up charges, as the forward solve had them
  CK(cudaMemcpyAsync(f->d_xin, f->h_xin, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, f->s0));
  CK(cudaMemcpyAsync(f->d_qin, f->q_in.data(), sizeof(double) * n, cudaMemcpyHostToDevice, f->s0));
  CK(launch_gather_bodies(f->d_xin, f->d_qin, f->d_perm, (int)n, f->d_body64, f->s0));
  f->grad_q_valid = false;
  f->pos_on_device = true;
  CK(cudaMemcpyAsync(f->d_adj_w, w, sizeof(double) * n, cudaMemcpyHostToDevice, f->s0));
  rc = adjoint_core(f, f->d_adj_w, f->d_adj_dq, f->d_adj_dx);
  if (rc) return rc;
  if (dLdq) CK(cudaMemcpyAsync(dLdq, f->d_adj_dq, sizeof(double) * n, cudaMemcpyDeviceToHost, f->s0));
  if (dLdx) CK(cudaMemcpyAsync(dLdx, f->d_adj_dx, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, f->s0));
  CK(cudaStreamSynchronize(f->s0));
  CK(cudaGetLastError());
  f->pass_done = true;
  return RTFMM_OK;
}

int rtfmm_b200_adjoint_device(rtfmm_fmm* f, const double* w_dev, double* dLdq_dev, double* dLdx_dev, float* ms) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (f->shard_n > 1) return fail(RTFMM_ESTATE, "sharded handle: run the pass with rtfmm_b200_shard_upward/_downward");
  if (!f->setup_done || !f->device_ready) return fail(RTFMM_ESTATE, "upload has not run");
  if (ms) *ms = 0;
  if (f->plan.n == 0) return RTFMM_OK;
  if (!w_dev) return fail(RTFMM_EINVAL, "null weights");
  CK(cudaSetDevice(f->dev));
  CK(cudaEventRecord(f->ev_adj0, f->s0));
  int rc = adjoint_core(f, w_dev, dLdq_dev, dLdx_dev);
  if (rc) return rc;
  CK(cudaEventRecord(f->ev_adj1, f->s0));
  CK(cudaEventSynchronize(f->ev_adj1));
  CK(cudaGetLastError());
  float t = 0;
  CK(cudaEventElapsedTime(&t, f->ev_adj0, f->ev_adj1));
  if (ms) *ms = t;
  f->pass_done = true;
  return RTFMM_OK;
}

int rtfmm_b200_shard(rtfmm_fmm* f, int rank, int nranks) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (nranks < 1 || rank < 0 || rank >= nranks) return fail(RTFMM_EINVAL, "shard: need 0 <= rank < nranks");
  f->shard_rank = rank;
  f->shard_n = nranks;
  // the ownership is part of the plan: set up again
  f->setup_done = false;
  f->device_ready = false;
  drop_graph(f);
  return RTFMM_OK;
}

int rtfmm_b200_shard_sizes(rtfmm_fmm* f, int64_t* nbodies, int64_t* xbuf_doubles) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  int64_t nb = 0;
  for (const LeafInfo& L : f->leaves_own) nb += L.bnum;
  if (nbodies) *nbodies = nb;
  if (xbuf_doubles) *xbuf_doubles = (int64_t)f->leaves.size() * f->ops.ns;
  return RTFMM_OK;
}

int rtfmm_b200_shard_bodies(rtfmm_fmm* f, int64_t* idx, int64_t cap) {
  if (!f || !idx) return fail(RTFMM_EINVAL, "null argument");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  int rc = ensure_host_bodies(f);
  if (rc) return rc;
  std::vector<int64_t> v;
  for (const LeafInfo& L : f->leaves_own)
    for (int b = 0; b < L.bnum; ++b) v.push_back(f->plan.perm[L.boff + b]);
  std::sort(v.begin(), v.end());
  if ((int64_t)v.size() > cap) return fail(RTFMM_EINVAL, "shard_bodies: cap too small");
  std::copy(v.begin(), v.end(), idx);
  return RTFMM_OK;
}

int rtfmm_b200_shard_upward(rtfmm_fmm* f, double* xbuf_dev) {
  if (!f || !xbuf_dev) return fail(RTFMM_EINVAL, "null argument");
  if (!f->setup_done || !f->device_ready || !f->pos_on_device)
    return fail(RTFMM_ESTATE, "upload (or an evaluate) has not run");
  if (f->plan.n == 0) return RTFMM_OK;
  CK(cudaSetDevice(f->dev));
  int rc = ensure_close_pairs(f);
  if (rc) return rc;
  rc = enqueue_pass(f, false, false, 1, xbuf_dev);
  if (rc) return rc;
  CK(cudaStreamSynchronize(f->s0));  // the buffer is complete; P2P may still run
  CK(cudaGetLastError());
  f->shard_up = true;
  return RTFMM_OK;
}

int rtfmm_b200_shard_downward(rtfmm_fmm* f, const double* xbuf_dev, double* phi_dev, double* grad_dev, float* ms) {
  if (!f || !xbuf_dev) return fail(RTFMM_EINVAL, "null argument");
  if (!f->shard_up) return fail(RTFMM_ESTATE, "shard_upward has not run");
  if (ms) *ms = 0;
  const int64_t n = f->plan.n;
  if (n == 0) return RTFMM_OK;
  CK(cudaSetDevice(f->dev));
  CK(cudaEventRecord(f->ev_g0, f->s0));
  int rc = enqueue_pass(f, false, false, 2, const_cast<double*>(xbuf_dev));
  if (rc) return rc;
  if (phi_dev) CK(cudaMemcpyAsync(phi_dev, f->d_out_phi, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->s0));
  if (grad_dev)
    CK(cudaMemcpyAsync(grad_dev, f->d_out_grad, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, f->s0));
  CK(cudaEventRecord(f->ev_g1, f->s0));
  CK(cudaEventSynchronize(f->ev_g1));
  CK(cudaGetLastError());
  float t = 0;
  CK(cudaEventElapsedTime(&t, f->ev_g0, f->ev_g1));
  if (ms) *ms = t;
  f->shard_up = false;
  f->grad_q_valid = false;
  f->pass_done = true;
  return RTFMM_OK;
}

int rtfmm_b200_stage_times(rtfmm_fmm* f, double* ms, int cap) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  for (int k = 0; k < ST_N && k < cap; ++k) ms[k] = f->stage_ms[k];
  return ST_N;
}

int rtfmm_b200_launch_count(rtfmm_fmm* f, int64_t* launches) {
  if (!f || !launches) return fail(RTFMM_EINVAL, "null argument");
  *launches = f->launches;
  return RTFMM_OK;
}

int rtfmm_b200_flush_l2(rtfmm_fmm* f) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (!f->s0) return fail(RTFMM_ESTATE, "no device state");
  CK(cudaSetDevice(f->dev));
  if (!f->d_flush) {
    char* fl = nullptr;
    int rc = dalloc(f, &fl, (size_t)256 << 20, &f->d_flush);
    if (rc) return rc;
    f->d_flush = fl;
    f->flush_bytes = (size_t)256 << 20;
  }
  CK(cudaMemsetAsync(f->d_flush, f->launches & 0xff, f->flush_bytes, f->s0));
  CK(cudaStreamSynchronize(f->s0));
  return RTFMM_OK;
}

int rtfmm_b200_setup_times(rtfmm_fmm* f, double* s, int cap) {
  if (!f || !s) return fail(RTFMM_EINVAL, "null argument");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  for (int k = 0; k < 12 && k < cap; ++k) s[k] = f->setup_s[k];
  return RTFMM_OK;
}

int rtfmm_b200_info(rtfmm_fmm* f, int64_t* info, int cap) {
  if (!f || !info) return fail(RTFMM_EINVAL, "null argument");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  const int64_t pairs = f->p2p_pairs;
  int64_t td = 0;
  for (int v8 : f->tsrc8) td += v8 >= 0;
  int64_t v[13] = {(int64_t)f->plan.cells.size(), (int64_t)f->leaves.size(), f->plan.dmin, f->plan.dmax,
                   f->plan.n_p2p, (int64_t)f->plan.m2l.size(), f->plan.n_m2l, f->ops.ns, pairs, td, f->nS8, f->nT8,
                   f->close_valid ? f->n_close : 0};
  for (int k = 0; k < 13 && k < cap; ++k) info[k] = v[k];
  return 13;
}

int rtfmm_b200_get_cells(rtfmm_fmm* f, int32_t* ints, double* reals) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  for (size_t c = 0; c < f->plan.cells.size(); ++c) {
    const Cell& cl = f->plan.cells[c];
    if (ints) {
      int32_t* o = ints + 7 * c;
      o[0] = cl.octant;
      o[1] = cl.depth;
      o[2] = cl.coff;
      o[3] = cl.cnum;
      o[4] = cl.boff;
      o[5] = cl.bnum;
      o[6] = 0;
    }
    if (reals) {
      double* o = reals + 4 * c;
      o[0] = cl.r;
      o[1] = cl.x[0];
      o[2] = cl.x[1];
      o[3] = cl.x[2];
    }
  }
  return RTFMM_OK;
}

int rtfmm_b200_get_perm(rtfmm_fmm* f, int64_t* perm) {
  if (!f || !perm) return fail(RTFMM_EINVAL, "null argument");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  int rc = ensure_host_bodies(f);
  if (rc) return rc;
  std::memcpy(perm, f->plan.perm.data(), sizeof(int64_t) * f->plan.perm.size());
  return RTFMM_OK;
}

int rtfmm_b200_get_p2p(rtfmm_fmm* f, int32_t* ints, double* off) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  if (f->p2p_lists_on_device) {
    std::string msg;
    if (device_walk_host_lists(f->dwalk, f->plan, f->s0, msg) != kTreeOk) return fail(RTFMM_ECUDA, msg);
    f->p2p_lists_on_device = false;
  }
  size_t e = 0;
  for (const auto& kv : f->plan.p2p)
    for (const P2PEntry& s : kv.second) {
      if (ints) {
        ints[2 * e] = kv.first;
        ints[2 * e + 1] = s.src;
      }
      if (off)
        for (int k = 0; k < 3; ++k) off[3 * e + k] = s.off[k];
      ++e;
    }
  return RTFMM_OK;
}

int rtfmm_b200_get_leaf_lists(rtfmm_fmm* f, int32_t* list_off, int32_t* src_leaf, double* off, int64_t cap) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  const int nlf = (int)f->leaves.size();
  const bool mixed = f->args.precision == RTFMM_FP32_MIXED;
  std::vector<int> lo;
  std::vector<P2PSrc32> l32;
  std::vector<P2PSrc64> l64;
  if (f->p2p_on_device) {  // built on the GPU: fetch them
    lo.resize(nlf + 1);
    CK(cudaSetDevice(f->dev));
    CK(cudaMemcpy(lo.data(), f->d_list_off, sizeof(int) * (nlf + 1), cudaMemcpyDeviceToHost));
    if (mixed) {
      l32.resize(lo[nlf]);
      if (!l32.empty())
        CK(cudaMemcpy(l32.data(), f->d_list32, sizeof(P2PSrc32) * l32.size(), cudaMemcpyDeviceToHost));
    } else {
      l64.resize(lo[nlf]);
      if (!l64.empty())
        CK(cudaMemcpy(l64.data(), f->d_list64, sizeof(P2PSrc64) * l64.size(), cudaMemcpyDeviceToHost));
    }
  }
  const std::vector<int>& L = f->p2p_on_device ? lo : f->list_off;
  const std::vector<P2PSrc32>& A = f->p2p_on_device ? l32 : f->list32;
  const std::vector<P2PSrc64>& B = f->p2p_on_device ? l64 : f->list64;
  const int64_t m = L.empty() ? 0 : L[nlf];
  for (int l = 0; l <= nlf && list_off && !L.empty(); ++l) list_off[l] = L[l];
  if (!src_leaf && !off) return RTFMM_OK;  // a size query
  if (cap < m) return fail(RTFMM_EINVAL, "cap smaller than the number of list entries");
  for (int t = 0; t < nlf && m > 0; ++t) {
    const Cell& T = f->plan.cells[f->leaves[t].cell];
    for (int64_t e = L[t]; e < L[t + 1]; ++e) {
      const int sl = mixed ? A[e].leaf : B[e].leaf;
      if (src_leaf) src_leaf[e] = sl;
      if (!off) continue;
      if (mixed) {
        // the FP32 form keeps c_src + offset - c_tar; the offset is a whole
        // number of periods
        const Cell& S = f->plan.cells[f->leaves[sl].cell];
        const double d[3] = {A[e].dx, A[e].dy, A[e].dz};
        for (int k = 0; k < 3; ++k)
          off[3 * e + k] = std::nearbyint((d[k] - (S.x[k] - T.x[k])) / f->args.cycle) * f->args.cycle;
      } else {
        off[3 * e + 0] = B[e].ox;
        off[3 * e + 1] = B[e].oy;
        off[3 * e + 2] = B[e].oz;
      }
    }
  }
  return RTFMM_OK;
}

int rtfmm_b200_get_m2l(rtfmm_fmm* f, int32_t* ints, double* off) {
  if (!f) return fail(RTFMM_EINVAL, "null handle");
  if (!f->setup_done) return fail(RTFMM_ESTATE, "setup has not run");
  size_t e = 0;
  for (const auto& kv : f->plan.m2l)
    for (const M2LEntry& s : kv.second) {
      if (ints) {
        ints[3 * e] = kv.first;
        ints[3 * e + 1] = s.src;
        ints[3 * e + 2] = s.single;
      }
      if (off)
        for (int k = 0; k < 3; ++k) off[3 * e + k] = s.off[k];
      ++e;
    }
  return RTFMM_OK;
}

int rtfmm_b200_get_cell_vectors(rtfmm_fmm* f, int which, double* out) {
  if (!f || !out) return fail(RTFMM_EINVAL, "null argument");
  if (!f->pass_done) return fail(RTFMM_ESTATE, "no pass has run");
  if (which != 0 && which != 1) return fail(RTFMM_EINVAL, "which must be 0 or 1");
  CK(cudaSetDevice(f->dev));
  CK(cudaMemcpy(out, which == 0 ? f->d_qeq : f->d_pchk, sizeof(double) * f->plan.cells.size() * f->ops.ns,
                cudaMemcpyDeviceToHost));
  return RTFMM_OK;
}

int rtfmm_b200_get_operator(rtfmm_fmm* f, int which, double* out, int64_t cap) {
  if (!f || !out) return fail(RTFMM_EINVAL, "null argument");
  if (!f->ops_valid) return fail(RTFMM_ESTATE, "setup has not run");
  const Operators& o = f->ops;
  const size_t nn = (size_t)o.ns * o.ns;
  std::vector<double> v;
  if (which == 0) {
    v = o.pinv_up;
  } else if (which == 1) {
    v.resize(8 * nn);
    for (int k = 0; k < 8; ++k) std::memcpy(&v[k * nn], o.m2m[k].data(), sizeof(double) * nn);
  } else if (which == 2) {
    v = o.m2m_img_sum;
  } else if (which == 3) {
    v = o.cc8;
  } else if (which == 4) {
    v = o.U;
  } else if (which == 5) {
    v = o.VSinv;
  } else if (which == 6) {
    v = o.cc27sum;
  } else if (which == 7) {
    v = o.l2l_img;
  } else {
    return fail(RTFMM_EINVAL, "unknown operator");
  }
  if ((int64_t)v.size() > cap) return fail(RTFMM_EINVAL, "output buffer too small");
  std::memcpy(out, v.data(), sizeof(double) * v.size());
  return RTFMM_OK;
}

const char* rtfmm_b200_last_error(void) { return g_err.c_str(); }

void rtfmm_b200_clear_operator_cache(void) {
  std::lock_guard<std::mutex> lock(g_ops_mu);
  g_ops_cache.clear();
}

int rtfmm_b200_save_operators(rtfmm_fmm* f, const char* path) {
  if (!f || !path) return fail(RTFMM_EINVAL, "null argument");
  if (!f->ops_valid) return fail(RTFMM_ESTATE, "setup has not run");
  std::string err = save_operators(f->ops, path);
  if (!err.empty()) return fail(RTFMM_EINVAL, err);
  return RTFMM_OK;
}

int rtfmm_b200_load_operators(const char* path) {
  if (!path) return fail(RTFMM_EINVAL, "null path");
  try {
    Operators o;
    std::string err = load_operators(o, path);
    if (!err.empty()) return fail(RTFMM_EINVAL, err);
    if (!ops_lookup(o.P, o.images, o.r0)) ops_store(o);
  } catch (const std::bad_alloc&) {
    return fail(RTFMM_ENOMEM, "host allocation failed while loading operators");
  }
  return RTFMM_OK;
}

const char* rtfmm_b200_version(void) { return "rtfmm_b200 0.1 (sm_100a)"; }

}  // extern "C"
