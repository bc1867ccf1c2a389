// GPU octree construction for bodies already in device memory.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "rtfmm_kernels.cuh"
#include "rtfmm_plan.h"

namespace rtfmm_b200 {

constexpr int kTreeOk = 0;
constexpr int kTreeTooDeep = 1;  // needs more than 21 levels: build on the host
constexpr int kTreeError = -1;   // CUDA error or non-finite position (msg says which)

// Device scratch by slot (0, 1, 2, ...): a buffer of at least `bytes`,
// nullptr when none can be had.  The caller keeps the buffers between calls.
using TreeScratchFn = std::function<void*(int slot, size_t bytes)>;

// Fills plan.cells (tree cells, breadth-first), plan.ntree, plan.n and
// plan.r0 from n bodies in device memory (x_dev n x 3, q_dev n), with
// plan.args set, and writes the body permutation (tree position -> input
// index) to d_perm (n, device).  The result equals build_tree's on the same
// positions.  Work runs on `st`; the permutation may still be in flight on
// return.  Non-finite positions or charges give kTreeError.
int device_build_tree(const double* x_dev, const double* q_dev, int64_t n, cudaStream_t st, Plan& plan,
                      int64_t* d_perm, const TreeScratchFn& scratch, std::string& msg);

// The P2P lists of the dual-tree walk from `roots` (traverse_begin) on the
// GPU: the same entries in the same order as traverse_p2p, into plan.p2p
// when host_lists (else left on the device, plan.p2p empty: see
// device_walk_host_lists).  Scratch slots slot_base .. slot_base + 27.
// kTreeTooDeep: the walk is deeper than 40 divisions or the tree has 2^25
// cells or more (use traverse_p2p).
// What the GPU walk leaves on the device (in its scratch slots, valid until
// they are reused): the pairs sorted by target cell, depth-first within one
// (target << 30 | source << 5 | walk), the walks' offsets, the cells' body
// ranges.
struct DeviceWalk {
  const unsigned long long* pairs = nullptr;
  int npairs = 0;
  const double* offs = nullptr;
  int nwalk = 0, ncell = 0;
  const int* cboff = nullptr;
  const int* cbnum = nullptr;
  std::vector<V3> host_offs;  // the walks' offsets (roots' order)
};
int device_p2p_walk(Plan& plan, const std::vector<WalkRoot>& roots, cudaStream_t st, const TreeScratchFn& scratch,
                    int slot_base, DeviceWalk* dw, std::string& msg, bool host_lists = true);
// plan.p2p from a walk left on the device (its pairs copied back).
int device_walk_host_lists(const DeviceWalk& dw, Plan& plan, cudaStream_t st, std::string& msg);

// The pass's P2P tables built on the GPU from the walk's pairs: list
// offsets by target leaf, the list entries (FP32 or FP64 form) and the work
// items, equal to the host build's.  Inputs on the device: the leaf table,
// the cells' parents (-1 at the root), each body's leaf, the leaves in
// first-body order and each leaf's position in it.
struct DeviceLeafInput {
  const LeafInfo* leaves;
  int nlf;
  const int* parent;
  const int* body_leaf;
  const int* dfs;
  const int* dfs_pos;
};
// Device buffers of the outputs, from the caller (nullptr on failure).
struct P2PTableAlloc {
  std::function<int*(int)> list_off;
  std::function<P2PSrc32*(int)> list32;
  std::function<P2PSrc64*(int)> list64;
  std::function<P2PItem32*(int)> items;
};
struct P2PTablesOut {
  int nlist = 0, nitems = 0;
  int64_t pairs = 0;  // body pairs: sum over entries of n_target * n_source
};
int device_p2p_tables(const DeviceWalk& w, const DeviceLeafInput& in, bool mixed, cudaStream_t st,
                      const TreeScratchFn& scratch, int slot_base, const P2PTableAlloc& alloc, P2PTablesOut* out,
                      std::string& msg);

}  // namespace rtfmm_b200
