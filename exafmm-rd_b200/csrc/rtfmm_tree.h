// GPU octree construction for bodies already in device memory.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

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
// GPU, into plan.p2p: the same entries in the same order as traverse_p2p.
// Scratch slots slot_base .. slot_base + 27.  kTreeTooDeep: the walk is
// deeper than 40 divisions or the tree has 2^25 cells or more (use
// traverse_p2p).
int device_p2p_walk(Plan& plan, const std::vector<WalkRoot>& roots, cudaStream_t st, const TreeScratchFn& scratch,
                    int slot_base, std::string& msg);

}  // namespace rtfmm_b200
