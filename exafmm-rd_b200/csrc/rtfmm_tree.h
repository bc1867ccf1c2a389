// GPU octree construction for bodies already in device memory.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "rtfmm_plan.h"

namespace rtfmm_b200 {

constexpr int kTreeOk = 0;
constexpr int kTreeTooDeep = 1;  // needs more than 21 levels: build on the host
constexpr int kTreeError = -1;   // CUDA error or non-finite position (msg says which)

// Fills plan.cells (tree cells, breadth-first), plan.ntree, plan.perm, plan.n
// and plan.r0 from n positions x_dev (n x 3, device memory), with plan.args
// set; the result equals build_tree's on the same positions.  Runs on `st`
// and returns when the host-side plan is complete.
int device_build_tree(const double* x_dev, int64_t n, cudaStream_t st, Plan& plan, std::string& msg);

}  // namespace rtfmm_b200
