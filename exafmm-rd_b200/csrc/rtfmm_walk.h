// One step of the P2P dual-tree walk, shared by the host walk
// (rtfmm_plan.cpp) and the GPU walk (rtfmm_lists.cu) so that both take the
// same decisions with the same floating-point operations.
//
// Traverser::horizontal_origin (3dpp/src/traverser.cpp:70-148): a frame is
// (target, source, target's parent, source's parent) under one periodic
// offset.  Non-adjacent pairs whose parents are adjacent become P2P when the
// leaf side is no deeper than the other side's parent (the reference's
// M2P/P2L cases, traverser.cpp:75-86); pairs whose parents are same-depth
// neighbours are M2L pairs of the parent map (not emitted here); adjacent
// leaf pairs are P2P; everything else divides the larger (or the non-leaf)
// side, children in order.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define RTFMM_HD __host__ __device__ __forceinline__
#else
#define RTFMM_HD inline
#endif

namespace rtfmm_b200 {

struct WalkFrame {
  int tc, sc, tcp, scp;
};

// C provides x(c, k), r(c), depth(c), cnum(c), coff(c) for cell c.
template <class C>
RTFMM_HD bool walk_adjacent(const C& cells, int a, int b, const double* off) {
  // |x_a - x_b - offset| <= (r_a + r_b) * 1.001 per axis (traverser.cpp:314-321)
  const double dist = (cells.r(a) + cells.r(b)) * 1.001;
  for (int k = 0; k < 3; ++k) {
    const double d = fabs((cells.x(a, k) - cells.x(b, k)) - off[k]);
    if (!(d <= dist)) return false;
  }
  return true;
}

// Returns 1 and sets *hit (the source cell) for a P2P pair; -k and the k
// child frames in visiting order for a division; 0 otherwise.
template <class C>
RTFMM_HD int walk_step(const C& cells, const WalkFrame& f, const double* off, int* hit, WalkFrame* kids) {
  int divide = 0;
  const bool tleaf = cells.cnum(f.tc) == 0, sleaf = cells.cnum(f.sc) == 0;
  if (!walk_adjacent(cells, f.tc, f.sc, off)) {
    if (walk_adjacent(cells, f.tc, f.scp, off) && tleaf && cells.depth(f.scp) >= cells.depth(f.tc)) {
      *hit = f.sc;
      return 1;
    } else if (walk_adjacent(cells, f.tcp, f.sc, off) && sleaf && cells.depth(f.tcp) >= cells.depth(f.sc)) {
      *hit = f.sc;
      return 1;
    } else if (walk_adjacent(cells, f.tcp, f.scp, off) && cells.depth(f.tcp) == cells.depth(f.scp)) {
      // an M2L pair of the dual walk; served by the parent map
    } else {
      if (tleaf && sleaf) {
      } else if (!tleaf && sleaf) {
        divide = 1;
      } else if (tleaf && !sleaf) {
        divide = 2;
      } else {
        divide = cells.r(f.tc) >= cells.r(f.sc) ? 1 : 2;
      }
    }
  } else {
    if (tleaf && sleaf) {
      *hit = f.sc;
      return 1;
    } else if (!tleaf && sleaf) {
      divide = 1;
    } else if (tleaf && !sleaf) {
      divide = 2;
    } else {
      divide = cells.r(f.tc) >= cells.r(f.sc) ? 1 : 2;
    }
  }
  if (divide == 1) {
    const int n = cells.cnum(f.tc), c0 = cells.coff(f.tc);
    for (int i = 0; i < n; ++i) kids[i] = {c0 + i, f.sc, f.tc, f.scp};
    return -n;
  }
  if (divide == 2) {
    const int n = cells.cnum(f.sc), c0 = cells.coff(f.sc);
    for (int i = 0; i < n; ++i) kids[i] = {f.tc, c0 + i, f.tcp, f.sc};
    return -n;
  }
  return 0;
}

}  // namespace rtfmm_b200
