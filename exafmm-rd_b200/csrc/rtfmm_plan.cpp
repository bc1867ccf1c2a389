// Host-side set-up: adaptive octree, interaction lists and FP64 operator
// tables.  These restate the reference's algorithms so that the lists and the
// operators are the same sets the reference builds; the evaluation pass
// itself runs on the GPU (rtfmm_kernels.cu).
#include "rtfmm_plan.h"
#include "rtfmm_walk.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <utility>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace rtfmm_b200 {

static const int kMaxDepth = 40;

static double wall_now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// octree: Tree::build_nonuniform_octree (3dpp/src/tree.cpp:102-188)
// ---------------------------------------------------------------------------
static V3 child_center(const V3& xp, double rp, int octant) {
  // Tree::get_child_cell_x, non-periodic branch (tree.cpp:198-209)
  V3 c;
  c[0] = xp[0] + ((octant & 4) ? rp / 2 : -rp / 2);
  c[1] = xp[1] + ((octant & 2) ? rp / 2 : -rp / 2);
  c[2] = xp[2] + ((octant & 1) ? rp / 2 : -rp / 2);
  return c;
}

// Splits one cell's bodies into its octants: a stable counting partition of
// perm[b0, b0+nb) by the octant code 4(x>cx)+2(y>cy)+(z>cz).  Large cells are
// partitioned by all threads (per-thread counts over contiguous chunks, so the
// result is the same stable order); small ones by the calling thread.
static void split_cell(const double* xin, const Cell& cell, std::vector<int64_t>& perm, std::vector<int64_t>& tmp,
                       std::vector<uint8_t>& code, int count[8], bool parallel) {
  const int64_t b0 = cell.boff, nb = cell.bnum;
  auto octant = [&](int64_t i) {
    const double* p = xin + 3 * perm[b0 + i];
    return ((p[0] > cell.x[0]) << 2) + ((p[1] > cell.x[1]) << 1) + (p[2] > cell.x[2]);
  };
  int nt = 1;
#ifdef _OPENMP
  if (parallel) nt = std::max(1, std::min(omp_get_max_threads(), (int)(nb / 16384)));
#endif
  std::vector<int64_t> cnt((size_t)nt * 8, 0), off((size_t)nt * 8, 0);
#pragma omp parallel for num_threads(nt) schedule(static, 1) if (nt > 1)
  for (int t = 0; t < nt; ++t) {
    const int64_t i0 = nb * t / nt, i1 = nb * (t + 1) / nt;
    for (int64_t i = i0; i < i1; ++i) {
      const int o = octant(i);
      code[b0 + i] = (uint8_t)o;
      cnt[(size_t)t * 8 + o]++;
    }
  }
  int64_t run = 0;
  for (int o = 0; o < 8; ++o) {
    int64_t c = 0;
    for (int t = 0; t < nt; ++t) {
      off[(size_t)t * 8 + o] = run + c;
      c += cnt[(size_t)t * 8 + o];
    }
    count[o] = (int)c;
    run += c;
  }
#pragma omp parallel for num_threads(nt) schedule(static, 1) if (nt > 1)
  for (int t = 0; t < nt; ++t) {
    const int64_t i0 = nb * t / nt, i1 = nb * (t + 1) / nt;
    int64_t fill[8];
    for (int o = 0; o < 8; ++o) fill[o] = off[(size_t)t * 8 + o];
    for (int64_t i = i0; i < i1; ++i) tmp[b0 + fill[code[b0 + i]]++] = perm[b0 + i];
  }
#pragma omp parallel for num_threads(nt) schedule(static) if (nt > 1)
  for (int64_t i = 0; i < nb; ++i) perm[b0 + i] = tmp[b0 + i];
}

std::string build_tree(Plan& plan, const double* xin, const double* qin) {
  const int64_t n = plan.n;
  const Args& a = plan.args;
  plan.r0 = a.cycle / 2;
  plan.cells.clear();
  plan.perm.resize(n);
  for (int64_t i = 0; i < n; ++i) plan.perm[i] = i;
  std::vector<int64_t> tmp(n);
  std::vector<uint8_t> code(n);

  Cell root;
  root.octant = 13;
  root.depth = 0;
  root.r = plan.r0;
  root.x = a.x;
  root.coff = 0;
  root.cnum = 0;
  root.boff = 0;
  root.bnum = (int)n;
  plan.cells.push_back(root);
  // Breadth-first, one level at a time: the cells of a level split their own
  // body ranges independently (in parallel), then their children are appended
  // in cell order, octants in order -- the queue order of the reference's
  // breadth-first build, so cells and the body permutation are the same.
  size_t lev0 = 0, lev1 = 1;
  const int64_t big = 1 << 18;
  while (lev0 < lev1) {
    const int nl = (int)(lev1 - lev0);
    std::vector<std::array<int, 8>> counts(nl);
    int deep = 0;
    for (int k = 0; k < nl; ++k) {
      const Cell& c = plan.cells[lev0 + k];
      if (c.bnum > a.ncrit && c.depth >= kMaxDepth) deep = 1;
    }
    if (deep) return "octree deeper than 40 levels: more than ncrit bodies share a position";
    // large cells: every thread on one cell; the rest: one cell per thread
    for (int k = 0; k < nl; ++k) {
      const Cell& c = plan.cells[lev0 + k];
      if (c.bnum > a.ncrit && c.bnum >= big) split_cell(xin, c, plan.perm, tmp, code, counts[k].data(), true);
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < nl; ++k) {
      const Cell& c = plan.cells[lev0 + k];
      if (c.bnum > a.ncrit && c.bnum < big) split_cell(xin, c, plan.perm, tmp, code, counts[k].data(), false);
    }
    for (int k = 0; k < nl; ++k) {
      const int ci = (int)(lev0 + k);
      const Cell cell = plan.cells[ci];
      if (cell.bnum <= a.ncrit) continue;
      const int* count = counts[k].data();
      int nchild = 0, s = 0;
      const int insert = (int)plan.cells.size();
      for (int o = 0; o < 8; ++o) {
        if (count[o] == 0) {
          continue;
        }
        Cell ch;
        ch.octant = o;
        ch.depth = cell.depth + 1;
        ch.r = cell.r / 2;
        ch.x = child_center(cell.x, cell.r, o);
        ch.coff = 0;
        ch.cnum = 0;
        ch.boff = cell.boff + s;
        ch.bnum = count[o];
        plan.cells.push_back(ch);
        s += count[o];
        nchild++;
      }
      plan.cells[ci].coff = insert;
      plan.cells[ci].cnum = nchild;
    }
    lev0 = lev1;
    lev1 = plan.cells.size();
  }
  plan.ntree = (int)plan.cells.size();
  plan.x.resize(3 * n);
  plan.q.resize(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t k = plan.perm[i];
    plan.x[3 * i + 0] = xin[3 * k + 0];
    plan.x[3 * i + 1] = xin[3 * k + 1];
    plan.x[3 * i + 2] = xin[3 * k + 2];
    plan.q[i] = qin[k];
  }
  return "";
}

// ---------------------------------------------------------------------------
// lists: Traverser (3dpp/src/traverser.cpp)
// ---------------------------------------------------------------------------
namespace {

struct Walker {
  Plan& p;
  explicit Walker(Plan& pl) : p(pl) {}

  // adjacent(a, b, offset): |x_a - x_b - offset| <= (r_a + r_b) * 1.001 per axis
  // (traverser.cpp:314-321), evaluated with the same operation order.
  bool adjacent(int a, int b, const V3& off) const {
    const Cell& ca = p.cells[a];
    const Cell& cb = p.cells[b];
    const double dist = (ca.r + cb.r) * 1.001;
    for (int k = 0; k < 3; ++k) {
      double d = std::fabs((ca.x[k] - cb.x[k]) - off[k]);
      if (!(d <= dist)) return false;
    }
    return true;
  }
  bool neighbour(int a, int b, const V3& off) const {
    return adjacent(a, b, off) && p.cells[a].depth == p.cells[b].depth;
  }
  bool leaf(int c) const { return p.cells[c].cnum == 0; }

  // horizontal_origin (traverser.cpp:70-148) as a stack of frames; children
  // are visited in the reference's recursion order.  M2P/P2L cases become P2P
  // (traverser.cpp:75-86); M2L pairs of the dual walk are counted only (the
  // M2L of the pass uses the parent map).  The step itself is walk_step
  // (rtfmm_walk.h), which the GPU walk runs too.
  using Frame = WalkFrame;
  struct Cells {
    const std::vector<Cell>& c;
    double x(int i, int k) const { return c[i].x[k]; }
    double r(int i) const { return c[i].r; }
    int depth(int i) const { return c[i].depth; }
    int cnum(int i) const { return c[i].cnum; }
    int coff(int i) const { return c[i].coff; }
  };
  int step(const Frame& f, const V3& off, int* hit, Frame* kids) const {
    return walk_step(Cells{p.cells}, f, off.data(), hit, kids);
  }

  // The walk below one frame, its P2P pairs (target, source) appended in the
  // order the recursion emits them.
  void walk(const Frame& f0, const V3& off, std::vector<std::pair<int, int>>& out) const {
    std::vector<Frame> stack;
    stack.push_back(f0);
    Frame kids[8];
    while (!stack.empty()) {
      const Frame f = stack.back();
      stack.pop_back();
      int hit = -1;
      const int r = step(f, off, &hit, kids);
      if (r == 1) {
        out.push_back({f.tc, hit});
      } else if (r < 0) {
        for (int i = -r - 1; i >= 0; --i) stack.push_back(kids[i]);
      }
    }
  }

  // The walks of all root frames (one per periodic offset), split into the
  // subtrees of their first frames and run in parallel.  A frame either emits
  // one pair or divides, so the output of a walk is the concatenation of its
  // subtrees' outputs in visiting order; they are merged in that order, and
  // the lists are the ones the sequential recursion builds.
  void walks(const std::vector<Frame>& roots, const std::vector<V3>& offs) {
    struct Item {
      Frame f;
      int walk;
      int hit;  // >= 0: an emitted pair, no frame
    };
    std::vector<Item> items;
    for (size_t w = 0; w < roots.size(); ++w) items.push_back({roots[w], (int)w, -1});
    Frame kids[8];
    for (int round = 0; round < 6 && items.size() < 4096; ++round) {
      std::vector<Item> next;
      next.reserve(items.size() * 8);
      for (const Item& it : items) {
        if (it.hit >= 0) {
          next.push_back(it);
          continue;
        }
        int hit = -1;
        const int r = step(it.f, offs[(size_t)it.walk], &hit, kids);
        if (r == 1) {
          next.push_back({it.f, it.walk, hit});
        } else if (r < 0) {
          for (int i = 0; i < -r; ++i) next.push_back({kids[i], it.walk, -1});
        }
      }
      items.swap(next);
    }
    std::vector<std::vector<std::pair<int, int>>> outs(items.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < (int)items.size(); ++i) {
      const Item& it = items[(size_t)i];
      if (it.hit >= 0)
        outs[(size_t)i].push_back({it.f.tc, it.hit});
      else
        walk(it.f, offs[(size_t)it.walk], outs[(size_t)i]);
    }
    // Merge in item order: chunks of items count their pairs per target,
    // the counts give each chunk its place in every target's list, and the
    // chunks fill their places in parallel -- the lists of the sequential
    // merge, entry for entry.
    const int ni = (int)items.size();
    int T = 1;
#ifdef _OPENMP
    T = std::max(1, std::min(omp_get_max_threads(), ni));
#endif
    int ncell = 0;
    for (const auto& o : outs)
      for (const auto& pr : o) ncell = std::max(ncell, pr.first + 1);
    std::vector<int> cnt((size_t)T * ncell, 0);
#pragma omp parallel for num_threads(T) schedule(static, 1) if (T > 1)
    for (int t = 0; t < T; ++t) {
      int* c = &cnt[(size_t)t * ncell];
      for (int i = ni * t / T; i < ni * (t + 1) / T; ++i)
        for (const auto& pr : outs[(size_t)i]) c[pr.first]++;
    }
    if ((int)p.p2p.v.size() < ncell) p.p2p.v.resize(ncell);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < ncell; ++c) {
      int run = (int)p.p2p.v[(size_t)c].size();
      for (int t = 0; t < T; ++t) {
        const int k = cnt[(size_t)t * ncell + c];
        cnt[(size_t)t * ncell + c] = run;
        run += k;
      }
      p.p2p.v[(size_t)c].resize(run);
    }
#pragma omp parallel for num_threads(T) schedule(static, 1) if (T > 1)
    for (int t = 0; t < T; ++t) {
      int* at = &cnt[(size_t)t * ncell];
      for (int i = ni * t / T; i < ni * (t + 1) / T; ++i)
        for (const auto& pr : outs[(size_t)i])
          p.p2p.v[(size_t)pr.first][(size_t)at[pr.first]++] = {pr.second, offs[(size_t)items[(size_t)i].walk]};
    }
  }
};

}  // namespace

std::vector<WalkRoot> traverse_begin(Plan& plan) {
  const Args& a = plan.args;
  const double cycle = a.cycle;
  plan.p2p.clear();
  plan.m2l.clear();
  // The depth -1 super-cell exists before the tree-level M2L parent map is
  // built (traverser.cpp:30-35); deeper image cells are added afterwards.
  if (a.images == 0) return {WalkRoot{0, 0, 0, 0, V3{0, 0, 0}}};
  Cell c;
  c.octant = 13;
  c.depth = -1;
  c.r = plan.cells[0].r * 3;
  c.x = plan.cells[0].x;
  c.coff = 0;
  c.cnum = 1;
  c.boff = 0;
  c.bnum = plan.cells[0].bnum;
  plan.cells.push_back(c);
  const int cidx = (int)plan.cells.size() - 1;
  std::vector<WalkRoot> roots;
  for (int pz = -1; pz <= 1; ++pz)
    for (int py = -1; py <= 1; ++py)
      for (int px = -1; px <= 1; ++px) roots.push_back({0, 0, cidx, cidx, V3{px * cycle, py * cycle, pz * cycle}});
  return roots;
}

void traverse_p2p(Plan& plan, const std::vector<WalkRoot>& roots) {
  Walker w(plan);
  std::vector<Walker::Frame> frames;
  std::vector<V3> offs;
  for (const WalkRoot& r : roots) {
    frames.push_back({r.tc, r.sc, r.tcp, r.scp});
    offs.push_back(r.off);
  }
  w.walks(frames, offs);
}

void traverse(Plan& plan) {
  traverse_p2p(plan, traverse_begin(plan));
  traverse_finish(plan);
}

void traverse_finish(Plan& plan) {
  const Args& a = plan.args;
  const double cycle = a.cycle;
  Walker w(plan);
  // M2L parent map over the tree cells (make_M2L_parent_map and the
  // periodic part of make_M2L_parent_map_i1, traverser.cpp:234-282).  The
  // reference tests every cell pair; same-depth cells sit on a lattice of
  // spacing 2r, so the same predicate is evaluated here for the cell at each
  // lattice displacement v in {-1,0,1}^3 (wrapped periodically when images
  // >= 1, with offset p * cycle).  A cell at depth d and lattice coordinate m
  // is found by descending from the root along the bits of m (bit d - l of
  // each axis gives the octant at level l).
  const V3 lo{a.x[0] - plan.r0, a.x[1] - plan.r0, a.x[2] - plan.r0};
  std::vector<std::array<int64_t, 3>> coord(plan.ntree);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < plan.ntree; ++c) {
    const Cell& cl = plan.cells[c];
    for (int k = 0; k < 3; ++k)
      coord[c][k] = (int64_t)std::llround((cl.x[k] - lo[k]) / (2 * cl.r) - 0.5);
  }
  // each tree cell's child by octant (-1: none)
  std::vector<std::array<int, 8>> child(plan.ntree);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < plan.ntree; ++c) {
    const Cell& cl = plan.cells[c];
    child[c].fill(-1);
    for (int k = 0; k < cl.cnum; ++k) child[c][plan.cells[cl.coff + k].octant & 7] = cl.coff + k;
  }
  // the non-leaf tree cell at (depth, m), or -1
  auto lattice_cell = [&](int depth, const int64_t m[3]) {
    int c = 0;
    for (int l = 1; l <= depth && c >= 0; ++l) {
      const int sh = depth - l;
      c = child[c][(((m[0] >> sh) & 1) << 2) | (((m[1] >> sh) & 1) << 1) | ((m[2] >> sh) & 1)];
    }
    return c >= 0 && plan.cells[c].cnum > 0 ? c : -1;
  };
  // each parent's list is written by one thread (lists sized up front; the
  // lattice is only read)
  if ((int)plan.m2l.v.size() < plan.ntree) plan.m2l.v.resize(plan.ntree);
#pragma omp parallel for schedule(dynamic, 256)
  for (int j = 0; j < plan.ntree; ++j) {
    const Cell& T = plan.cells[j];
    if (T.cnum == 0) continue;
    const int64_t nside = (int64_t)1 << T.depth;
    M2LEntry near[26], far[26];
    int nn = 0, nf = 0;
    for (int vz = -1; vz <= 1; ++vz)
      for (int vy = -1; vy <= 1; ++vy)
        for (int vx = -1; vx <= 1; ++vx) {
          if (vx == 0 && vy == 0 && vz == 0) continue;
          int64_t m[3] = {coord[j][0] + vx, coord[j][1] + vy, coord[j][2] + vz};
          int pw[3] = {0, 0, 0};
          bool inside = true;
          for (int k = 0; k < 3; ++k) {
            if (m[k] < 0) { m[k] += nside; pw[k] = -1; }
            else if (m[k] >= nside) { m[k] -= nside; pw[k] = 1; }
            if (pw[k] != 0) inside = false;
          }
          if (!inside && a.images == 0) continue;
          const int src = lattice_cell(T.depth, m);
          if (src < 0) continue;
          V3 off{pw[0] * cycle, pw[1] * cycle, pw[2] * cycle};
          // confirm with the reference's own predicate
          if (!w.neighbour(j, src, off)) continue;
          if (inside)
            near[nn++] = {src, off, 0};
          else
            far[nf++] = {src, off, 0};
        }
    if (nn + nf > 0) {
      auto& lst = plan.m2l.v[(size_t)j];
      lst.reserve(lst.size() + nn + nf);
      lst.insert(lst.end(), near, near + nn);
      lst.insert(lst.end(), far, far + nf);
    }
  }

  if (a.images >= 2) {
    // horizontal_periodic_far: image super-cells at depth -2 .. -images
    // (traverser.cpp:178-196), each the single parent of the one above.
    int child = (int)plan.cells.size() - 1;
    for (int m = 1; m < a.images; ++m) {
      Cell c;
      c.octant = 13;
      c.depth = -1 - m;
      c.r = plan.cells[child].r * 3;
      c.x = plan.cells[child].x;
      c.coff = child;
      c.cnum = 1;
      c.boff = 0;
      c.bnum = 0;
      plan.cells.push_back(c);
      child = (int)plan.cells.size() - 1;
    }
    // image-level parent entries (traverser.cpp:43-64)
    const int idx = (int)plan.cells.size() - 1 - a.images;
    for (int m = 1; m < a.images; ++m) {
      const int ci = idx + m;
      const double r = plan.cells[ci].r;
      for (int pz = -1; pz <= 1; ++pz)
        for (int py = -1; py <= 1; ++py)
          for (int px = -1; px <= 1; ++px) {
            if (px == 0 && py == 0 && pz == 0) continue;
            V3 off{px * r * 2, py * r * 2, pz * r * 2};
            plan.m2l[ci].push_back({ci, off, 1});
          }
    }
  }
  plan.dmin = plan.dmax = plan.cells[0].depth;
  for (const Cell& c : plan.cells) {
    plan.dmin = std::min(plan.dmin, c.depth);
    plan.dmax = std::max(plan.dmax, c.depth);
  }
  plan.n_p2p = 0;
  for (const auto& kv : plan.p2p) plan.n_p2p += (int64_t)kv.second.size();
  plan.n_m2l = 0;
  for (const auto& kv : plan.m2l) plan.n_m2l += (int64_t)kv.second.size();
}

// ---------------------------------------------------------------------------
// dense helpers
// ---------------------------------------------------------------------------
// One-sided (Hestenes) Jacobi SVD of a square row-major matrix: rotate column
// pairs of W = A V until they are mutually orthogonal; then W = U S.  Pairs
// follow a round-robin tournament so that each round's rotations are
// independent and run in parallel.
std::vector<int> jacobi_pairs(int n) {
  const int m = n + (n & 1);
  std::vector<int> ring(m), out;
  for (int i = 0; i < m; ++i) ring[i] = i;
  for (int round = 0; round < m - 1; ++round) {
    for (int k = 0; k < m / 2; ++k) {
      int p = ring[k], q = ring[m - 1 - k];
      if (p > q) std::swap(p, q);
      out.push_back(p);
      out.push_back(q);
    }
    // rotate the tournament ring, keeping ring[0] fixed
    int last = ring[m - 1];
    for (int i = m - 1; i > 1; --i) ring[i] = ring[i - 1];
    ring[1] = last;
  }
  return out;
}

// The three inner products of a column pair in the order of a 32-lane warp:
// lane l sums the terms i = l, l + 32, ... in order, then the lanes are
// combined by the butterfly of a warp reduction (partner l ^ 16, l ^ 8, ...,
// l ^ 1; FP addition commutes, so every lane ends with the same sum).
void jacobi_dots(int n, const double* wp, const double* wq, double& alpha, double& beta, double& gamma) {
  double a[32] = {}, b[32] = {}, g[32] = {};
  int i0 = 0;
  for (; i0 + 32 <= n; i0 += 32)
    for (int l = 0; l < 32; ++l) {
      a[l] += wp[i0 + l] * wp[i0 + l];
      b[l] += wq[i0 + l] * wq[i0 + l];
      g[l] += wp[i0 + l] * wq[i0 + l];
    }
  for (int l = 0; i0 + l < n; ++l) {
    a[l] += wp[i0 + l] * wp[i0 + l];
    b[l] += wq[i0 + l] * wq[i0 + l];
    g[l] += wp[i0 + l] * wq[i0 + l];
  }
  // lanes l and l ^ o hold equal sums after each step, so lanes 0..o-1 carry
  // all of them
  for (int o = 16; o >= 1; o >>= 1)
    for (int l = 0; l < o; ++l) {
      a[l] = a[l] + a[l + o];
      b[l] = b[l] + b[l + o];
      g[l] = g[l] + g[l + o];
    }
  alpha = a[0];
  beta = b[0];
  gamma = g[0];
}

void jacobi_sweeps_host(int n, std::vector<double>& W, std::vector<double>& Vc) {
  const int m = n + (n & 1);
  const std::vector<int> pairs = jacobi_pairs(n);
  for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
    double off_max = 0.0;
    for (int round = 0; round < m - 1; ++round) {
      const int* pr = &pairs[(size_t)round * m];
#pragma omp parallel for schedule(static) reduction(max : off_max)
      for (int k = 0; k < m / 2; ++k) {
        const int p = pr[2 * k], q = pr[2 * k + 1];
        if (q >= n) continue;  // padding column
        double* wp = &W[(size_t)p * n];
        double* wq = &W[(size_t)q * n];
        double alpha, beta, gamma;
        jacobi_dots(n, wp, wq, alpha, beta, gamma);
        if (alpha == 0.0 || beta == 0.0) continue;
        const double rel = std::fabs(gamma) / std::sqrt(alpha * beta);
        off_max = std::max(off_max, rel);
        if (rel < kJacobiTol) continue;
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / std::sqrt(1.0 + t * t);
        const double sn = c * t;
        for (int i = 0; i < n; ++i) {
          const double a1 = wp[i], b1 = wq[i];
          wp[i] = c * a1 - sn * b1;
          wq[i] = sn * a1 + c * b1;
        }
        double* vp = &Vc[(size_t)p * m];
        double* vq = &Vc[(size_t)q * m];
        for (int i = 0; i < n; ++i) {
          const double a1 = vp[i], b1 = vq[i];
          vp[i] = c * a1 - sn * b1;
          vq[i] = sn * a1 + c * b1;
        }
      }
    }
    if (off_max < kJacobiTol) break;
  }
}

// Classical Gram-Schmidt, two passes, on the rows of Q (n x n) in order:
// row k loses its components along rows 0..k-1, then is normalised (a zero
// row stays zero).  Every inner product runs over its index in order.
void reorthogonalize_host(int n, double* Q) {
  std::vector<double> h(n);
  for (int k = 0; k < n; ++k) {
    double* u = &Q[(size_t)k * n];
    double nrm = 0;
    for (int i = 0; i < n; ++i) nrm += u[i] * u[i];
    if (nrm == 0.0) continue;  // s_k = 0: not inverted
    for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel for schedule(static)
      for (int j = 0; j < k; ++j) {
        const double* qj = &Q[(size_t)j * n];
        double d = 0;
        for (int i = 0; i < n; ++i) d += qj[i] * u[i];
        h[j] = d;
      }
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; ++i) {
        double acc = 0;
        for (int j = 0; j < k; ++j) acc += h[j] * Q[(size_t)j * n + i];
        u[i] -= acc;
      }
    }
    nrm = 0;
    for (int i = 0; i < n; ++i) nrm += u[i] * u[i];
    nrm = std::sqrt(nrm);
    for (int i = 0; i < n; ++i) u[i] = nrm > 0 ? u[i] / nrm : 0.0;
  }
}

void jacobi_svd(int n, const double* A, std::vector<double>& U, std::vector<double>& s, std::vector<double>& V,
                const DenseBackend* be, const std::function<void()>& after_sweeps) {
  const int m = n + (n & 1);
  std::vector<double> W((size_t)m * n, 0.0), Vc((size_t)m * m, 0.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) W[(size_t)j * n + i] = A[(size_t)i * n + j];
  for (int j = 0; j < m; ++j) Vc[(size_t)j * m + j] = 1.0;
  if (be && be->jacobi_sweeps)
    be->jacobi_sweeps(n, W, Vc);
  else
    jacobi_sweeps_host(n, W, Vc);
  if (after_sweeps) after_sweeps();
  std::vector<std::pair<double, int>> sv(n);
  for (int j = 0; j < n; ++j) {
    double nr = 0;
    for (int i = 0; i < n; ++i) nr += W[(size_t)j * n + i] * W[(size_t)j * n + i];
    sv[j] = {std::sqrt(nr), j};
  }
  std::sort(sv.begin(), sv.end(), [](const std::pair<double, int>& x, const std::pair<double, int>& y) {
    return x.first > y.first;
  });
  U.assign((size_t)n * n, 0.0);
  V.assign((size_t)n * n, 0.0);
  s.assign(n, 0.0);
  for (int k = 0; k < n; ++k) {
    const int j = sv[k].second;
    s[k] = sv[k].first;
    for (int i = 0; i < n; ++i) {
      U[(size_t)i * n + k] = s[k] > 0 ? W[(size_t)j * n + i] / s[k] : 0.0;
      V[(size_t)i * n + k] = Vc[(size_t)j * m + i];
    }
  }
  // u_k = A v_k / s_k carries the rounding of A v_k (about eps * s_max)
  // divided by s_k, so the columns of singular values near eps * s_max are
  // far from orthogonal to the dominant ones (0.7 at P = 10, cond 1.3e16),
  // and the pseudo-inverse then turns smooth check potentials into huge
  // equivalent densities.  An orthogonal factorisation (the reference's
  // dgesvd) returns an orthonormal U; re-orthogonalise the columns in order
  // of decreasing s (classical Gram-Schmidt, two passes) to the same effect.
  // At P <= 8 this changes U by ~1e-15.
  std::vector<double> Q((size_t)n * n);
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i) Q[(size_t)k * n + i] = U[(size_t)i * n + k];
  if (be && be->reorthogonalize)
    be->reorthogonalize(n, Q.data());
  else
    reorthogonalize_host(n, Q.data());
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i) U[(size_t)i * n + k] = Q[(size_t)k * n + i];
}

// Real-to-complex 3D DFT of an N^3 grid stored [z][y][x] (x fastest), forward
// sign e^{-2 pi i k.n / N}, unnormalised; output [kz][ky][kx] with
// kx in [0, N/2] (the half-spectrum layout of an r2c transform).
void dft3_r2c(int N, const double* in, double* out) {
  const int Nh = N / 2 + 1;
  std::vector<double> cs(N), sn(N);
  for (int m = 0; m < N; ++m) {
    cs[m] = std::cos(2.0 * M_PI * m / N);
    sn[m] = -std::sin(2.0 * M_PI * m / N);
  }
  std::vector<double> a((size_t)N * N * Nh * 2), b((size_t)N * N * Nh * 2);
  for (int z = 0; z < N; ++z)
    for (int y = 0; y < N; ++y)
      for (int kx = 0; kx < Nh; ++kx) {
        double re = 0, im = 0;
        for (int x = 0; x < N; ++x) {
          const int t = (kx * x) % N;
          const double v = in[((size_t)z * N + y) * N + x];
          re += v * cs[t];
          im += v * sn[t];
        }
        size_t o = (((size_t)z * N + y) * Nh + kx) * 2;
        a[o] = re;
        a[o + 1] = im;
      }
  for (int z = 0; z < N; ++z)
    for (int ky = 0; ky < N; ++ky)
      for (int kx = 0; kx < Nh; ++kx) {
        double re = 0, im = 0;
        for (int y = 0; y < N; ++y) {
          const int t = (ky * y) % N;
          size_t o = (((size_t)z * N + y) * Nh + kx) * 2;
          re += a[o] * cs[t] - a[o + 1] * sn[t];
          im += a[o] * sn[t] + a[o + 1] * cs[t];
        }
        size_t o = (((size_t)z * N + ky) * Nh + kx) * 2;
        b[o] = re;
        b[o + 1] = im;
      }
  for (int kz = 0; kz < N; ++kz)
    for (int ky = 0; ky < N; ++ky)
      for (int kx = 0; kx < Nh; ++kx) {
        double re = 0, im = 0;
        for (int z = 0; z < N; ++z) {
          const int t = (kz * z) % N;
          size_t o = (((size_t)z * N + ky) * Nh + kx) * 2;
          re += b[o] * cs[t] - b[o + 1] * sn[t];
          im += b[o] * sn[t] + b[o + 1] * cs[t];
        }
        size_t o = (((size_t)kz * N + ky) * Nh + kx) * 2;
        out[o] = re;
        out[o + 1] = im;
      }
}

// ---------------------------------------------------------------------------
// operators: LaplaceKernel::precompute / precompute_m2l (kernel.cpp:1638-1849)
// ---------------------------------------------------------------------------
static void surface(const Operators& o, double r, const V3& c, std::vector<double>& pts) {
  pts.resize((size_t)o.ns * 3);
  for (int i = 0; i < o.ns; ++i)
    for (int k = 0; k < 3; ++k) pts[3 * i + k] = o.surf_unit[3 * i + k] * r + c[k];
}

// G[t][s] = 1/|x_t - y_s| (0 when coincident), get_p2p_matrix (kernel.cpp:1535-1556)
static void p2p_matrix(int nt, const double* xt, int ns, const double* xs, std::vector<double>& G) {
  G.resize((size_t)nt * ns);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < nt; ++t)
    for (int s = 0; s < ns; ++s) {
      double d0 = xt[3 * t] - xs[3 * s], d1 = xt[3 * t + 1] - xs[3 * s + 1], d2 = xt[3 * t + 2] - xs[3 * s + 2];
      double r = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
      G[(size_t)t * ns + s] = r == 0 ? 0.0 : 1.0 / r;
    }
}

void matmul_host(int n, const double* A, const double* B, double* C) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double* c = C + (size_t)i * n;
    for (int j = 0; j < n; ++j) c[j] = 0.0;
    for (int k = 0; k < n; ++k) {
      const double a = A[(size_t)i * n + k];
      const double* b = B + (size_t)k * n;
      for (int j = 0; j < n; ++j) c[j] += a * b[j];
    }
  }
}

static int hash_rel(int i, int j, int k) {
  // LaplaceKernel::hash (3dpp/include/kernel.h:136-141)
  int signs = ((i < 0 ? 1 : 0) << 2) + ((j < 0 ? 1 : 0) << 1) + (k < 0 ? 1 : 0);
  return std::abs(i) * 1000 + std::abs(j) * 100 + std::abs(k) * 10 + signs;
}

// Kernel spectra (kernel.cpp:1721-1769): for each offset n (in units of the
// parent edge 2 r0), the R2C DFT (dft3_r2c) of 1/|p - rel_n| sampled on the
// N^3 convolution grid p = -gsize + (i, j, k) delta (0 where p = rel_n).
void kernel_spectra_host(int N, int noff, const int* offs, double r0, double delta, double gsize, double* gk) {
  const size_t Nf = (size_t)N * N * (N / 2 + 1);
#pragma omp parallel for schedule(dynamic)
  for (int n = 0; n < noff; ++n) {
    std::vector<double> g((size_t)N * N * N);
    const double rel[3] = {offs[3 * n] * r0 * 2, offs[3 * n + 1] * r0 * 2, offs[3 * n + 2] * r0 * 2};
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          const double px = (-gsize + i * delta) - rel[0];
          const double py = (-gsize + j * delta) - rel[1];
          const double pz = (-gsize + k * delta) - rel[2];
          const double r = std::sqrt(px * px + py * py + pz * pz);
          g[((size_t)k * N + j) * N + i] = r == 0 ? 0.0 : 1.0 / r;
        }
    dft3_r2c(N, g.data(), &gk[(size_t)n * Nf * 2]);
  }
}

void build_operators(Operators& o, int P, double r0, int images, const DenseBackend* be) {
  auto matmul = [be](int n, const double* A, const double* B, double* C) {
    if (be && be->matmul)
      be->matmul(n, A, B, C);
    else
      matmul_host(n, A, B, C);
  };
  o.P = P;
  o.r0 = r0;
  o.images = images;
  o.ns = surface_point_num(P);
  o.N = 2 * P - 1;
  o.Nh = o.N / 2 + 1;
  o.Nf = o.N * o.N * o.Nh;
  const int ns = o.ns, N = o.N, Nf = o.Nf;
  // surface points (get_surface_points, surface.cpp:3-47, dir 0)
  o.surf_unit.clear();
  o.surf_ijk.clear();
  for (int i = 0; i < P; ++i)
    for (int j = 0; j < P; ++j)
      for (int k = 0; k < P; ++k)
        if (i == 0 || i == P - 1 || j == 0 || j == P - 1 || k == 0 || k == P - 1) {
          o.surf_ijk.push_back(i);
          o.surf_ijk.push_back(j);
          o.surf_ijk.push_back(k);
          o.surf_unit.push_back(-1.0 + i * 2.0 / (P - 1));
          o.surf_unit.push_back(-1.0 + j * 2.0 / (P - 1));
          o.surf_unit.push_back(-1.0 + k * 2.0 / (P - 1));
        }
  double tb = wall_now();
  auto lap = [&](int k) {
    const double t = wall_now();
    o.build_s[k] = t - tb;
    tb = t;
  };
  std::vector<double> xc, xe, e2c;
  surface(o, r0 * 2.95, V3{0, 0, 0}, xc);
  surface(o, r0 * 1.05, V3{0, 0, 0}, xe);
  p2p_matrix(ns, xc.data(), ns, xe.data(), e2c);
  std::vector<double> U, s, V;
  jacobi_svd(ns, e2c.data(), U, s, V, be, [&]() { lap(0); });
  // pseudo_inverse: drop singular values <= 4e-16 * s_max (mathfunc.cpp:154-169)
  double smax = 0;
  for (double v : s) smax = std::max(smax, std::fabs(v));
  std::vector<double> sinv(ns);
  for (int k = 0; k < ns; ++k) sinv[k] = s[k] > smax * 4e-16 ? 1.0 / s[k] : 0.0;
  o.UT.assign((size_t)ns * ns, 0);
  o.VSinv.assign((size_t)ns * ns, 0);
  for (int i = 0; i < ns; ++i)
    for (int k = 0; k < ns; ++k) {
      o.UT[(size_t)k * ns + i] = U[(size_t)i * ns + k];
      o.VSinv[(size_t)i * ns + k] = V[(size_t)i * ns + k] * sinv[k];
    }
  o.U = U;
  o.V = V;
  o.sinv = sinv;
  o.pinv_up.assign((size_t)ns * ns, 0);
  matmul(ns, o.VSinv.data(), o.UT.data(), o.pinv_up.data());
  o.pinv_down.assign((size_t)ns * ns, 0);
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j) o.pinv_down[(size_t)i * ns + j] = o.pinv_up[(size_t)j * ns + i];
  lap(1);
  // out_k = VSinv (UT G_k) for a batch of child check matrices G_k
  auto chain = [&](std::vector<std::vector<double>>& Gs, std::vector<std::vector<double>>& outs) {
    outs.assign(Gs.size(), std::vector<double>((size_t)ns * ns, 0.0));
    if (be && be->chain) {
      std::vector<const double*> g(Gs.size());
      std::vector<double*> r(Gs.size());
      for (size_t k = 0; k < Gs.size(); ++k) {
        g[k] = Gs[k].data();
        r[k] = outs[k].data();
      }
      be->chain(ns, o.VSinv.data(), o.UT.data(), (int)Gs.size(), g.data(), r.data());
      return;
    }
    std::vector<double> m1((size_t)ns * ns);
    for (size_t k = 0; k < Gs.size(); ++k) {
      matmul(ns, o.UT.data(), Gs[k].data(), m1.data());
      matmul(ns, o.VSinv.data(), m1.data(), outs[k].data());
    }
  };
  // M2M[octant] = VSinv (UT G_child) (kernel.cpp:1660-1668)
  {
    std::vector<std::vector<double>> Gs(8), outs;
    for (int oc = 0; oc < 8; ++oc) {
      V3 cc = child_center(V3{0, 0, 0}, r0, oc);
      std::vector<double> xch;
      surface(o, r0 / 2 * 1.05, cc, xch);
      p2p_matrix(ns, xc.data(), ns, xch.data(), Gs[oc]);
    }
    chain(Gs, outs);
    for (int oc = 0; oc < 8; ++oc) o.m2m[oc].swap(outs[oc]);
  }
  lap(2);
  // image M2M over the 27 children of a 3x3x3 super-cell (kernel.cpp:1671-1683)
  o.m2m_img_sum.assign((size_t)ns * ns, 0);
  o.l2l_img.assign((size_t)ns * ns, 0);
  if (images > 0) {
    std::vector<std::vector<double>> Gs(27), outs;
    for (int oc = 0; oc < 27; ++oc) {
      int kk = oc / 9 - 1, jj = (oc % 9) / 3 - 1, ii = oc % 3 - 1;
      V3 cc{ii * (r0 * 2 / 3.0), jj * (r0 * 2 / 3.0), kk * (r0 * 2 / 3.0)};
      std::vector<double> xch;
      surface(o, r0 / 3 * 1.05, cc, xch);
      p2p_matrix(ns, xc.data(), ns, xch.data(), Gs[oc]);
    }
    chain(Gs, outs);
    for (int oc = 0; oc < 27; ++oc) {
      const std::vector<double>& mi = outs[oc];
      for (size_t e = 0; e < mi.size(); ++e) o.m2m_img_sum[e] += mi[e];
      if (oc == 13)
        for (int i = 0; i < ns; ++i)
          for (int j = 0; j < ns; ++j) o.l2l_img[(size_t)i * ns + j] = mi[(size_t)j * ns + i];
    }
  }
  lap(3);
  // kernel spectra over every non-adjacent child offset (kernel.cpp:1721-1769)
  const int rng = images >= 2 ? 4 : 3;
  std::vector<std::array<int, 3>> offs;
  for (int k = -rng; k <= rng; ++k)
    for (int j = -rng; j <= rng; ++j)
      for (int i = -rng; i <= rng; ++i)
        if (std::abs(i) >= 2 || std::abs(j) >= 2 || std::abs(k) >= 2) offs.push_back({i, j, k});
  std::unordered_map<int, int> gidx;
  for (size_t n = 0; n < offs.size(); ++n) gidx[hash_rel(offs[n][0], offs[n][1], offs[n][2])] = (int)n;
  std::vector<double> gk(offs.size() * (size_t)Nf * 2);
  const double delta = 2 * r0 / (P - 1) * 1.05;
  const double gsize = r0 * 2 * 1.05;
  std::vector<int> offv(offs.size() * 3);
  for (size_t n = 0; n < offs.size(); ++n)
    for (int k = 0; k < 3; ++k) offv[3 * n + k] = offs[n][k];
  if (be && be->spectra)
    be->spectra(N, (int)offs.size(), offv.data(), r0, delta, gsize, gk.data());
  else
    kernel_spectra_host(N, (int)offs.size(), offv.data(), r0, delta, gsize, gk.data());
  lap(4);
  // 8x8 sibling blocks per parent direction (kernel.cpp:1783-1811), stored
  // [d][isrc][itar][f]; adjacent child pairs stay zero.
  o.cc8.assign((size_t)26 * 64 * Nf * 2, 0.0);
  int d = 0;
  std::vector<std::array<int, 3>> dirs;
  for (int k = -1; k <= 1; ++k)
    for (int j = -1; j <= 1; ++j)
      for (int i = -1; i <= 1; ++i)
        if (i || j || k) dirs.push_back({i, j, k});
#pragma omp parallel for schedule(static)
  for (d = 0; d < 26; ++d) {
    for (int isrc = 0; isrc < 8; ++isrc)
      for (int itar = 0; itar < 8; ++itar) {
        // child centres of parents of radius 1: parent offset 2*dir, child +-0.5
        int dx[3];
        const int sb[3] = {(isrc >> 2) & 1, (isrc >> 1) & 1, isrc & 1};
        const int tb[3] = {(itar >> 2) & 1, (itar >> 1) & 1, itar & 1};
        for (int k = 0; k < 3; ++k) dx[k] = 2 * dirs[d][k] + sb[k] - tb[k];
        auto it = gidx.find(hash_rel(dx[0], dx[1], dx[2]));
        if (it == gidx.end()) continue;
        std::memcpy(&o.cc8[(((size_t)d * 8 + isrc) * 8 + itar) * Nf * 2], &gk[(size_t)it->second * Nf * 2],
                    sizeof(double) * Nf * 2);
      }
  }
  // 1x27 image blocks (kernel.cpp:1813-1849), summed over the 27 copies
  o.cc27sum.assign((size_t)26 * Nf * 2, 0.0);
  if (images >= 2) {
    for (d = 0; d < 26; ++d)
      for (int pz = -1; pz <= 1; ++pz)
        for (int py = -1; py <= 1; ++py)
          for (int px = -1; px <= 1; ++px) {
            const int sx = 3 * dirs[d][0] + px, sy = 3 * dirs[d][1] + py, sz = 3 * dirs[d][2] + pz;
            const int g = gidx.at(hash_rel(sx, sy, sz));
            for (int f = 0; f < 2 * Nf; ++f) o.cc27sum[(size_t)d * Nf * 2 + f] += gk[(size_t)g * Nf * 2 + f];
          }
  }
  lap(5);
}

// ---------------------------------------------------------------------------
// operator tables on disk
// ---------------------------------------------------------------------------
namespace {

const char kOpsMagic[8] = {'R', 'T', 'F', 'M', 'M', 'O', 'P', '1'};

struct OpsFields {
  // every table of an operator set, in file order, with its expected length
  template <typename O, typename F>
  static void each(O& o, F&& f) {
    const size_t nn = (size_t)o.ns * o.ns, nf = (size_t)o.Nf;
    f(o.pinv_up, nn);
    f(o.pinv_down, nn);
    f(o.UT, nn);
    f(o.VSinv, nn);
    f(o.U, nn);
    f(o.V, nn);
    f(o.sinv, (size_t)o.ns);
    for (int k = 0; k < 8; ++k) f(o.m2m[k], nn);
    f(o.m2m_img_sum, nn);
    f(o.l2l_img, nn);
    f(o.cc8, (size_t)26 * 64 * nf * 2);
    f(o.cc27sum, (size_t)26 * nf * 2);
    f(o.surf_unit, (size_t)o.ns * 3);
  }
};

struct File {
  FILE* fp;
  explicit File(FILE* f) : fp(f) {}
  ~File() {
    if (fp) fclose(fp);
  }
};

}  // namespace

std::string save_operators(const Operators& ops, const std::string& path) {
  File f(fopen(path.c_str(), "wb"));
  if (!f.fp) return "cannot open " + path + " for writing";
  const Operators& o = ops;
  const int32_t hdr[6] = {o.P, o.images, o.ns, o.N, o.Nh, o.Nf};
  bool ok = fwrite(kOpsMagic, 1, 8, f.fp) == 8 && fwrite(hdr, sizeof(hdr), 1, f.fp) == 1 &&
            fwrite(&o.r0, sizeof(double), 1, f.fp) == 1;
  OpsFields::each(o, [&](const std::vector<double>& v, size_t) {
    const uint64_t len = v.size();
    ok = ok && fwrite(&len, sizeof(len), 1, f.fp) == 1 && (len == 0 || fwrite(v.data(), sizeof(double), len, f.fp) == len);
  });
  const uint64_t li = o.surf_ijk.size();
  ok = ok && fwrite(&li, sizeof(li), 1, f.fp) == 1 &&
       (li == 0 || fwrite(o.surf_ijk.data(), sizeof(int), li, f.fp) == li);
  if (!ok) return "write failed: " + path;
  return "";
}

std::string load_operators(Operators& out, const std::string& path) {
  File f(fopen(path.c_str(), "rb"));
  if (!f.fp) return "cannot open " + path;
  char magic[8];
  int32_t hdr[6];
  Operators o;
  if (fread(magic, 1, 8, f.fp) != 8 || std::memcmp(magic, kOpsMagic, 8) != 0) return "not an operator file: " + path;
  if (fread(hdr, sizeof(hdr), 1, f.fp) != 1 || fread(&o.r0, sizeof(double), 1, f.fp) != 1) return "truncated header";
  o.P = hdr[0];
  o.images = hdr[1];
  o.ns = hdr[2];
  o.N = hdr[3];
  o.Nh = hdr[4];
  o.Nf = hdr[5];
  if (o.P < 2 || o.P > 64 || o.images < 0 || o.ns != surface_point_num(o.P) || o.N != 2 * o.P - 1 ||
      o.Nh != o.N / 2 + 1 || o.Nf != o.N * o.N * o.Nh || !(o.r0 > 0) || !std::isfinite(o.r0))
    return "inconsistent header";
  std::string err;
  OpsFields::each(o, [&](std::vector<double>& v, size_t want) {
    if (!err.empty()) return;
    uint64_t len = 0;
    if (fread(&len, sizeof(len), 1, f.fp) != 1 || len != want) {
      err = "table size does not match P";
      return;
    }
    v.resize(len);
    if (fread(v.data(), sizeof(double), len, f.fp) != len) err = "truncated table";
  });
  if (!err.empty()) return err;
  uint64_t li = 0;
  if (fread(&li, sizeof(li), 1, f.fp) != 1 || li != (uint64_t)o.ns * 3) return "table size does not match P";
  o.surf_ijk.resize(li);
  if (fread(o.surf_ijk.data(), sizeof(int), li, f.fp) != li) return "truncated table";
  char extra;
  if (fread(&extra, 1, 1, f.fp) != 0) return "trailing data";
  out = std::move(o);
  return "";
}

}  // namespace rtfmm_b200
