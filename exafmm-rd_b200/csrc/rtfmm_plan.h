// Host-side plan of one FMM evaluation: octree, interaction lists and
// operator tables, in the layouts the device kernels consume.
#pragma once

#include <array>
#include <functional>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace rtfmm_b200 {

using V3 = std::array<double, 3>;

// One octree cell; the fields and their meaning follow Cell3
// (3dpp/include/tree.h:9-47).  octant 13 marks the single central child of an
// image super-cell (and the root).
struct Cell {
  int octant;
  int depth;
  double r;
  V3 x;
  int coff, cnum;   // children: contiguous range
  int boff, bnum;   // bodies in tree order: contiguous range
};

struct P2PEntry {
  int src;   // source leaf
  V3 off;    // periodic offset added to the source positions
};

struct M2LEntry {
  int src;
  V3 off;
  int single;  // is_single_parent (image-level 1x27 interaction)
};

// Operator tables for one (P, images) pair, built at the root radius r0 and
// rescaled at use (kernel.cpp:1638-1849).
struct Operators {
  int P = 0, images = -1;
  double r0 = 0;
  int ns = 0;             // surface points
  int N = 0, Nh = 0, Nf = 0;  // conv grid edge, half-spectrum edge, frequencies
  std::vector<double> pinv_up;     // ns x ns: V S^-1 U^T of the upward e2c
  std::vector<double> pinv_down;   // ns x ns: U S^-1 V^T (its transpose)
  std::vector<double> UT, VSinv;   // factors as the reference keeps them
  std::vector<double> U, V, sinv;  // e2c = U diag(s) V^T (row-major), sinv = pseudo-inverted s
  std::vector<double> m2m[8];      // ns x ns each
  std::vector<double> m2m_img_sum; // sum of the 27 image M2M matrices
  std::vector<double> l2l_img;     // M2M_img[13]^T
  std::vector<double> cc8;         // [d][isrc][itar][f] complex (re,im)
  std::vector<double> cc27sum;     // [d][f] complex: sum of the 27 image spectra
  std::vector<double> surf_unit;   // ns x 3 unit-cube surface points
  std::vector<int> surf_ijk;       // ns x 3 lattice coordinates (x,y,z)
  // wall seconds of the build: SVD (surfaces, e2c, sweeps), Gram-Schmidt and
  // pseudo-inverse, M2M products, image products, kernel spectra, the 8x8 and
  // 1x27 blocks
  double build_s[6] = {0, 0, 0, 0, 0, 0};
};

// Per-cell lists indexed by cell: a vector of vectors that reads like the
// map it replaces (lists[c] grows the index; iteration visits the cells with
// a non-empty list in cell order as (first = cell, second = list)).
template <typename E>
struct CellLists {
  std::vector<std::vector<E>> v;
  std::vector<E>& operator[](int c) {
    if (c >= (int)v.size()) v.resize((size_t)c + 1);
    return v[(size_t)c];
  }
  const std::vector<E>& at(int c) const {
    static const std::vector<E> empty;
    return c < (int)v.size() ? v[(size_t)c] : empty;
  }
  void clear() { v.clear(); }
  size_t size() const {  // cells with a non-empty list
    size_t k = 0;
    for (const auto& l : v) k += !l.empty();
    return k;
  }
  struct Item {
    int first;
    const std::vector<E>& second;
  };
  struct Iter {
    const CellLists* L;
    int i;
    void skip() {
      while (i < (int)L->v.size() && L->v[(size_t)i].empty()) ++i;
    }
    Item operator*() const { return {i, L->v[(size_t)i]}; }
    Iter& operator++() {
      ++i;
      skip();
      return *this;
    }
    bool operator!=(const Iter& o) const { return i != o.i; }
  };
  Iter begin() const {
    Iter it{this, 0};
    it.skip();
    return it;
  }
  Iter end() const { return Iter{this, (int)v.size()}; }
};

struct Args {
  int P = 4, ncrit = 16, images = 0;
  double cycle = 6.283185307179586;
  V3 x{0, 0, 0};
  int dipole_correction = 1, divide_4pi = 0, precision = 0;
  unsigned stages = 3;
  int device = 0;
};

struct Plan {
  Args args;
  double r0 = 0;
  int64_t n = 0;
  std::vector<double> x, q;        // bodies in tree order (x: n*3)
  std::vector<int64_t> perm;       // perm[i] = input index of tree-order body i
  std::vector<Cell> cells;         // tree cells, then image cells
  int ntree = 0;                   // cells before the image super-cells
  int dmin = 0, dmax = 0;
  CellLists<P2PEntry> p2p;  // by target cell
  CellLists<M2LEntry> m2l;  // by target parent
  int64_t n_p2p = 0, n_m2l = 0;
};

// Tree and lists (exact restatement of the reference's algorithms).
std::string build_tree(Plan& plan, const double* x, const double* q);
void traverse(Plan& plan);  // = traverse_begin, traverse_p2p, traverse_finish

// One root frame of the P2P dual-tree walk: (target, source, target parent,
// source parent) and the periodic offset of the walk.
struct WalkRoot {
  int tc, sc, tcp, scp;
  V3 off;
};
// Clears the lists, adds the depth -1 image super-cell (images >= 1) and
// returns the walk's root frames, one per periodic offset, in walk order.
std::vector<WalkRoot> traverse_begin(Plan& plan);
// The P2P lists by the dual-tree walk from the roots (horizontal_origin,
// traverser.cpp:70-176), on the host.
void traverse_p2p(Plan& plan, const std::vector<WalkRoot>& roots);
// The M2L parent map, the deeper image cells and the list counts.
void traverse_finish(Plan& plan);


// Dense kernels of the operator build that another backend (the GPU) may
// run instead of the host: the Jacobi sweeps (on W, the n columns of A, and
// Vc, m x m, column-major, m = n rounded up to even) and C = A B (n x n,
// row-major).  A backend gives the host's results bit for bit.
struct DenseBackend {
  std::function<void(int n, std::vector<double>& W, std::vector<double>& Vc)> jacobi_sweeps;
  std::function<void(int n, const double* A, const double* B, double* C)> matmul;
  // out[k] = A (B G[k]) for k < nG, each product as matmul
  std::function<void(int n, const double* A, const double* B, int nG, const double* const* G, double* const* out)>
      chain;
  // as kernel_spectra_host and reorthogonalize_host
  std::function<void(int N, int noff, const int* offs, double r0, double delta, double gsize, double* gk)> spectra;
  std::function<void(int n, double* Q)> reorthogonalize;
};

// Operator tables.
void build_operators(Operators& ops, int P, double r0, int images, const DenseBackend* be = nullptr);
// The tables as a versioned binary file (native byte order) and back; ""
// on success, else what is wrong (a load checks every size against P).
std::string save_operators(const Operators& ops, const std::string& path);
std::string load_operators(Operators& ops, const std::string& path);

// Dense helpers.  The one-sided Jacobi SVD pairs columns by a round-robin
// tournament: jacobi_pairs lists (p, q), p < q, for each of the m - 1
// rounds of a sweep (m/2 pairs a round; q >= n is the padding column);
// sweeps end when every pair's |gamma|/sqrt(alpha beta) is below kJacobiTol
// or after kJacobiMaxSweeps.  The inner products alpha, beta, gamma of a pair
// are summed as a 32-lane warp sums them (jacobi_dots), so that the GPU
// sweeps give the same rotations bit for bit.
constexpr double kJacobiTol = 1e-15;
constexpr int kJacobiMaxSweeps = 40;
std::vector<int> jacobi_pairs(int n);
void jacobi_dots(int n, const double* wp, const double* wq, double& alpha, double& beta, double& gamma);
void jacobi_sweeps_host(int n, std::vector<double>& W, std::vector<double>& Vc);
// Gram-Schmidt (two passes) of the rows of Q (n x n, row-major) in order
void reorthogonalize_host(int n, double* Q);
// gk[n] (N*N*(N/2+1) complex) = DFT of 1/|p - 2 r0 offs[n]| on the grid
// p = -gsize + (i, j, k) delta, i, j, k < N
void kernel_spectra_host(int N, int noff, const int* offs, double r0, double delta, double gsize, double* gk);
// after_sweeps (if set) runs when the sweeps are done
void jacobi_svd(int n, const double* A, std::vector<double>& U, std::vector<double>& s, std::vector<double>& V,
                const DenseBackend* be = nullptr, const std::function<void()>& after_sweeps = nullptr);
// C = A B, each C[i][j] summed over k in order (multiply, then add)
void matmul_host(int n, const double* A, const double* B, double* C);
void dft3_r2c(int N, const double* in, double* out);  // out: N*N*(N/2+1) complex

inline int surface_point_num(int p) { return 6 * (p - 1) * (p - 1) + 2; }

}  // namespace rtfmm_b200
