// Device kernels of the evaluation pass (sm_100a).  Declarations shared by
// rtfmm_kernels.cu and the orchestration in rtfmm_capi.cu.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace rtfmm_b200 {

// Leaf table: one entry per leaf cell.
struct LeafInfo {
  double cx, cy, cz;   // centre
  double r;            // half edge
  double scale;        // 0.5^depth (P2M / L2P operator rescaling)
  int cell;            // cell index
  int boff, bnum;      // bodies in tree order
};

// P2P work item: nt <= W targets of one leaf, W = 1 << lw
// lanes per target group; the 32/W groups of a warp split every source tile
// between them, so a leaf's last few targets do not leave most lanes idle.
struct P2PItem32 {
  int leaf;   // leaf-table index of the target leaf (its source list)
  int boff;   // first target body (tree order)
  int nt;     // targets in this item (1..W)
  int lw;     // log2 W, W in {4, 8, 16, 32}
};

// One P2P list entry (source leaf) of a target leaf, FP32 form.  Both forms
// carry the source's body range so that the kernels read bodies with one
// dependent load.
struct alignas(16) P2PSrc32 {
  float dx, dy, dz;   // c_src + offset - c_tar, for leaf-relative FP32 positions
  int leaf;           // leaf-table index of the source leaf
  int self;           // source == target with zero offset (mask r == 0)
  int boff, bnum;     // source bodies (tree order)
  int pad;
};
struct P2PSrc64 {
  double ox, oy, oz;  // periodic offset added to the source positions
  int leaf;
  int self;
  int boff, bnum;     // source bodies (tree order)
};

// Batched FP64 operator application (see k_apply_f64).
struct ApplyBatch {
  const double* A;      // input vectors, row stride ns
  const int* inrow;     // rows*S input row indices (-1 = zero vector)
  const double* B;      // groups x S x ns x ns operator stack, row-major [s][j][n]
  const int* outrow;    // output row indices
  const double* scale;  // per-row scale (nullptr = 1)
  const int* group_off; // groups+1 row offsets
  double* C;            // output vectors, row stride ns
  int groups, S, ns, beta;
  int max_rows;         // rows of the largest group (grid sizing)
};

// Launch helpers (all asynchronous on `st`; return cudaGetLastError()).
// body_leaf[b] = leaf of tree-order body b (the leaves partition [0, n))
cudaError_t launch_body_leaf(const LeafInfo* leaves, int nleaf, int n, int* body_leaf, cudaStream_t st);
cudaError_t launch_prep32(const double4* body64, const int* body_leaf, const LeafInfo* leaves,
                          float4* body32, int n, cudaStream_t st);
cudaError_t launch_p2p32(const float4* body32, const P2PItem32* items, int nitems, const int* list_off,
                         const P2PSrc32* list, double* phi, double* grad, cudaStream_t st);
cudaError_t launch_p2p64(const double4* body64, const P2PItem32* items, int nitems, const int* list_off,
                         const P2PSrc64* list, double* phi, double* grad, cudaStream_t st);
// Close-pair refinement of the FP32 P2P: per-target counts of the pairs
// closer than a fraction of their leaves (cnt[t], tree order), their list
// (source body, list entry) at pairs[off[t]...], and the per-pass fix that
// replaces their FP32 terms in phi / grad (P2P outputs) by FP64 ones.
cudaError_t launch_close_count(const float4* body32, const P2PItem32* items, int nitems, const int* list_off,
                               const P2PSrc32* list, const LeafInfo* leaves, int* cnt, cudaStream_t st);
cudaError_t launch_close_emit(const float4* body32, const P2PItem32* items, int nitems, const int* list_off,
                              const P2PSrc32* list, const LeafInfo* leaves, const int* off, int2* pairs,
                              cudaStream_t st);
// cycle > 0: periodic (nearest image); 0: free space
cudaError_t launch_close_fix(const double4* body64, const float4* body32, const P2PSrc32* list, const int* off,
                             const int2* pairs, int n, double cycle, double* phi, double* grad, cudaStream_t st);
// off = exclusive prefix sum of cnt (n values); tmp == nullptr: *tmp_bytes
// = the scratch it needs
cudaError_t launch_count_scan(const int* cnt, int* off, int n, void* tmp, size_t* tmp_bytes, cudaStream_t st);
// newton: Newton steps of the FP64 reciprocal square root (1: ~1e-13, for
// the FP32-mixed form; 2: full FP64)
cudaError_t launch_p2m_check(const double4* body64, const LeafInfo* leaves, int nleaf,
                             const double* surf_unit, int ns, double* out, cudaStream_t st, int newton = 2);
cudaError_t launch_apply(const ApplyBatch& b, cudaStream_t st);
// q[parent] = sum of Y[child] over the parent's children; `list` holds
// (parent, coff, cnum) triplets
cudaError_t launch_sum_children(const int* list, int nparents, const double* Y, int ns, double* q,
                                cudaStream_t st);
// FFT-M2L spectra are frequency-major: Q[f][src][slot], Pk[f][tar][slot],
// G[f][d][isrc*8+itar] (complex, interleaved re/im).
// items hold 10 ints per block: parent, first slot, child cell of each of the
// sp slots of the group (-1 = absent); sp from m2l_up_slots / m2l_down_slots.
template <typename T>
int m2l_up_slots(int P);
template <typename T>
int m2l_down_slots(int P);
template <typename T>
cudaError_t launch_m2l_up(const double* q_equiv, const int* items, int nitems, const int* surf_ijk,
                          const double* twiddle, int P, int ns, int nsrc, int sp, T* Q, cudaStream_t st);
template <typename T>
cudaError_t launch_m2l_hadamard8(const T* Q, const T* G, const int* tsrcT /*[26][ntar]*/, int ntar, int nsrc,
                                 int Nf, T* Pk, cudaStream_t st);
// G (frequency-major, the Hadamard's layout) from cc8 [d][pair][f] (device)
template <typename T>
cudaError_t launch_g8_layout(const double* cc8, int Nf, T* G, cudaStream_t st);
cudaError_t launch_m2l_hadamard27(const double* Q, const double* G27 /*[d][f]*/, const int* tsrc /*[ntar][26]*/,
                                  int ntar, int nsrc, int Nf, double* Pk, cudaStream_t st);
template <typename T>
cudaError_t launch_m2l_down(const T* Pk, const int* items, const double* tscale, int nitems,
                            const int* surf_ijk, const double* twiddle, int P, int ns, int ntar, int sp,
                            double* p_check, cudaStream_t st);
cudaError_t launch_l2p_eval(const double4* body64, const LeafInfo* leaves, int nleaf,
                            const double* surf_unit, int ns, const double* q_down, double* phi,
                            double* grad, cudaStream_t st, int newton = 2);
// sums of q x, q y, q z and q into partial[4 * kDipoleBlocks + 0..3]; partial
// holds kDipoleScratch doubles (per-block sums, then the totals)
constexpr int kDipoleBlocks = 256;
constexpr int kDipoleScratch = 4 * kDipoleBlocks + 4;
cudaError_t launch_dipole(const double4* body64, int n, double* partial, cudaStream_t st);
// adjoint: weights into the tree-order bodies (charges kept in qsave), the
// charges back, and dL/dx = w grad(phi_q) + q grad(psi_w) in input order
cudaError_t launch_swap_charges(double4* body64, const double* w, const int64_t* perm, int n, double* qsave,
                                cudaStream_t st);
cudaError_t launch_restore_charges(double4* body64, const double* qsave, int n, cudaStream_t st);
// new charges (input order) into bodies whose positions are on the device
cudaError_t launch_set_charges(double4* body64, const double* q, const int64_t* perm, int n, cudaStream_t st);
cudaError_t launch_adj_combine(const int64_t* perm, const double* w, const double* qsave, const double* grad_q,
                               const double* grad_w, int n, double* dLdx, cudaStream_t st);
// a sharded pass's exchange: leaf rows of v (nrow rows, stride ns) into a
// leaf-ordered buffer (scatter = false; rows of leaves with own[l] == 0 are
// zero, own null keeps all) or back (scatter = true)
cudaError_t launch_leaf_rows(double* v, int nrow, const int* cells, const char* own, int nleaf, int ns,
                             double* buf, bool scatter, cudaStream_t st);
// dipole: 0 none, 1 the reference's per-body form, 2 the surface term's
// potential; centre: the box centre (3), the dipole's origin
cudaError_t launch_post(const double* phi_far, const double* grad_far, const double* phi_near,
                        const double* grad_near, const double4* body64, const int64_t* perm, int n,
                        const double* dipole_partial, double coef, int dipole, const double* centre,
                        double out_scale, double* out_phi, double* out_grad, cudaStream_t st);
cudaError_t launch_gather_bodies(const double* x_in, const double* q_in, const int64_t* perm, int n,
                                 double4* body64, cudaStream_t st);

}  // namespace rtfmm_b200
