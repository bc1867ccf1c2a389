/*
 * rtfmm_b200 -- C ABI of the B200 (sm_100a) periodic kernel-independent
 * Laplace FMM evaluation pass.
 *
 * The reference (mumairsadiq/exafmm-rd, variant 3dpp) has no FFI: its
 * interface is the C++ driver class and its argument struct.  Each entry
 * point below replaces one piece of that interface; the comment on each names
 * the reference interface it replaces (path:line inside the reference
 * project).  All pointers are plain host pointers unless the name says
 * "_device"; sizes are element counts.  Nothing here allocates memory the
 * caller must free, and no call ever exits the process: every function
 * returns an rtfmm_status and rtfmm_b200_last_error() describes the last
 * failure of the calling thread.
 *
 * Units and conventions follow the reference: the kernel is 1/r (1/(4 pi r)
 * when divide_4pi is set), `grad` is the gradient of the potential (the
 * reference's Body3::f, 3dpp/include/body.h:8-15), and outputs are in the
 * caller's input order (the reference re-sorts by idx, 3dpp/src/fmm.cpp:80).
 */
#ifndef RTFMM_B200_H
#define RTFMM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rtfmm_status {
  RTFMM_OK = 0,
  RTFMM_EINVAL = 1,   /* bad argument (sizes, P, ncrit, NaN/Inf inputs, ...) */
  RTFMM_ENOMEM = 2,   /* host or device allocation failed                   */
  RTFMM_ECUDA = 3,    /* a CUDA runtime call or kernel launch failed         */
  RTFMM_ESTATE = 4,   /* call out of order (e.g. evaluate before setup)      */
  RTFMM_ENOTSUP = 5,  /* option not supported by this build                  */
  RTFMM_ETIMEOUT = 6  /* reserved for a bounded wait that gave up; no call of
                         this build returns it (no kernel waits on another
                         block, stream or GPU)                                */
} rtfmm_status;

/* Arithmetic of the evaluation pass. */
typedef enum rtfmm_precision {
  RTFMM_FP64 = 0,        /* every stage in FP64                                  */
  RTFMM_FP32_MIXED = 1   /* P2P and, for P <= 8, the 8x8 FFT-M2L in FP32 with FP64
                            accumulation; surface operators, image levels, outputs
                            in FP64.  For P >= 10 the FFT-M2L stays FP64: its FP32
                            rounding, through operators of condition ~1e16, costs
                            3e-5 (uniform) to 3e-4 (lattice) in the gradient   */
} rtfmm_precision;

/* Stage mask bits for rtfmm_args.stages (all set = the full pass). */
#define RTFMM_STAGE_NEAR 1u   /* P2P                                  */
#define RTFMM_STAGE_FAR  2u   /* P2M, M2M, M2L, L2L, L2P              */
#define RTFMM_STAGE_ALL  3u
/* Diagnostic bit: run P2P after the far field on one stream (no overlap), so
 * that per-stage times are those of each stage alone. */
#define RTFMM_STAGE_SERIAL 4u
/* Diagnostic bit: record per-stage events (rtfmm_b200_stage_times).  Without
 * it, and without RTFMM_STAGE_SERIAL, a forward pass is captured as a CUDA
 * graph on first use and replayed by every later call on the same device
 * tables; rtfmm_b200_stage_times then reports zeros. */
#define RTFMM_STAGE_TIMED 8u

/*
 * Run parameters.  Replaces rtfmm::Argument (3dpp/include/argument.h:11-45,
 * 3dpp/src/argument.cpp:7-70): same field names and meaning; `r` is derived
 * as cycle/2 and the box centre is `x` (the reference fixes it at the origin,
 * argument.cpp:61-62).
 */
typedef struct rtfmm_args {
  int P;                  /* surface points per edge (expansion order), >= 2      */
  int ncrit;              /* a cell splits while it holds more bodies than this   */
  int images;             /* periodic image levels (0 = free space)               */
  double cycle;           /* period / root cell edge                              */
  double x[3];            /* root cell centre                                     */
  int dipole_correction;  /* 0 none; 1 the reference's dipole correction
                             (kernel.cpp:1580-1596): grad -= c mu, phi_i -=
                             c |mu|^2 / (N q_i); 2 the same gradient with the
                             surface term's potential phi_i -= c mu.(x_i - x).
                             mu = sum q (x - x) about the centre x,
                             c = 4 pi / (3 cycle^3)                          */
  int divide_4pi;         /* scale outputs by 1/(4 pi)                            */
  int precision;          /* rtfmm_precision                                      */
  unsigned stages;        /* RTFMM_STAGE_* mask; 0 means RTFMM_STAGE_ALL          */
  int device;             /* CUDA device ordinal                                  */
} rtfmm_args;

typedef struct rtfmm_fmm rtfmm_fmm;

/* Fills `a` with the reference's defaults (argument.cpp:11-31): P=4,
 * ncrit=16, images=0, cycle=2*pi, dipole_correction=1, divide_4pi=0, plus
 * precision=FP64, stages=ALL, device=0. */
void rtfmm_b200_default_args(rtfmm_args* a);

/* Creates a solver.  Replaces LaplaceFMM::LaplaceFMM(const Bodies3&,
 * const Argument&) (3dpp/include/fmm.h:12-16, 3dpp/src/fmm.cpp:7-11) minus the
 * body copy, which moves to rtfmm_b200_setup.  Touches no GPU. */
int rtfmm_b200_create(const rtfmm_args* args, rtfmm_fmm** out);

/* Releases the solver and every buffer it owns (host and device). */
int rtfmm_b200_destroy(rtfmm_fmm* fmm);

/*
 * Host-side set-up for one body set: builds the adaptive octree
 * (Tree::build_nonuniform_octree, 3dpp/src/tree.cpp:102-188), the P2P and
 * M2L lists with the periodic image cells (Traverser::traverse,
 * 3dpp/src/traverser.cpp:19-68) and the operator tables
 * (LaplaceKernel::precompute / precompute_m2l, 3dpp/src/kernel.cpp:1638-1849;
 * kept by the handle across calls and shared with other handles of the same
 * P, images and cycle through a process-wide cache).
 * This is LaplaceFMM::solve up to its hot block (fmm.cpp:15-49).  x is n*3
 * (x0,y0,z0,x1,...), q is n.  Touches no GPU.
 */
int rtfmm_b200_setup(rtfmm_fmm* fmm, int64_t n, const double* x, const double* q);

/*
 * rtfmm_b200_setup for bodies already in device memory (x_dev n*3, q_dev n,
 * on the handle's device).  The octree is built on the GPU (path keys, a
 * radix sort, one split pass per level) and equals rtfmm_b200_setup's tree
 * and body order exactly; a tree deeper than 21 levels is built on the host
 * instead.  The lists, operators and tables follow as in rtfmm_b200_setup,
 * then the device tables are uploaded and the bodies gathered into tree
 * order on the device, so rtfmm_b200_evaluate_device and
 * rtfmm_b200_forward_device can run at once (no rtfmm_b200_upload).  Host
 * copies of x and q are kept for the host-buffer entry points.  Same error
 * codes as rtfmm_b200_setup.
 */
int rtfmm_b200_setup_device(rtfmm_fmm* fmm, int64_t n, const double* x_dev, const double* q_dev);

/*
 * The evaluation pass with host buffers: copies q (and, on the first call
 * after setup, the positions the tree was built on; they then stay on the
 * device) to the device, runs P2M, M2M, M2L, L2L, L2P and P2P
 * (the hot block, 3dpp/src/fmm.cpp:51-60), then the dipole correction, the
 * 1/(4 pi) scaling and the re-sort (fmm.cpp:75-80) on the device, and copies
 * phi (n) and grad (n*3) back.  q may be NULL to reuse the charges given to
 * setup.
 */
int rtfmm_b200_evaluate(rtfmm_fmm* fmm, const double* q, double* phi, double* grad);

/* setup + evaluate: replaces LaplaceFMM::solve() (3dpp/src/fmm.cpp:13-81).
 * From 65536 bodies the set-up runs on the GPU (the bodies are copied to the
 * device and rtfmm_b200_setup_device builds the tree, lists and P2P tables,
 * the same plan bit for bit as rtfmm_b200_setup); below that, and on a
 * sharded handle, on the host. */
int rtfmm_b200_solve(rtfmm_fmm* fmm, int64_t n, const double* x, const double* q,
                     double* phi, double* grad);

/*
 * The evaluation pass on device-resident data: the bodies uploaded by the
 * last evaluate/upload call, results left in device memory.  Returns the
 * pass time in milliseconds measured with CUDA events on the solver's own
 * stream (`ms` may be NULL).  For throughput measurement.
 */
int rtfmm_b200_upload(rtfmm_fmm* fmm);
int rtfmm_b200_evaluate_device(rtfmm_fmm* fmm, float* ms);

/*
 * The evaluation pass on device buffers: q_dev (n charges, input order; NULL
 * keeps the bodies' current charges) replaces the charges of the bodies on
 * the device, and phi_dev (n) / grad_dev (n*3), device pointers in input
 * order (either may be NULL), receive the results.  Needs rtfmm_b200_upload
 * (or an evaluate) first; charges are not checked for NaN/Inf.  *ms (may be
 * NULL) receives the pass time; returns when the results are complete.
 * Together with rtfmm_b200_adjoint_device this is a forward/backward step
 * without host copies.
 */
int rtfmm_b200_forward_device(rtfmm_fmm* fmm, const double* q_dev, double* phi_dev, double* grad_dev, float* ms);

/* Copies the outputs of the last device pass to the host (input order). */
int rtfmm_b200_download(rtfmm_fmm* fmm, double* phi, double* grad);

/*
 * Adjoint of the evaluation pass (no reference counterpart: the reference
 * has no gradient code).  For L = sum_i w_i phi_i it returns dL/dq (n) and
 * dL/dx (n*3) by applying the transposed operator chain P2P^T, L2P^T, L2L^T,
 * M2L^T (conjugated kernel spectra), M2M^T, P2M^T; upward coefficients are
 * recomputed.  Works on the bodies and charges given to setup (w is n, in
 * input order; dLdq n, dLdx n*3, either may be NULL).  For a quadratic L
 * (w depending on q) the caller adds the explicit term.  The divide_4pi
 * scaling applies; the dipole correction is excluded.
 */
int rtfmm_b200_adjoint(rtfmm_fmm* fmm, const double* w, double* dLdq, double* dLdx);

/*
 * The adjoint on device memory (no reference counterpart): w_dev (n),
 * dLdq_dev (n) and dLdx_dev (n*3) are device pointers on the handle's
 * device, in input order (the outputs may be NULL).  It works on the bodies
 * and charges the device holds (those of the last upload, evaluate or solve)
 * and needs rtfmm_b200_upload (or an evaluate) first.  When the last pass
 * was a forward pass of these charges without the dipole correction, its
 * gradient is reused and the call runs one transposed pass; otherwise it
 * runs two.  Weights are not checked for NaN/Inf.  *ms (may be NULL)
 * receives the device time of the call; it returns when the results are
 * complete.  Afterwards rtfmm_b200_download returns intermediate fields.
 */
int rtfmm_b200_adjoint_device(rtfmm_fmm* fmm, const double* w_dev, double* dLdq_dev, double* dLdx_dev,
                              float* ms);

/* ---- The pass sharded over ranks (one process per GPU) ----
 *
 * No counterpart in the reference (it runs on one node with OpenMP; the
 * pass it shards is LaplaceFMM::solve's hot block, fmm.cpp:51-60).  Every
 * rank sets up the same bodies; rank r then computes the outputs of the
 * leaves whose first body (in tree order) lies in its share
 * [r n / R, (r + 1) n / R) of the bodies, and the cells above them:
 *
 *   rtfmm_b200_shard(h, r, R);              before rtfmm_b200_setup (host
 *                                           bodies; setup_device is refused)
 *   rtfmm_b200_setup(...); rtfmm_b200_upload(h);
 *   per pass:
 *     rtfmm_b200_shard_upward(h, xbuf);     P2M of this rank's leaves, every
 *                                           leaf's q_equiv row into xbuf
 *                                           (rows of other ranks' leaves 0);
 *                                           P2P starts, on its own stream
 *     all-reduce (sum) xbuf over the ranks  the one exchange (NCCL / gloo)
 *     rtfmm_b200_shard_downward(h, xbuf, phi, grad, &ms);
 *                                           M2M on the whole tree, M2L, L2L,
 *                                           L2P of this rank's cells, post
 *
 * xbuf is device memory of nleaf * num_surf doubles
 * (rtfmm_b200_shard_sizes).  phi / grad (device, input order, n and 3n)
 * hold this rank's bodies (rtfmm_b200_shard_bodies gives their input
 * indices); other entries are not computed.  The outputs of a body equal
 * the unsharded pass's bit for bit.  The whole-pass entry points and the
 * adjoint return RTFMM_ESTATE on a sharded handle; rtfmm_b200_shard(h, 0,
 * 1) undoes sharding (at the next set-up). */
int rtfmm_b200_shard(rtfmm_fmm* fmm, int rank, int nranks);
int rtfmm_b200_shard_sizes(rtfmm_fmm* fmm, int64_t* nbodies, int64_t* xbuf_doubles);
int rtfmm_b200_shard_bodies(rtfmm_fmm* fmm, int64_t* idx, int64_t cap);
int rtfmm_b200_shard_upward(rtfmm_fmm* fmm, double* xbuf_dev);
int rtfmm_b200_shard_downward(rtfmm_fmm* fmm, const double* xbuf_dev, double* phi_dev, double* grad_dev,
                              float* ms);

/*
 * Accuracy references on sampled targets, FP64 on the GPU (device `device`),
 * for sizes where a CPU sum would take hours.  x is n*3, q is n (host),
 * targets holds nt body indices; phi (nt) and grad (nt*3) receive the
 * potential and its gradient at those bodies, without 1/(4 pi) and without
 * a dipole term.  Both allocate and free their own device memory.
 *
 * rtfmm_b200_ewald_sampled replaces EwaldSolver (3dpp/include/ewald.h,
 * 3dpp/src/ewald.cpp): alpha = ksize/cycle, real-space sum over r < cycle/2,
 * reciprocal sum over the (2 ksize + 1)^3 - 1 integer waves, self term;
 * ksize in [1, 16] (the reference's default is 11).  The real-space image of
 * a pair is the per-particle minimum image (the converged sum); the
 * reference takes one image per pair of leaf cells, which can drop pairs
 * that are close across the periodic boundary.  rtfmm_b200_direct_sampled is
 * the free-space direct sum over all bodies.
 */
int rtfmm_b200_ewald_sampled(int device, int64_t n, const double* x, const double* q, double cycle, int ksize,
                             int64_t nt, const int64_t* targets, double* phi, double* grad);
int rtfmm_b200_direct_sampled(int device, int64_t n, const double* x, const double* q, int64_t nt,
                              const int64_t* targets, double* phi, double* grad);

/* Per-stage device times of the last pass, in ms, in this order:
 * prep, P2M, M2M, M2L_up, M2L_hadamard, M2L_down, L2L, L2P, P2P, post.
 * Writes min(cap, 10) values; returns the number of stages. */
int rtfmm_b200_stage_times(rtfmm_fmm* fmm, double* ms, int cap);

/* Counters of the last pass: kernels launched by this library. */
int rtfmm_b200_launch_count(rtfmm_fmm* fmm, int64_t* launches);

/* Writes L2-sized garbage on the solver's stream (cache flush between timed
 * passes). */
int rtfmm_b200_flush_l2(rtfmm_fmm* fmm);

/* ---- introspection (host data after setup; used by parity tests) ---- */

/* Set-up wall times of the last set-up, in seconds: s[0] octree, s[1]
 * interaction lists, s[2] operator tables (0 when the handle's cached tables
 * were reused), s[3] host tables of the pass, s[4] the whole setup call,
 * s[5] the upload of the device tables (done by rtfmm_b200_setup_device, or
 * by the first upload/evaluate after rtfmm_b200_setup).  s[6..11] split s[2]
 * when the tables were built in this set-up (else 0): the SVD (surfaces,
 * check matrix, Jacobi sweeps), the Gram-Schmidt pass and pseudo-inverse,
 * the M2M products, the image products, the kernel spectra, and their 8x8
 * and 1x27 blocks.  The reference times the same phases separately from the
 * evaluation (3dpp/src/fmm.cpp:13-50).  Writes min(cap, 12) values. */
int rtfmm_b200_setup_times(rtfmm_fmm* fmm, double* s, int cap);

/* Tree and list sizes.  info[0..11] = ncell (incl. image cells), nleaf,
 * depth_min, depth_max, n_p2p_entries, n_m2l_parents, n_m2l_entries,
 * num_surf, P2P body pairs (sum over list entries of n_target * n_source),
 * 8x8 M2L (target, direction) pairs, 8x8 M2L source parents, 8x8 M2L
 * target parents, and (FP32-mixed form, after its first pass on the
 * set-up's positions; else 0) the P2P body pairs whose FP32 terms every pass
 * replaces by FP64 ones (pairs closer than 1/8 of the larger of their
 * leaves' half edges).  Returns the number of values available (13). */
int rtfmm_b200_info(rtfmm_fmm* fmm, int64_t* info, int cap);

/* Cells in the reference's order (Cell3, 3dpp/include/tree.h:9-47):
 * ints[7*c..] = octant, depth, crange.offset, crange.number, brange.offset,
 * brange.number, 0; reals[4*c..] = r, x, y, z.  Either pointer may be NULL. */
int rtfmm_b200_get_cells(rtfmm_fmm* fmm, int32_t* ints, double* reals);

/* perm[i] = input index of the i-th body in tree order. */
int rtfmm_b200_get_perm(rtfmm_fmm* fmm, int64_t* perm);

/* P2P lists (Traverser::P2P_map, traverser.cpp:70-148): entry e is
 * (target leaf, source leaf) = ints[2e], ints[2e+1] with source offset
 * off[3e..3e+2]. */
int rtfmm_b200_get_p2p(rtfmm_fmm* fmm, int32_t* ints, double* off);

/* The pass's P2P lists by target leaf, every entry leaf to leaf (a
 * reference pair of a leaf and a non-leaf cell expanded into the leaves
 * beneath it, in first-body order): list_off (nleaf + 1), src_leaf and the
 * periodic offset off (3 per entry), leaves numbered in cell order.  cap is
 * the room in src_leaf / off (list_off[nleaf] entries are written); with
 * both null only list_off is written (a size query). */
int rtfmm_b200_get_leaf_lists(rtfmm_fmm* fmm, int32_t* list_off, int32_t* src_leaf, double* off, int64_t cap);

/* M2L parent map (Traverser::M2L_parent_map, traverser.cpp:234-282 and
 * 43-64): entry e is (target, source, is_single_parent) = ints[3e..3e+2]
 * with offset off[3e..3e+2]. */
int rtfmm_b200_get_m2l(rtfmm_fmm* fmm, int32_t* ints, double* off);

/* Per-cell surface vectors after the last pass (device -> host):
 * which = 0 for q_equiv, 1 for p_check; out is ncell*num_surf. */
int rtfmm_b200_get_cell_vectors(rtfmm_fmm* fmm, int which, double* out);

/* Operator tables (host FP64), for comparison with the reference's
 * LaplaceKernel members (3dpp/include/kernel.h:197-229):
 * which = 0: pinv of the upward equivalent->check operator (ns*ns),
 *         1: M2M for octants 0..7 (8*ns*ns),  2: sum of the 27 image M2M
 *            (ns*ns),  3: 8x8 kernel spectra (26*8*8*Nfreq complex, as
 *            interleaved re,im),  4: U and 5: V S^-1 of the SVD
 *            e2c = U S V^T with the pseudo-inverted S (UT_p2m_precompute^T
 *            and VSinv_p2m_precompute, kernel.h:197-200), row-major ns*ns,
 *         6: 1x27 image kernel spectra summed over the 27 copies
 *            (26*Nfreq complex),  7: the centre image L2L (ns*ns). */
int rtfmm_b200_get_operator(rtfmm_fmm* fmm, int which, double* out, int64_t cap);

/* ---- P2M that allocates no device memory ----
 *
 * No counterpart in the reference.  For callers that cannot call cudaMalloc,
 * for example code running under another framework's device-memory pool,
 * where an allocation outside the pool would escape its accounting or fail
 * against its limits.  The call computes the P2M stage for a batch of leaves
 * (check-surface potentials of the leaves' bodies, then
 * q_equiv = 0.5^depth * (V S^-1) (U^T p_check)) exactly as the evaluation
 * pass does, and allocates nothing: inputs and the output are the caller's
 * device buffers, and its scratch is one fixed array of
 * RTFMM_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds
 * until the process exits.
 *
 *   d_leaves   nleaf leaf records (rtfmm_leaf, in device memory)
 *   d_bodies   bodies as (x, y, z, q) doubles, grouped by leaf
 *   d_U        U of the SVD e2c = U S V^T, row-major num_surf x num_surf
 *   d_VSinvT   (V S^-1)^T, row-major num_surf x num_surf
 *              (rtfmm_b200_get_operator gives U and V S^-1 for a set-up)
 *   d_q_equiv  output, nleaf x num_surf, row l for leaf l
 *   stream     cudaStream_t to run on (NULL: the default stream)
 *
 * d_bodies, d_U, d_VSinvT and d_q_equiv must be 16-byte aligned and
 * d_leaves 8-byte aligned (RTFMM_EINVAL otherwise).  The batch must fit the
 * scratch: 2*nleaf*num_surf + 3*num_surf + nleaf + ceil((nleaf + 2) / 2)
 * doubles (at P=8, up to 1765 leaves); larger batches return RTFMM_EINVAL
 * and should be split.  A call looks up the scratch array's device address
 * (cudaGetSymbolAddress) unless its stream is capturing, in which case it
 * uses the address found by an earlier call on the device: make the first
 * call on a device before any stream capture.  Every call reuses the same scratch and
 * overwrites what it reads, so nothing carries over between calls; calls
 * that overlap on the GPU (other streams, other host threads) race on it and
 * must be serialised by the caller. */
#define RTFMM_NOALLOC_SCRATCH_BYTES (8u << 20)

typedef struct rtfmm_leaf {
  double cx, cy, cz;   /* leaf centre                         */
  double r;            /* half edge                           */
  double scale;        /* 0.5^depth                           */
  int32_t cell;        /* caller's cell id (not read)         */
  int32_t boff, bnum;  /* the leaf's bodies in d_bodies       */
  int32_t pad;
} rtfmm_leaf;

int rtfmm_b200_p2m_noalloc(int P, int64_t nleaf, const rtfmm_leaf* d_leaves, const double* d_bodies,
                           const double* d_U, const double* d_VSinvT, double* d_q_equiv, void* stream);

/* Handles share their operator tables through a process-wide cache keyed by
 * (P, images, cycle): a set-up whose tables are cached copies them instead of
 * building them (the SVD, the M2M products and the kernel spectra).  This
 * frees the cache (up to 4 sets; about 0.1 GB each at P = 10); handles keep
 * their own copies. */
void rtfmm_b200_clear_operator_cache(void);

/* The handle's operator tables to a file (a versioned binary image in the
 * host's byte order; about 0.1 GB at P = 10), and a saved file back into the
 * process-wide cache, so that set-ups with the same (P, images, cycle) skip
 * the build (0.2-0.6 s) in a later process.  The reference recomputes the
 * tables in every solve() (fmm.cpp:37-48).  A load checks every table's size
 * against P and returns RTFMM_EINVAL for a file that does not match. */
int rtfmm_b200_save_operators(rtfmm_fmm* fmm, const char* path);
int rtfmm_b200_load_operators(const char* path);

/* Last error message of the calling thread ("" if none). */
const char* rtfmm_b200_last_error(void);

/* Library version string. */
const char* rtfmm_b200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RTFMM_B200_H */
