/*
 * xfmm.h -- C ABI of libexafmm_b200.so, the B200 (sm_100a) implementation of
 * exafmm-t's kernel-independent FMM evaluate path.
 *
 * The entry points replace, one for one, the reference's C++ API for this path
 * (namespace exafmm_t; file:line citations are relative to the exafmm-t tree):
 *
 *   xfmm_fmm_create      LaplaceFmm(p, ncrit, filename)                 include/laplace.h:15-22
 *   xfmm_fmm_set_operator_file  the filename argument + save_matrix/load_matrix
 *                                                                       include/fmm_scale_invariant.h:86-160
 *                        ModifiedHelmholtzFmm(p, ncrit, wavek, filename)include/modified_helmholtz.h:17-25
 *                        HelmholtzFmm(p, ncrit, wavek, filename)        include/helmholtz.h:16-24
 *   xfmm_build_tree      get_bounds + build_tree + balance_tree         include/build_tree.h:20-35, 181-199, 336-359
 *                        (uniform variant)                              include/build_non_adaptive_tree.h:17-194
 *   xfmm_build_list      init_rel_coord + set_colleagues + build_list   include/geometry.h:198-215,
 *                                                                       include/build_list.h:123-197
 *   xfmm_m2l_setup       Fmm::M2L_setup                                 include/fmm_scale_invariant.h:277-341, fmm.h:265-333
 *   xfmm_precompute      Fmm::precompute                                include/fmm_scale_invariant.h:151-160, fmm.h:141-153
 *   xfmm_set_charges     update_charges                                 python/exafmm.cpp:275-305
 *   xfmm_upward_pass     FmmBase::upward_pass                           include/fmm_base.h:162-171
 *   xfmm_downward_pass   FmmBase::downward_pass                         include/fmm_base.h:179-200
 *   xfmm_get_values      result scatter of evaluate                     python/exafmm.cpp:190-267
 *   xfmm_evaluate        clear_values + upward + downward + scatter     python/exafmm.cpp:190-267, 313-323
 *   xfmm_gradient_p2p    <Kernel>Fmm::gradient_P2P                      include/laplace.h:91-164 (and twins)
 *   xfmm_verify          FmmBase::verify                                include/fmm_base.h:208-267
 *
 * Conventions
 *   - Every function returns an xfmm_status; xfmm_last_error() gives the message
 *     of the last failure on the calling thread.  No C++ exception crosses the ABI.
 *   - Coordinates are FP64, interleaved (x0,y0,z0,x1,...).  Charges and results are
 *     FP64 reals (Laplace, modified Helmholtz) or interleaved FP64 complex pairs
 *     (Helmholtz).  Results are (ntrg, 4): potential, d/dx, d/dy, d/dz, in the
 *     caller's original target order.
 *   - `on_device` != 0 means the pointer is device memory on the current device;
 *     otherwise it is host memory and the call copies it (stream-ordered, then
 *     synchronises for host outputs).
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  All device work
 *     of a call is ordered on that stream.
 *   - The library holds no global mutable state: different handles may be used
 *     from different host threads concurrently; one handle must not be.
 */
#ifndef XFMM_H
#define XFMM_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  XFMM_OK = 0,
  XFMM_ERR_ARG = 1,         /* invalid argument / shape (python/exafmm.cpp:37-40 analogue) */
  XFMM_ERR_OOM = 2,         /* device or host allocation failed */
  XFMM_ERR_CUDA = 3,        /* a CUDA runtime or library call failed */
  XFMM_ERR_TIMEOUT = 4,     /* a bounded device-side wait ran out */
  XFMM_ERR_STATE = 5,       /* call order violated (e.g. evaluate before precompute) */
  XFMM_ERR_UNSUPPORTED = 6, /* configuration outside the implemented range */
  XFMM_ERR_NUMERIC = 7      /* non-finite input or a failed factorisation */
} xfmm_status;

typedef enum { XFMM_LAPLACE = 0, XFMM_MODIFIED_HELMHOLTZ = 1, XFMM_HELMHOLTZ = 2 } xfmm_kernel;

/* Arithmetic of the evaluate path.
 *   XFMM_FP64  : every stage in FP64, operators as the reference (pinv threshold 4e-16*smax).
 *   XFMM_MIXED : FP32 near field (FP64-accumulated per source tile), FP32 FFT/Hadamard M2L,
 *                FP32 translations; operators precomputed in FP64 with the check-to-equivalent
 *                pinv regularised at 4e-10*smax so FP32 equivalent densities lose nothing. */
typedef enum { XFMM_FP64 = 0, XFMM_MIXED = 1 } xfmm_precision;

typedef struct xfmm_fmm xfmm_fmm;
typedef struct xfmm_tree xfmm_tree;

const char* xfmm_last_error(void);
const char* xfmm_version(void);

/* Fmm object: kernel, expansion order p (2..16), ncrit, wavenumber, precision. */
xfmm_status xfmm_fmm_create(int kernel, int p, int ncrit, double k_re, double k_im, int precision, xfmm_fmm** out);
xfmm_status xfmm_fmm_free(xfmm_fmm* fmm);
/* The constructor's filename argument (include/laplace.h:15-22 and twins; fmm_scale_invariant.h:86-160,
 * fmm.h:83-153): xfmm_precompute reads the operators from this file when its size and r0 match the
 * current tree, as the reference's load_matrix does, and otherwise computes them and writes the file.
 * The file holds the reference's FP64 operators in its .dat layout (r0; per level UC2E_U, UC2E_V, DC2E_U,
 * DC2E_V, M2M[8], L2L[8]; the M2L tables), so files written by the reference's FP64 build and by this
 * library are interchangeable.  The mixed precision derives its operators from the same FP64 ones.
 * NULL or "" (the default) keeps the operators in memory only. */
xfmm_status xfmm_fmm_set_operator_file(xfmm_fmm* fmm, const char* filename);
/* Public fields of FmmBase (fmm_base.h:13-23): p, nsurf, nconv, nfreq, ncrit, depth, and x0[3], r0. */
xfmm_status xfmm_fmm_info(const xfmm_fmm* fmm, int64_t* ints6, double* x0r0_4);

/* Tree over device-resident bodies.  nonadaptive_depth < 0: adaptive tree + 2:1 balance
 * (python/exafmm.cpp:129-140); >= 0: uniform tree to that depth (NON_ADAPTIVE build).
 * Sets fmm->x0, r0 and depth exactly as get_bounds/balance_tree do. */
xfmm_status xfmm_build_tree(xfmm_fmm* fmm, const double* src_xyz, int64_t nsrc, const double* trg_xyz, int64_t ntrg,
                            int nonadaptive_depth, int on_device, void* stream, xfmm_tree** out);
xfmm_status xfmm_tree_free(xfmm_tree* tree);
xfmm_status xfmm_build_list(xfmm_fmm* fmm, xfmm_tree* tree, void* stream);
xfmm_status xfmm_m2l_setup(xfmm_fmm* fmm, xfmm_tree* tree, void* stream);
xfmm_status xfmm_precompute(xfmm_fmm* fmm, xfmm_tree* tree, void* stream);

/* Charges in the caller's original source order (nsrc reals, or nsrc complex pairs). */
xfmm_status xfmm_set_charges(xfmm_fmm* fmm, xfmm_tree* tree, const double* q, int on_device, void* stream);
xfmm_status xfmm_clear_values(xfmm_fmm* fmm, xfmm_tree* tree, void* stream);
xfmm_status xfmm_upward_pass(xfmm_fmm* fmm, xfmm_tree* tree, void* stream);
xfmm_status xfmm_downward_pass(xfmm_fmm* fmm, xfmm_tree* tree, void* stream);
xfmm_status xfmm_get_values(xfmm_fmm* fmm, xfmm_tree* tree, double* out, int on_device, void* stream);
/* clear_values + upward_pass + downward_pass + get_values.  With a host output both return
 * XFMM_ERR_TIMEOUT when a bounded device-side wait of the pass ran out (the results are then
 * incomplete); with a device output that is reported by xfmm_stage_times. */
xfmm_status xfmm_evaluate(xfmm_fmm* fmm, xfmm_tree* tree, double* out, int on_device, void* stream);

/* Tree statistics: nnodes, nleafs, nnonleafs, depth, np2p, nm2p, np2l, n_m2l_src,
 * p2p_pairs, m2p_pairs, l2p_pairs, m2l_pairs (12 int64). */
xfmm_status xfmm_tree_info(const xfmm_tree* tree, int64_t* info12);
/* Flat dump of the tree and lists in the reference's node order; array shapes as
 * oracle/ref_capi.cpp's ref_dump (nnodes from xfmm_tree_info).  Host pointers. */
xfmm_status xfmm_tree_dump(const xfmm_tree* tree, double* geo, uint64_t* key, int32_t* ni, double* nx, int32_t* leafs,
                           int32_t* nonleafs, int32_t* src_perm, int32_t* trg_perm, int32_t* colleagues,
                           int32_t* m2l, int64_t* p2p_off, int32_t* p2p, int64_t* m2p_off, int32_t* m2p,
                           int64_t* p2l_off, int32_t* p2l);
/* Device times (ms, CUDA events) of the last upward + downward pass on this tree: P2M, M2M, P2L,
 * M2L, L2L, L2P check-to-equivalent, target evaluation (P2P + M2P + L2P), total; then the M2L
 * sub-stages forward transform, Hadamard, backward transform; the number of this library's kernel
 * launches in the last evaluate (library GEMM and FFT launches not counted); then the target
 * evaluation split into its near field (P2P) and far field (M2P + L2P) (14 doubles).  Waits for the
 * last pass to finish; XFMM_ERR_TIMEOUT when a bounded device-side wait of that pass ran out (its
 * results are then incomplete). */
xfmm_status xfmm_stage_times(xfmm_fmm* fmm, xfmm_tree* tree, double* ms14);

/* Tuning options of a tree's evaluate (xfmm_set_tuning). */
enum {
  /* mixed path, sparse M2L Hadamard (k_hadamard_rt): target tiles of 512 covered by one CTA, which
   * builds the frequency's operator fragments once for all of them; 1..64, 0 restores the default (4) */
  XFMM_TUNE_SPARSE_HADAMARD_TILES_PER_CTA = 1
};
/* Sets a tuning option for the later evaluates of this tree; results change only within the mixed
 * path's run-to-run rounding.  No counterpart in the reference, whose loops have no tile parameters;
 * it lets a caller's autotuner (exafmm.batch.BatchedFmm.autotune) search tile shapes.  XFMM_ERR_ARG for
 * an unknown option or a value out of range. */
xfmm_status xfmm_set_tuning(xfmm_tree* tree, int option, int value);

/* Many independent systems evaluated together (no counterpart in the reference, which evaluates one
 * system per call).  A batch holds systems that share one kernel and one precision, each set up as for
 * xfmm_evaluate (tree, lists, M2L setup, precompute); the handles must outlive the batch and keep their
 * trees.  xfmm_batch_evaluate runs one evaluate of every system: charges[k] (device, caller's source
 * order; NULL array or entry: keep the system's current charges) in, outs[k] (device, caller's target
 * order) out.  Each system's stages before and after its near field run on `nstreams` concurrent streams
 * forked from `stream` (largest systems first, each to the least-loaded stream); the near field of all
 * systems is one persistent kernel draining a work queue of (system, target leaf) items, largest first,
 * and the exact close-pair corrections of all systems one more launch.  When every system uses the same
 * xfmm_fmm handle, mixed Laplace with one scale-invariant operator set, the work that shares the operators
 * is one launch over all systems too: the pseudo-inverse factors of P2M and L2P, the M2M and the L2L of
 * each level, the sparse M2L Hadamard between the systems' forward and backward M2L transforms, and the
 * far field (a persistent kernel over (system, leaf) items).  Asynchronous on `stream`, no
 * allocation: it may be captured into a CUDA graph (after one evaluate outside the capture). */
typedef struct xfmm_batch xfmm_batch;
enum {
  /* persistent near field: CTAs per SM (0: as many as fit; 1..32) */
  XFMM_BATCH_NEAR_CTAS_PER_SM = 1,
  /* persistent near field: most targets a lane holds, the height of a warp's target tile (1 or 2) */
  XFMM_BATCH_NEAR_TARGETS_PER_LANE = 2,
  /* one-launch sparse M2L Hadamard of mixed Laplace systems sharing one xfmm_fmm: 512-target tiles per CTA,
   * which share one operator fill per frequency and may belong to different systems (1..64; 0: 4) */
  XFMM_BATCH_HADAMARD_TILES_PER_CTA = 3
};
xfmm_status xfmm_batch_create(xfmm_fmm* const* fmms, xfmm_tree* const* trees, int n, void* stream, xfmm_batch** out);
xfmm_status xfmm_batch_evaluate(xfmm_batch* batch, const double* const* charges, double* const* outs, int nstreams,
                                void* stream);
xfmm_status xfmm_batch_set_tuning(xfmm_batch* batch, int option, int value);
xfmm_status xfmm_batch_free(xfmm_batch* batch);
/* The stream each system of a batch of n runs its per-system stages on, as xfmm_batch_evaluate deals
 * them: systems by size (sizes[k], descending, ties in index order), each to the stream with the least
 * total size so far (ties: the lowest stream); min(nstreams, n) streams.  Host only, no device work. */
xfmm_status xfmm_batch_schedule(const int64_t* sizes, int n, int nstreams, int* stream_of);

/* Direct near-field kernel over raw arrays: out += potential and gradient at trg from (src, q); out is
 * ntrg x 4 doubles (Laplace, modified Helmholtz) or ntrg x 8 (Helmholtz: 4 interleaved complex values).
 * precision selects the FP64 or FP32 device kernel. */
xfmm_status xfmm_gradient_p2p(int kernel, double k_re, double k_im, int precision, const double* src_xyz,
                              int64_t nsrc, const double* q, const double* trg_xyz, int64_t ntrg, double* out,
                              int on_device, void* stream);

/* Size of the fixed device scratch of xfmm_gradient_p2p_noalloc (16 MiB): 40 bytes per source and
 * 32 per target, each region rounded up to 256 bytes. */
#define XFMM_NOALLOC_SCRATCH_BYTES (16u << 20)

/* xfmm_gradient_p2p with device pointers only and no allocation: the packed bodies live in one
 * static device array per device instead of memory allocated per call.  No counterpart in the
 * reference (its gradient_P2P, include/laplace.h:91-164, is a host loop).  For callers that must not
 * allocate device memory while they run (allocation can synchronise the device; their memory pool
 * is fixed at start-up).  The first call on each device looks the array up (make it before any
 * stream capture begins); sizes beyond XFMM_NOALLOC_SCRATCH_BYTES return XFMM_ERR_ARG; out is
 * accumulated into (start it at zero for the plain result); the scratch needs no initial contents;
 * the call is asynchronous on stream; overlapping calls on one device share the scratch and race.  The
 * array's address is looked up once per device and kept: a device reset (cudaDeviceReset) while the
 * library is loaded is not supported. */
xfmm_status xfmm_gradient_p2p_noalloc(int kernel, double k_re, double k_im, int precision, const double* src_xyz,
                                      int64_t nsrc, const double* q, const double* trg_xyz, int64_t ntrg,
                                      double* out, void* stream);

/* Self-test of the bounded device-side waits (no counterpart in the reference): one kernel waits on an
 * mbarrier phase that nothing completes, with a limit of limit_cycles SM clock cycles (1..1e9), then
 * gives up as the library's waiting kernels do.  Returns XFMM_ERR_TIMEOUT when the wait ran out and was
 * reported through the device status flag as designed; the device stays usable afterwards. */
xfmm_status xfmm_selftest_bounded_wait(int64_t limit_cycles);

/* FmmBase::verify on the device: relative L2 error of potential and gradient of the last
 * evaluate against FP64 direct summation over all sources, on every target (sample == 0)
 * or the targets of 10 leaves at stride nleafs/10 (sample != 0). */
xfmm_status xfmm_verify(xfmm_fmm* fmm, xfmm_tree* tree, int sample, double* err2, void* stream);

#ifdef __cplusplus
}
#endif
#endif
