/* fmmg.h -- C ABI of the B200 (sm_100a) kernel-independent FMM evaluator.
 *
 * This is the drop-in boundary for the single-rank, single-GPU evaluate() path
 * of the reference aashays/fmm-g.  Paths below are relative to the reference
 * root.  One handle replaces one reference FMM3d_MPI object
 * (fmm3d_mpi/fmm3d_mpi.hpp:36-249) together with the four GPU entry points
 * it called per evaluate:
 *   dense_inter_gpu(point3d_t*)  U-list P2P          fmm3d_mpi/gpu_setup.h:58
 *   gpu_up(upComp_t*)            S2M                 fmm3d_mpi/gpu_setup.h:60
 *   gpu_down(dnComp_t*)          L2T                 fmm3d_mpi/gpu_setup.h:62
 *   cudavlistfunc(...)           V-list Hadamard     fmm3d_mpi/gpu_vlist.h:1
 * Every stage of evaluate() runs on the GPU behind fmmg_evaluate*; the tree,
 * the interaction lists and the operators stay resident between calls.
 *
 * Conventions
 *  - Positions and normals are interleaved xyz, FP64, like the reference's
 *    PETSc Vecs (fmm3d_mpi/knlmat3d_mpi.hpp:50-56).  Densities hold srcDOF
 *    values per source and values trgDOF per target, interleaved.
 *  - Inputs and outputs are in the CALLER's point order.  (The reference
 *    redistributes the caller's Vecs inside setup(); at one rank that order is
 *    the input order.)  trg_val is overwritten, as in the reference
 *    (fmm3d_mpi/fmm3d_eval_mpi.cpp:427).
 *  - Every function returns an fmmg_status and never exits, aborts or traps.
 *    fmmg_last_error() gives a message for the last failure on a handle.
 *  - A handle is not thread safe; separate handles may be used concurrently.
 *    All GPU work of a handle is ordered on its stream.
 */
#ifndef FMMG_H_
#define FMMG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FMMG_OK = 0,
  FMMG_INVALID_ARG = 1,   /* bad option, size, pointer or non-finite input */
  FMMG_OOM = 2,           /* host or device allocation failed */
  FMMG_CUDA_ERROR = 3,    /* a CUDA call or kernel launch failed */
  FMMG_TIMEOUT = 4,       /* a bounded device wait ran out (results invalid) */
  FMMG_NOT_SUPPORTED = 5, /* kernel type / np / mode not built */
  FMMG_STATE = 6          /* call order violated (e.g. evaluate before setup) */
} fmmg_status;

/* Kernel ids of fmm3d_mpi/kernel3d_mpi.hpp:37-78 that setup() accepts
 * (fmm3d_mpi/fmm3d_setup_mpi.cpp:113-126). */
enum {
  FMMG_KNL_LAP_S_U = 111, FMMG_KNL_LAP_D_U = 121,
  FMMG_KNL_STK_S_U = 311, FMMG_KNL_STK_S_P = 312,
  FMMG_KNL_STK_D_U = 321, FMMG_KNL_STK_D_P = 322,
  FMMG_KNL_NAV_S_U = 511, FMMG_KNL_NAV_D_U = 521
};

/* Arithmetic of an evaluate. */
typedef enum {
  FMMG_PREC_FP64 = 0,  /* plain form: FP64 throughout */
  FMMG_PREC_MIXED = 1  /* FP32 bulk sums and M2L, FP64 final accumulation */
} fmmg_precision;

/* Options of FMM3d_MPI and its Let3d_MPI, as plain fields:
 *   np          -fmm3d_np            (fmm3d_mpi/fmm3d_setup_mpi.cpp:48)
 *   pts_max     -fmm3d_let3d_ptsMax  (fmm3d_mpi/let3d_mpi.cpp:231)
 *   max_level   -fmm3d_let3d_maxLevel (fmm3d_mpi/let3d_mpi.cpp:232)
 *   kernel_type -kt, coefs {mu, nu}  (fmm3d_mpi/tt0.cpp:164-183)
 *   ctr, root_level                  (FMM3d_MPI::ctr()/rootLevel(), fmm3d_mpi.hpp:177-179)
 * device < 0 builds the host plan only (tree, lists, operators): evaluate is
 * then refused with FMMG_STATE.  stream == NULL makes the handle create its own
 * non-blocking stream. */
typedef struct {
  int kernel_type;
  double coefs[2];
  int np;
  int pts_max;
  int max_level;
  double ctr[3];
  int root_level;
  int device;
  void* stream; /* cudaStream_t */
} fmmg_options;

typedef struct fmmg_handle fmmg_handle;

/* Fills *opt with the reference defaults: Laplace single layer, coefs {1, 0.25}
 * (tt0.cpp:179-183), np 6 (fmm3d_mpi.cpp:33), ptsMax 150 and maxLevel 30
 * (options_0:47-48), root box [0,1]^3 as ctr 0.5 / rootLevel 1 (tt0.cpp:435-436),
 * device 0. */
fmmg_status fmmg_default_options(fmmg_options* opt);

/* new FMM3d_MPI + knl()/np()/ctr()/rootLevel() setters.  Builds the operator
 * tables of (kernel_type, coefs, np), or copies them from the sets the process
 * keeps: the 4 most recently used, as the reference shares one operator
 * manager per kernel and order (fmm3d_mpi/matmgnt3d_mpi.cpp:526-543). */
fmmg_status fmmg_create(const fmmg_options* opt, fmmg_handle** out);

/* FMM3d_MPI::setup() (fmm3d_mpi/fmm3d_setup_mpi.cpp:41-567): builds the
 * adaptive octree over the sources, bins the targets, builds the U/V/W/X lists
 * (fmm3d_mpi/let3d_mpi.cpp:1637-1768) and their device CSR forms, the
 * operators, and uploads everything.  src_nrm may be NULL for single-layer
 * kernels.  All points must lie in the closed root box; n_src >= 1, n_trg >= 0.
 * May be called again on the same handle with new points (points that moved):
 * the tree, lists and device data are rebuilt and the operator tables reset to
 * the built ones (tables replaced through fmmg_operator are dropped).  A setup
 * again first waits for the handle's queued work; the previous setup's device
 * blocks serve the new one, and those it does not reuse stay with the handle
 * until the start of its second device call after the setup (so the first
 * call's own work arrays can reuse them too), or until an allocation needs
 * the memory.  The V lists expanded per spectrum slot (fmmg_worklist 6 and 7)
 * and the adjoint's lists are formed when first needed, not by setup. */
fmmg_status fmmg_setup(fmmg_handle* h, int64_t n_src, const double* src_xyz, const double* src_nrm,
                       int64_t n_trg, const double* trg_xyz);

/* FMM3d_MPI::evaluate(srcDen, trgVal) (fmm3d_mpi/fmm3d_eval_mpi.cpp:396-1515)
 * on HOST buffers: src_den [n_src*srcDOF], trg_val [n_trg*trgDOF].  Copies in,
 * runs every stage on the GPU, copies out and synchronises. */
fmmg_status fmmg_evaluate(fmmg_handle* h, const double* src_den, double* trg_val);

/* k right-hand sides on HOST buffers (pinned memory gives the fastest
 * copies): src_den [k][n_src*srcDOF], trg_val [k][n_trg*trgDOF].  Copies in,
 * evaluates with the given precision, copies out and synchronises. */
fmmg_status fmmg_evaluate_host(fmmg_handle* h, int k, const double* src_den, double* trg_val, int precision);

/* k right-hand sides on DEVICE buffers: d_src_den [k][n_src*srcDOF],
 * d_trg_val [k][n_trg*trgDOF], caller order.  Enqueued on the handle's stream;
 * returns without synchronising. */
fmmg_status fmmg_evaluate_device(fmmg_handle* h, int k, const double* d_src_den, double* d_trg_val,
                                 int precision);

/* Transposed evaluator (no counterpart in the reference, which has no adjoint).
 * With phi = A(x_t) sigma the map evaluated by fmmg_evaluate_device for the
 * set-up points, and w a weight per target value, it computes for each of k
 * right-hand sides, on DEVICE buffers in caller order, FP64:
 *   d_g      [k][n_src*srcDOF] = A^T w, the gradient of <w, phi> with respect
 *            to the source density (the forward stages transposed and run in
 *            reverse order on the same tree and operators); NULL skips it;
 *   d_grad_t [k][n_trg][3]     = the gradient of <w, phi> with respect to each
 *            target position (sources fixed), from kernel-gradient forms of
 *            the near-field, M2T and L2T sums after a forward upward, V-, X-
 *            and downward pass on d_src_den; NULL skips it.  Laplace kernels
 *            111 and 121 only (FMMG_NOT_SUPPORTED otherwise); needs d_src_den.
 * d_w is [k][n_trg*trgDOF], d_src_den [k][n_src*srcDOF] (may be NULL when
 * d_grad_t is NULL).  Uses the handle's work arrays (not concurrent with
 * evaluate on the same handle); enqueued on the handle's stream, returns
 * without synchronising.  Forward state is recomputed, never stored. */
fmmg_status fmmg_adjoint_device(fmmg_handle* h, int k, const double* d_src_den, const double* d_w, double* d_g,
                                double* d_grad_t);

/* fmmg_adjoint_device on HOST buffers: copies in, runs, copies out, synchronises. */
fmmg_status fmmg_adjoint_host(fmmg_handle* h, int k, const double* src_den, const double* w, double* g,
                              double* grad_t);

/* Waits for all work enqueued on the handle's stream. */
fmmg_status fmmg_synchronize(fmmg_handle* h);

/* Like fmmg_evaluate_device with k = 1 but only the stages in stage_mask
 * (bit 0 upward S2M/M2M/C2E, 1 U-list, 2 V-list, 3 W-list, 4 X-list,
 * 5 downward L2L/C2E/L2T) -- the reference's per-stage switches exposed for
 * stage-level checks. */
fmmg_status fmmg_evaluate_stages(fmmg_handle* h, const double* d_src_den, double* d_trg_val,
                                 int precision, int stage_mask);

/* FMM3d_MPI::check() (fmm3d_mpi/fmm3d_check_mpi.cpp:34-172): dense FP64 sums
 * on the GPU at n_chk caller-order target indices, compared with trg_val
 * (host, caller order).  Returns the relative L2 error and the max abs error;
 * dense_out (host, [n_chk*trgDOF]) may be NULL. */
fmmg_status fmmg_check(fmmg_handle* h, const double* src_den, const double* trg_val, int64_t n_chk,
                       const int64_t* chk_idx, double* rel_l2, double* max_abs, double* dense_out);

/* Sizes: srcDOF, trgDOF, number of tree nodes, leaves, maximum depth. */
fmmg_status fmmg_info(const fmmg_handle* h, int* src_dof, int* trg_dof, int64_t* n_nodes,
                      int64_t* n_leaves, int* max_depth);

/* Per-stage device time of the last evaluate, milliseconds, in the order of
 * the PETSc log events (fmm3d_mpi/manage_petsc_events.cpp:77-140): upward,
 * U-list, V-list, W-list, X-list, downward (incl. L2T), total.  n >= 7. */
fmmg_status fmmg_stage_times(const fmmg_handle* h, double* ms, int n);

/* Per-kernel device time of the last timed evaluate, milliseconds, n >= 12:
 * prep (density gather + clears), S2M, upward GEMMs (M2M + C2E), near-field
 * P2P (U, direct W and X), M2L forward FFT, M2L Hadamard, M2L inverse FFT,
 * W-list M2T, X-list S2L, downward GEMMs (L2L + C2E), L2T, value scatter. */
fmmg_status fmmg_kernel_times(const fmmg_handle* h, double* ms, int n);

/* Algorithmic work of one single-RHS evaluate, from the plan (n >= 16):
 * kernel-pair counts of the near-field P2P, S2M, S2L, M2T and L2T sums;
 * M2L source spectra, target spectra, target parents, (parent, neighbour)
 * pairs and V-list interactions; FLOPs of the upward and downward GEMMs;
 * spectrum length, equivalent-kernel source and target DOF, node count.  With
 * n >= 19 also the mixed form's own figures: spectrum length on its
 * (2np-1)^3 grid and the FLOPs of its upward GEMMs (parents through the folded
 * C2E x M2M product) and downward GEMMs (factored pseudo-inverses). */
fmmg_status fmmg_plan_stats(const fmmg_handle* h, int64_t* stats, int n);

/* on != 0 (the default for device handles): fmmg_setup builds the octree,
 * bins the targets and builds the U/V/W/X lists on the handle's GPU -- the
 * same tree, permutations, ranges and lists as the host build, which on == 0
 * selects.  Takes effect at the next fmmg_setup. */
fmmg_status fmmg_set_tree_device(fmmg_handle* h, int on);

/* Wall time of the last fmmg_setup, ms (n >= 9): input checks; the plan's
 * phases -- sources into the tree, targets binned, node flags and centres,
 * U/V/W/X lists, work lists, the adjoint's lists; the upload to the device
 * (and its work arrays); the total.  With n >= 13 also the build of the
 * handle's operator set at fmmg_create (0 when the process had it cached):
 * C2E up pseudo-inverse, C2E down pseudo-inverse, M2M / L2L tables, M2L
 * translation spectra.  With n >= 17 also the upload's parts: geometry and
 * tree arrays, work lists, operator tables, work arrays and the rest. */
fmmg_status fmmg_setup_times(const fmmg_handle* h, double* ms, int n);

/* Number of this library's kernels launched by the last evaluate call. */
fmmg_status fmmg_launch_count(const fmmg_handle* h, int64_t* n);

/* Arithmetic used by fmmg_evaluate (host buffers); FMMG_PREC_FP64 by default. */
fmmg_status fmmg_set_precision(fmmg_handle* h, int precision);

/* on != 0: every later evaluate records per-kernel CUDA events on the
 * handle's stream and waits for them (fmmg_evaluate always does). */
fmmg_status fmmg_set_timing(fmmg_handle* h, int on);

/* on != 0: fmmg_evaluate_device replays a CUDA graph of the whole evaluate.
 * The first call for given (k, precision, d_src_den, d_trg_val) runs eagerly
 * (and allocates what that form needs); the second captures the evaluate on
 * the handle's stream into a graph, and later calls with the same key launch
 * it (one key is cached; another key starts over).  The handle's stream must
 * not be the legacy default stream.  If capture is refused the handle stays
 * eager and fmmg_graph_state reports why.  Turning it on or off, a new setup
 * or a changed operator table drops the graph.  No counterpart in the
 * reference. */
fmmg_status fmmg_set_graph(fmmg_handle* h, int on);
/* active: 1 while a captured graph is cached; note: why capture was refused ("" if not). */
fmmg_status fmmg_graph_state(const fmmg_handle* h, int* active, const char** note);

/* The kernels of the mixed form's FP32 row GEMMs (leaf and downward C2E
 * factors, folded C2E x M2M, L2L).  path 1 (the default): the tensor cores
 * (tcgen05, 3xTF32 split products with every 32-wide K block summed in FP32),
 * for every GEMM whose X rows are 16-byte aligned with K % 4 == 0 (np = 3, 5
 * and 7 Laplace surfaces are not, and take path 0); path 0: the CUDA cores
 * with 128 x 160 tiles; 2: the CUDA cores with 128 x 64 tiles.  On the
 * 1M-point Laplace np=6 workload, 8 right-hand sides, path 1 gives 3.0e-6
 * against the dense sum where path 0 gives 2.5e-6.  FMMG_INVALID_ARG for
 * another path.  No counterpart in the reference. */
fmmg_status fmmg_set_gemm_path(fmmg_handle* h, int path);
/* flag = 1 if a kernel gave up a bounded wait since the last call (its
 * results are then invalid), else 0; clears the flag.  Synchronises.  The
 * synchronising calls (fmmg_evaluate, fmmg_evaluate_host, fmmg_adjoint_host)
 * read and clear the flag themselves and return FMMG_TIMEOUT when it was set. */
fmmg_status fmmg_device_error(fmmg_handle* h, int* flag);
/* The error path of the bounded device waits, for tests: one CTA allocates
 * tensor memory, waits on an mbarrier with a limit of limit_ns nanoseconds
 * (0 .. 2e9) and frees it.  arrive != 0: the mbarrier is arrived on first and
 * the call returns FMMG_OK; arrive == 0: nothing arrives (no tensor-core work
 * is ever issued), the wait runs out and the call returns FMMG_TIMEOUT with
 * the device still usable.  Synchronises the device.  No counterpart in the
 * reference. */
fmmg_status fmmg_selftest_wait(int device, int arrive, int64_t limit_ns);

/* Autotuner (no counterpart in the reference): times `reps` evaluates of
 * (k, precision) on the caller's device buffers for each candidate launch
 * shape -- for the mixed form with k >= 2 the form of the Hadamard kernel
 * (1..4, see fmmg_tuning), then rows per CTA of the Hadamard kernel (32, 64,
 * 128, 256), then for the mixed form the split-K threshold of the FP32 GEMMs
 * (0, 1, 2, 4 CTAs per SM) -- keeps the fastest in the handle and returns its
 * time in best_ms.  d_trg_val is overwritten.  Synchronises. */
fmmg_status fmmg_autotune(fmmg_handle* h, int k, int precision, const double* d_src_den, double* d_trg_val,
                          int reps, double* best_ms);
/* vals[0..2] = Hadamard rows per CTA (FP32 form), Hadamard rows per CTA (FP64
 * form), split-K threshold (CTAs per SM); with n >= 4, vals[3] = the form of
 * the FP32 Hadamard for k >= 2 (1, 2: 27 accumulators per right-hand side, 1
 * or 2 right-hand sides a thread; 3, 4: 8 output-child accumulators, 2 or 4
 * right-hand sides a thread; default 4); with n >= 5, vals[4] = the FP32 GEMM
 * classes on the tensor cores when path 1 is on (bit 0 leaf C2E F1, 1 leaf
 * C2E F2, 2 folded C2E x M2M, 3 L2L, 4 downward C2E F1, 5 downward C2E F2;
 * default 63); with n >= 6, vals[5] = the products of the 3xTF32 split (3, or
 * 4 with lo*lo).  set != 0 installs them (FMMG_INVALID_ARG for values out of
 * range), else reads. */
fmmg_status fmmg_tuning(fmmg_handle* h, int* vals, int n, int set);

/* Host-plan introspection (valid after setup, also with device < 0).
 * which: 0 U, 1 V, 2 W, 3 X lists in the reference form.  node_rec receives
 * per node {depth, path x, path y, path z, parent, first child, tag bits,
 * sources in subtree, targets in subtree}; ptr has n_nodes+1 entries; idx
 * entries are node ids of this handle's numbering.  NULL buffers only size.
 * Tag bits follow fmm3d_mpi/let3d_mpi.hpp:28-39 (1 contributor, 2 user,
 * 4 evaluator, 16 has-sources). */
fmmg_status fmmg_tree(const fmmg_handle* h, int32_t* node_rec, int64_t* perm_src, int64_t* perm_trg);
fmmg_status fmmg_lists(const fmmg_handle* h, int which, int64_t* ptr, int32_t* idx, int64_t* total);

/* The GPU work lists derived from those lists at setup (valid after setup,
 * also with device < 0), following the per-node decisions of the reference
 * evaluate() (fmm3d_mpi/fmm3d_eval_mpi.cpp:1146, 1249): which 0 the direct
 * sources of each evaluator leaf (its U list, the W boxes with fewer than
 * |UE| x srcDOF source values, and its X list when the leaf has fewer than
 * |DC| x trgDOF target values), 1 the other W boxes (applied from their UE
 * surface), 2 the X sources of the other nodes (summed onto their DC
 * surface), 3 per target parent the same-depth non-leaf neighbours whose
 * children feed its children's V lists, 4 the leaves with sources (S2M),
 * 5 the evaluator leaves at depth >= 2 (L2T), 6 the V lists expanded per
 * target spectrum slot, 7 the same inverted per source spectrum slot.  rows
 * receives *n_rows node ids; for which 0-3 ptr (n_rows + 1 entries) and idx
 * (*total entries) hold each row's node ids, for 4 and 5 *total is 0; for 6
 * and 7 the rows are the slots' nodes and each entry of a row is a pair
 * (slot on the other side, translation id 0..315) in idx, ptr counting pairs.
 * NULL buffers only size. */
fmmg_status fmmg_worklist(const fmmg_handle* h, int which, int32_t* rows, int64_t* ptr, int32_t* idx,
                          int64_t* n_rows, int64_t* total);

/* Operator tables built by this handle.  which: 0 UC->UE pseudo-inverse,
 * 1 UE->UC (octant idx 0..7), 2 DC->DE pseudo-inverse, 3 DE->DC (octant 0..7),
 * 4 UE->DC translation spectrum (idx 0..315, complex as pairs).  Matrices are
 * column-major as the reference NumMat (common/nummat.hpp:96-105); spectra use
 * the FFTW r2c layout.  *count receives the number of doubles.  With set != NULL
 * the table is replaced (before the next evaluate) -- used to run the GPU path
 * on an externally supplied operator set.  Read only, the mixed form's own
 * tables: 5 the translation spectra on its (2np-1)^3 grid (idx 0..315, derived
 * from table 4), 6 the folded upward operator C2E x M2M, (ue x 8 ue)
 * column-major with the 8 octants side by side (derived from tables 0 and 1);
 * set on 5 or 6 returns FMMG_INVALID_ARG.  No counterpart in the reference
 * for 5 and 6. */
fmmg_status fmmg_operator(fmmg_handle* h, int which, int idx, double* get, const double* set,
                          int64_t* count);

/* Dense FP64 direct sum that allocates no memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc where they need the
 * result -- work recorded while a stream is captured into a CUDA graph, code
 * whose device memory is owned by a pool that forbids driver allocations, or
 * latency-critical paths.  d_val[i*trgDOF+t] = sum over all sources of the
 * kernel block times the density, like the reference check()'s dense sum
 * (fmm3d_mpi/fmm3d_check_mpi.cpp:122-131); all arrays are device pointers in
 * the caller's layout (xyz interleaved positions/normals, DOF interleaved
 * densities/values); d_nrm may be NULL for single-layer kernels.  The
 * accumulation scratch is a fixed array of 2^20 doubles inside the library on
 * every GPU that loads it (held until the process exits): n_trg * trgDOF above
 * 1,048,576 is rejected with FMMG_INVALID_ARG, and so are the Navier kernels
 * with nu == 1 (as fmmg_create does); n_trg == 0 does nothing and returns
 * FMMG_OK.  The first call on a device resolves the scratch address for that
 * device and should come before any stream capture; the address is kept for
 * the process, so the entry point must not be used across a cudaDeviceReset.
 * All calls on a device share the scratch: calls that overlap on the GPU race.
 * Work is enqueued on `stream` (a cudaStream_t, NULL = the default stream) and
 * the call returns without synchronising.  Errors are reported by the status
 * code only. */
fmmg_status fmmg_dense_noalloc(int kernel_type, const double* coefs, int64_t n_src, const double* d_src,
                               const double* d_nrm, const double* d_den, int64_t n_trg, const double* d_trg,
                               double* d_val, void* stream);

/* Message of the last failure on h (or of the last failed fmmg_create when
 * h == NULL).  Never NULL. */
const char* fmmg_last_error(const fmmg_handle* h);

fmmg_status fmmg_destroy(fmmg_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* FMMG_H_ */
