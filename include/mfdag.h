/*
 * mfdag.h -- C ABI of the B200 (sm_100a) numeric phase for the supernodal
 * multifrontal Cholesky solver to-mo-ki/multifrontal-DAG.
 *
 * Two layers:
 *
 *  1. Handle API (mfd_*): the drop-in boundary.  A handle owns all device
 *     memory of one analysed system (or of a batch of independent systems):
 *     factor panels and update matrices resident in HBM, the device-built index
 *     maps, and the launch plan.  Plain pointers and sizes only; integer arrays
 *     are int32 with the reference's 1-based values; dense values are FP64,
 *     column-major.
 *
 *  2. Reference-named entry points (hppllt_*): the same calls as the
 *     reference's public Fortran API (src/main/hppllt.f90:8-9), with the same
 *     argument meaning and module-global single-instance state, for a C or
 *     ISO_C_BINDING caller.  They run the host symbolic analysis in C++ and the
 *     numeric phase on the GPU.
 *
 * Status codes: 0 ok; >0 = 1-based (permuted) column of the first
 * non-positive pivot (LAPACK convention); negative = MFD_E_*.
 */
#ifndef MFDAG_H
#define MFDAG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MFD_OK 0
#define MFD_E_ARG (-1)        /* bad argument or malformed symbolic input            */
#define MFD_E_CUDA (-2)       /* a CUDA call failed                                  */
#define MFD_E_NOMEM (-3)      /* device or host allocation failed                    */
#define MFD_E_TIMEOUT (-4)    /* a bounded device-side wait expired                  */
#define MFD_E_NOCONV (-5)     /* iterative refinement did not reach the tolerance     */
#define MFD_E_STATE (-6)      /* call out of order (e.g. solve before factorize)     */

#define MFD_PREC_FP64 0       /* FP64 factor and solve                               */
#define MFD_PREC_FP32_IR 1    /* FP32 factor + FP64 iterative refinement             */

typedef struct mfd_handle mfd_handle;

typedef struct {
  int32_t nb;              /* reference option OPTION_NB (options_m.f90:4): tile size of the
                              reference layout; used for the block-local index export        */
  int32_t max_zero;        /* reference option OPTION_MAX_ZERO (options_m.f90:5)             */
  int32_t precision;       /* MFD_PREC_*                                                      */
  int32_t ir_max_iter;     /* refinement iterations (precision FP32_IR), default 20           */
  double ir_tol;           /* target normwise backward error, default 1e-12                   */
  int32_t use_graph;       /* 1: replay factor/solve as CUDA graphs (default 1)               */
  int32_t device;          /* CUDA device ordinal (default 0)                                 */
  int32_t small_front_max; /* fronts up to this order run in the fused one-CTA kernel (0=auto)*/
  int32_t panel_width;     /* column panel of the blocked large-front factorization (0=auto) */
  int32_t reserved[7];     /* schedule switches, 0 = default: [0] trailing-update kind (1 FFMA
                              tiles, 2 single-pass TF32, 3 FP64 DMMA in whole 128 x 128 tiles),
                              [1] = 1 lookahead off, [2] = 1 programmatic launch along the panel
                              chain, [3] = 1 no programmatic launch between solve steps, [4] = 1
                              no side streams per level, [5] = panel steps per deferred trailing
                              update (1 = none), [6] = 1 single-RHS large-front solves one launch
                              per panel step instead of one per level                           */
} mfd_options;

/* Symbolic data exactly as the reference holds it after hppllt_analyze
 * (hppllt_data_m.f90:14-29, hppllt.f90:56-73); all arrays 1-based int32. */
typedef struct {
  int32_t n, nnz, num_node;
  const int32_t *node_ptr;  /* num_node+1 : node_sets%ptr                              */
  const int32_t *parent;    /* num_node   : supernodal parent, 0 for the root          */
  const int32_t *lrow_ptr;  /* num_node+1 : l_structure set                            */
  const int32_t *lrow;      /* sum nr     : L row lists, ascending, permuted numbering */
  const int32_t *acol_ptr;  /* n+1        : a_structure (permuted lower CCS)           */
  const int32_t *arow;      /* nnz        : a_structure rows (any order in a column)   */
  const int32_t *ccs_perm;  /* nnz        : entry k of a_structure takes a(ccs_perm(k)) */
  const int32_t *perm;      /* n          : permuted position i holds original perm(i) */
} mfd_symbolic;

typedef struct {
  int32_t iterations;       /* refinement steps taken (0 for FP64)                     */
  int32_t converged;        /* 1 if backward_error <= ir_tol                           */
  double backward_error;    /* ||b-Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf), FP64  */
  double residual_ref;      /* the reference driver's metric ||b-Ax||_2 / ||x||_2      */
  double time_ms;           /* device time of the whole solve (events)                 */
} mfd_report;

typedef struct {
  int64_t n, nnz_a, num_front, num_level;
  int64_t cost;             /* calculate_cost (cost_calculator_m.f90:9-20): sum_f sum_{k=nr+1}^{nr+nc} k^2 */
  int64_t nonzero;          /* count_nonzero (cost_calculator_m.f90:22-33), int64 here          */
  int64_t panel_bytes;      /* resident factor panels                                          */
  int64_t update_pool_bytes;/* statically planned update-matrix pool (peak of live updates)    */
  int64_t launches_factor;  /* kernels launched by one factorize                               */
  int64_t launches_solve;   /* kernels launched by one forward+backward solve                  */
  int64_t max_front;        /* largest front order                                             */
  double factor_ms;         /* device time of the last factorize (events)                      */
  double solve_ms;          /* device time of the last solve                                   */
  double time_info[7];      /* the reference's 7 phase timers (time_list_m.f90:3-10), seconds:
                               ordering, analyze, factorize, solve, forward, backward,
                               real_factorize                                                  */
  int64_t pivot_fallbacks;  /* FP32 factorization: 32-column diagonal sub-blocks whose FP32 pivot
                               chain met a small pivot and was redone in FP64 (last factorize) */
  double setup_s[4];        /* handle set-up, seconds: host symbolic analysis (mfd_analyze*),
                               level / memory plan, device index maps and their exports,
                               residual CSR and numeric storage                                */
} mfd_stats;

/* ---- handle API ------------------------------------------------------------ */

/* Default options (FP64, graphs on, device 0). */
void mfd_default_options(mfd_options *opt);

/* Replaces the device-side half of create_data_structure (hppllt.f90:83-106):
 * copies the symbolic arrays to the device, builds local_index, supernodal_index
 * and block_local_index on the GPU, and plans the level schedule and memory. */
int mfd_create(mfd_handle **h, const mfd_symbolic *sym, const mfd_options *opt);

/* Batch of independent systems analysed separately (one symbolic per system):
 * all systems share one handle, one level schedule and one launch per level. */
int mfd_create_batch(mfd_handle **h, int32_t num_systems, const mfd_symbolic *syms, const mfd_options *opt);

/* Host symbolic analysis (hppllt_analyze, hppllt.f90:24-81) + mfd_create.
 * order_perm (new->old, 1-based) stands in for METIS_NodeND's output
 * (hppllt.f90:47-51); NULL is the use_metis = 0 branch. */
int mfd_analyze(mfd_handle **h, int32_t n, const int32_t *ccs_col, const int32_t *ccs_row,
                const int32_t *order_perm, const mfd_options *opt);

/* Fill-reducing ordering (host, no device work) where the reference calls
 * METIS_NodeND (ordering_m.f90:11-36): nested dissection of the graph of the
 * lower CCS (1-based, any row order), by BFS level-structure bisection with a
 * refined separator.  order_perm (n) receives new -> old, 1-based -- the
 * argument mfd_analyze takes.  hppllt_analyze with use_metis = 1 uses it when
 * no ordering was supplied through hppllt_set_ordering. */
int mfd_order(int32_t n, const int32_t *ccs_col, const int32_t *ccs_row, int32_t *order_perm);

/* Subtree-to-GPU mapping of one system (host): the reference's tree_pruning
 * (src/main/algorithms/tree_pruning_m.f90:13-155), restated.  Inputs are the
 * supernodal tree as the reference holds it: node_size (supernode columns),
 * cc (update rows nr), num_child and the concatenated children (tree_child),
 * all 1-based, nodes in postorder with the root last.  Subtrees are split,
 * heaviest first (weight = sum over the subtree of sum_{k=nr+1}^{nr+nc} k^2),
 * until their weights pack into p or more bins with min / max > tol.  roots
 * (capacity num_node) receives the subtree roots in the reference's list
 * order and *count their number.  64-bit weights (no overflow for large
 * fronts). */
int mfd_subtree_partition(int32_t num_node, const int32_t *node_size, const int32_t *cc, const int32_t *num_child,
                          const int32_t *child, double tol, int32_t p, int32_t *roots, int32_t *count);

/* Host-only symbolic analysis (hppllt_analyze's symbolic half, no device work):
 * the result object owns the arrays; mfd_symbolic_view fills an mfd_symbolic
 * whose pointers stay valid until mfd_symbolic_free. */
typedef struct mfd_analysis mfd_analysis;
int mfd_symbolic_analyze(mfd_analysis **out, int32_t n, const int32_t *ccs_col, const int32_t *ccs_row,
                         const int32_t *order_perm, int32_t max_zero);
int mfd_symbolic_view(const mfd_analysis *a, mfd_symbolic *view);
int mfd_symbolic_free(mfd_analysis *a);

/* Batch analysis: system s is (n[s], ccs_col[s], ccs_row[s], order_perm[s]). */
int mfd_analyze_batch(mfd_handle **h, int32_t num_systems, const int32_t *n, const int32_t *const *ccs_col,
                      const int32_t *const *ccs_row, const int32_t *const *order_perm, const mfd_options *opt);

/* ---- input formats (the step before hppllt_analyze) ----------------------------
 * The reference's driver reads a Matrix Market file and converts its COO lists
 * to CCS before calling hppllt_analyze (example.f90:63-145).
 *
 * mfd_mm_read replaces read_data (example.f90:63-93): '%' lines are skipped,
 * then "n n nnz" and nnz lines "row col value" (1-based; pattern files get
 * value 1).  The arrays are allocated on the host; free them with mfd_coo_free.
 *
 * mfd_coo_to_ccs replaces coo_to_ccs (example.f90:95-145) and runs on GPU
 * `device`: CCS column pointers (n+1), rows and values (nnz), 1-based, rows
 * ascending in each column and entries with equal (row, col) in reverse input
 * order, as the reference's two counting sorts leave them.  Pointers may be
 * host or device memory (inputs and outputs each all one kind); val and
 * ccs_val may both be NULL (structure only).  An index outside 1..n is
 * MFD_E_ARG.
 *
 * mfd_analyze_csr: direct CSR input (no counterpart in the reference).  The
 * CSR (row pointers n+1, column indices; `base` 0 or 1) holds the lower
 * triangle or the whole symmetric matrix (entries above the diagonal are
 * ignored; the CSR of the upper triangle is the lower CCS and goes to
 * mfd_analyze as it is).  Its lower triangle is converted to CCS on the GPU
 * and analysed as by mfd_analyze; afterwards mfd_factorize takes the values
 * in the caller's CSR order (csr_ptr[n] - base of them). */
typedef struct {
  int32_t n;
  int64_t nnz;
  int32_t *row, *col;       /* 1-based coordinates, nnz each */
  double *val;
} mfd_coo;
int mfd_mm_read(const char *path, mfd_coo *out);
void mfd_coo_free(mfd_coo *coo);
int mfd_coo_to_ccs(int32_t n, int64_t nnz, const int32_t *row, const int32_t *col, const double *val,
                   int32_t *ccs_col, int32_t *ccs_row, double *ccs_val, int32_t device);
int mfd_analyze_csr(mfd_handle **h, int32_t n, const int32_t *csr_ptr, const int32_t *csr_col, int32_t base,
                    const int32_t *order_perm, const mfd_options *opt);

/* Replaces the body of hppllt_factorize (hppllt.f90:134-149): permutate,
 * set_zero, set_coefficient, seq/StarPU factorize.  a: original-order lower-CCS
 * values (for a batch, systems concatenated), host or device pointer. */
int mfd_factorize(mfd_handle *h, const double *a);

/* Replaces the body of hppllt_solve (hppllt.f90:160-172): b (n x nrhs,
 * column-major, leading dimension ldb; for a batch, systems concatenated) is
 * overwritten with x.  Host or device pointer.  rep may be NULL. */
int mfd_solve(mfd_handle *h, double *b, int32_t nrhs, int64_t ldb, mfd_report *rep);

/* Factorize + solve in one call (the batched configuration's single launch
 * sequence). */
int mfd_factorize_solve(mfd_handle *h, const double *a, double *b, int32_t nrhs, int64_t ldb, mfd_report *rep);

int mfd_get_stats(mfd_handle *h, mfd_stats *st);

/* Autotuner (no counterpart in the reference): times the factorization of the
 * values `a` (host or device pointer, as for mfd_factorize) under candidate
 * settings, each on a temporary handle built from h's symbolic data (one
 * warm-up, then the median of `repeats` timed factorizations).  Stage 1: the
 * schedule -- the small-front / blocked split small_front_max in
 * {32, 64, 96, 128} and the lookahead on / off.  Stage 2, at the best
 * schedule: the trailing-update kernel (reserved[0]: FP64 DMMA in 128 x 64
 * halves, whole 128 x 128 tiles, or FFMA tiles; FP32 3xTF32 tcgen05 or FFMA)
 * and the deferral depth reserved[5] in {1, 2}.  Writes the fastest options
 * to *best and their factor time (ms) to *best_ms; h is left unchanged: create
 * a handle with *best to use them.  Returns a pivot column > 0 if a
 * factorization fails. */
int mfd_autotune(mfd_handle *h, const double *a, int32_t repeats, mfd_options *best, double *best_ms);

/* Export of the device-built index maps for parity checks.
 * which: 1 local_index (sum nr), 2 supernodal_index (nnz), 3 block-local node
 * pointer (num_node+1), 4 block pointer (groups+1), 5 parent tile numbers,
 * 6 child tile numbers, 7 rebuilt (mod nb) local values (sum nr), 8 block
 * offsets (get_block_offset, per group).  Returns the element count; out may
 * be NULL to query the size.  system selects one system of a batch. */
int64_t mfd_get_index(mfd_handle *h, int32_t system, int32_t which, int32_t *out);

/* Export of the symbolic arrays held by the handle (same ids as mfd_symbolic
 * fields: 1 node_ptr, 2 parent, 3 lrow_ptr, 4 lrow, 5 acol_ptr, 6 arow,
 * 7 ccs_perm, 8 perm).  Returns the element count; out may be NULL. */
int64_t mfd_get_symbolic(mfd_handle *h, int32_t system, int32_t which, int32_t *out);

/* Copy the FP64 factor column block of one front to the host: rows 0..nf-1,
 * columns 0..nc-1 of the front (row = front position, column-major, ld = nf).
 * node is 1-based within the system.  Returns nf*nc or a negative status. */
int64_t mfd_get_front_panel(mfd_handle *h, int32_t system, int32_t node, double *out);

/* Per-kernel-class timing.  While enabled, factorize and solve run without
 * graphs and record CUDA events around every launch on the handle's stream;
 * each class accumulates its launches, device time and algorithmic work
 * (flops and bytes of the algorithm, not hardware counters). */
#define MFD_K_SMALL_FRONT 0   /* fused one-CTA fronts                         */
#define MFD_K_ZERO 1          /* large-front zero fill                         */
#define MFD_K_ASSEMBLE 2      /* large-front assembly of A                     */
#define MFD_K_EXTEND_ADD 3    /* large-front extend-add                        */
#define MFD_K_PANEL 4         /* diagonal-block POTRF + inverse                */
#define MFD_K_UPDATE 5        /* trailing SYRK/GEMM update                     */
#define MFD_K_SOLVE_SMALL 6   /* one-CTA forward/backward solves               */
#define MFD_K_SOLVE_LARGE 7   /* blocked forward/backward solves               */
#define MFD_K_OTHER 8         /* permutations, residuals, norms                */
#define MFD_K_TRSM 9          /* panel TRSM (rows below the diagonal block)    */
#define MFD_K_COUNT 10
typedef struct {
  int64_t launches;
  double ms;
  double flops;
  double bytes;
} mfd_kernel_profile;
int mfd_set_profiling(mfd_handle *h, int32_t enable);
int mfd_get_profile(mfd_handle *h, int32_t kind, mfd_kernel_profile *out);

/* Test of the failure path (no counterpart in the reference).  While enabled,
 * every CTA of the FP32 tensor-core trailing update first waits on an mbarrier
 * that nothing arrives at, with a ~1 ms limit, before issuing any MMA; the
 * expired wait raises the handle's error flag and the kernel returns, so the
 * next mfd_factorize returns MFD_E_TIMEOUT (no GPU fault: every wait is
 * bounded).  Disable it and the handle factors normally again.  FP64 handles
 * and fronts that use no tensor-core update factor normally.  While enabled,
 * the single-RHS large-front solve sweeps' device waits (one launch per level,
 * tasks waiting on other tasks' flags) likewise wait for a value nothing
 * writes, with a ~1 ms limit: mfd_solve returns MFD_E_TIMEOUT, and solves
 * normally once the request is withdrawn. */
int mfd_test_expire_waits(mfd_handle *h, int32_t enable);

int mfd_destroy(mfd_handle *h);

/* ---- dense fronts without allocation ------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc -- code that owns all device memory through its own arena (e.g. a
 * Fortran driver or framework that reserved HBM up front), or a latency-
 * critical loop that must not take the allocator's lock.  Partially factors
 * `count` dense fronts held in one caller-owned device buffer `fronts`: front i
 * is an nf[i] x nc[i] column-major panel at element offset panel_off[i]
 * (ld = nf[i], lower triangle used) and an (nf-nc) x (nf-nc) update matrix at
 * update_off[i] (ld = nf-nc; ignored when nf == nc).  On return the panel holds
 * the factor columns and the update matrix has the Schur complement subtracted;
 * info points to `count` entries: info[i] is 0, or the 1-based column of front
 * i where its first non-positive pivot was met (that front's factor is then
 * not valid; the other fronts are unaffected).
 * Scratch: a static device array of MFD_NOALLOC_MAX_FRONTS x 128 x 128 doubles
 * (1 MiB) plus small tables, held by every GPU that loads the library until the
 * process exits; count > MFD_NOALLOC_MAX_FRONTS is rejected with MFD_E_ARG.
 * The first call on a device looks up the array's device address and sets
 * kernel attributes.  No call can be captured into a CUDA graph: each copies
 * its tables from host memory and waits for the info read-back, so a call on
 * a stream that is being captured returns MFD_E_ARG and issues nothing.  All
 * calls share the one array, so calls that overlap on the GPU (other streams,
 * other host threads) race.  Host-synchronous on `stream` (NULL = default). */
#define MFD_NOALLOC_MAX_FRONTS 8
int mfd_factor_fronts_noalloc(double *fronts, int32_t count, const int64_t *panel_off, const int64_t *update_off,
                              const int32_t *nf, const int32_t *nc, int32_t *info, void *stream);
const char *mfd_noalloc_last_error(void);

/* Last error text of this thread. */
const char *mfd_last_error(void);

/* ---- reference-named entry points (module-global state, hppllt.f90) ------- */

/* hppllt_init(options(4)) (hppllt.f90:13-22): [nb, max_zero, use_starpu, use_metis].
 * Returns 0, or -1 if noptions != 4 (the reference prints and returns). */
int hppllt_init(const int32_t *options, int32_t noptions);
/* Selects the arithmetic (MFD_PREC_*) of the next factorize; not in the reference. */
int hppllt_set_precision(int32_t precision);
/* hppllt_analyze(ccs_col, ccs_row, n) (hppllt.f90:24-81); with use_metis = 1 the
 * ordering is the one supplied through hppllt_set_ordering, or else mfd_order's
 * nested dissection (the reference calls METIS_NodeND there). */
int hppllt_analyze(const int32_t *ccs_col, const int32_t *ccs_row, int32_t n);
/* Supplies the fill-reducing ordering used when use_metis = 1 (new->old, 1-based). */
int hppllt_set_ordering(const int32_t *order_perm, int32_t n);
/* hppllt_factorize(a) (hppllt.f90:123-150) */
int hppllt_factorize(const double *a);
/* hppllt_solve(b) (hppllt.f90:152-173), b in/out, length n */
int hppllt_solve(double *b);
/* hppllt_finalize (hppllt.f90:175-184) */
int hppllt_finalize(void);
double hppllt_get_time_info(int32_t num);   /* hppllt.f90:186-189 */
int64_t hppllt_get_cost(void);              /* hppllt.f90:191-194 */
int64_t hppllt_get_nonzero(void);           /* hppllt.f90:196-199 (int64 here) */
int64_t hppllt_get_array_size(int32_t num); /* hppllt.f90:201-211: 1 supernode, 2 work, 3 border
                                               (sizes of the reference's three FP64 buffers) */

#ifdef __cplusplus
}
#endif

#endif /* MFDAG_H */
