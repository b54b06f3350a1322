// Launch wrappers of the sm_100a kernels (kernels.cu).  Every wrapper enqueues
// on `st` and returns nothing; errors surface through cudaGetLastError /
// stream synchronisation in the caller.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "plan.hpp"

namespace mfd {

constexpr int kSmallFrontMax = 128;   // widest front of the one-CTA / one-warp small-front kernels
constexpr int kFactB = 128;          // column panel of the blocked large-front factorization
constexpr int kTrRowsH = 64;         // rows per CTA of the panel TRSM
constexpr int kUpdTile = 128;        // trailing-update output tile (tensor path)
constexpr int kUpdTileSimt = 64;     // trailing-update output tile (FMA path)
constexpr int kSolveB = kFactB;      // column step of the large-front solves (one inverted diagonal block)
constexpr int kSolveRows = 64;       // rows per CTA of the backward large-front partial sums
constexpr int kMrhsRows = 64;        // rows per CTA of the many-RHS backward partial sums
static_assert(kSolveRows >= kMrhsRows, "solve scratch is sized for kMrhsRows-row chunks");

// Trailing-update work of panel step s of a front (columns c0 = s * kFactB
// .. c0 + w, base = c0 + w): the lower triangle of the trailing matrix (rows
// and columns >= base) in T x T tiles of width tw.  A launch covers one band
// of tile columns, given in 128-column blocks relative to base: block b holds
// tile columns [b c1, (b + 1) c1) with c1 = kFactB / tw; bhi < 0 means "to the
// end".  Block 0 is the next panel's columns.
//
// Deferred updates: the panel steps are taken in groups of `defer` (a group
// also ends at the front's last step and at the step before it, so the last,
// possibly partial, panel starts a group of its own).  Block 0 takes, at every
// step, the updates of the current group's steps so far (K range [g0 kFactB,
// base)); the other blocks take the whole group at once at its last step, and
// nothing at the others.  Every tile thus receives the same K sequence in the
// same order as with defer = 1, in fewer passes over C.
#ifdef __CUDACC__
__device__ __forceinline__ int update_grid_dev(int T, int tw, int blo, int bhi) {
  const int c1 = kFactB / tw, jlo = blo * c1;
  if (jlo >= T) return 0;
  if (bhi < 0) {
    const int t = T - jlo;
    return t * (t + 1) / 2;
  }
  return (T - jlo) * ((bhi - blo) * c1);
}
// Tile (ti, tj) handled by CTA x of a launch over band [blo, bhi).
__device__ __forceinline__ bool select_tile(int T, int tw, int blo, int bhi, int x, int& ti, int& tj) {
  const int c1 = kFactB / tw, jlo = blo * c1;
  if (jlo >= T) return false;
  if (bhi < 0) {                              // the sub-triangle of tile columns >= jlo, row by row
    const int t = T - jlo;
    if (x >= t * (t + 1) / 2) return false;
    int i = (int)((sqrtf(8.0f * (float)x + 1.0f) - 1.0f) * 0.5f);
    while ((i + 1) * (i + 2) / 2 <= x) ++i;
    while (i * (i + 1) / 2 > x) --i;
    ti = jlo + i;
    tj = jlo + (x - i * (i + 1) / 2);
    return true;
  }
  const int wdt = (bhi - blo) * c1;
  ti = jlo + x / wdt;
  tj = jlo + x % wdt;
  return ti < T && tj <= ti;
}
// K range [kbeg, kend) (front columns) that tile column tj of step `step`
// applies; false: nothing to apply at this step.
__device__ __forceinline__ bool update_k_range(int nc, int step, int defer, int tj, int tw, int& kbeg, int& kend) {
  const int last = (nc - 1) / kFactB;
  const int g0 = step >= last ? last : (step / defer) * defer;
  const bool bulk = (step + 1) % defer == 0 || step >= last - 1;
  if (tj * tw >= kFactB && !bulk) return false;
  kbeg = g0 * kFactB;
  kend = min(nc, (step + 1) * kFactB);
  return true;
}
#endif

// Programmatic dependent launch: a kernel launched with `pdl` may start while
// the previous kernel of its stream is still running; it calls pdl_wait()
// before touching anything that kernel writes (work that does not depend on
// it goes first), and pdl_trigger(), always issued after pdl_wait() so that
// every older kernel has completed, lets the next kernel start early.  Both
// are no-ops for a kernel launched without the attribute.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
#endif
template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                     Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Opt every shared-memory-heavy kernel into the large dynamic shared memory
// carve-out; called once per process before any launch or capture.
cudaError_t prepare_kernels();

// ---- index maps (built once per handle) ------------------------------------
void launch_local_index(const DevFronts& F, int32_t* local, int num_front, cudaStream_t st);
void launch_assembly_map(const DevFronts& F, const int32_t* col_front, const int32_t* acol_ptr, const int32_t* arow,
                         const int32_t* ccs_src, int32_t* sidx, int32_t* a_src, int32_t* a_pos, int n_total,
                         cudaStream_t st);
void launch_bli_count(const DevFronts& F, const int32_t* fronts, int count, int nb, int32_t* groups, cudaStream_t st);
void launch_bli_fill(const DevFronts& F, const int32_t* fronts, int count, int nb, const int32_t* group_base,
                     const int32_t* index_base, int32_t* block_ptr, int32_t* pnum, int32_t* cnum, int32_t* offset,
                     int32_t* rebuilt, cudaStream_t st);

// ---- factorization -----------------------------------------------------------
template <typename T>
void launch_small_fronts(const DevFronts& F, const int32_t* list, int count, int nf_max, const double* a, T* panel,
                         T* upool, int32_t* info, cudaStream_t st);
template <typename T>
void launch_zero_large(const DevFronts& F, const int32_t* list, int count, int64_t max_cols, T* panel, T* upool,
                       cudaStream_t st);
template <typename T>
void launch_assemble_large(const DevFronts& F, const int32_t* list, int count, int max_entries, const double* a,
                           T* panel, cudaStream_t st);
template <typename T>
void launch_extend_add(const DevFronts& F, const int32_t* list, int count, int max_nr, T* panel, T* upool,
                       cudaStream_t st);
// Panel step s of the blocked large-front factorization (columns s*kFactB ..):
//   potrf  : one CTA per front; L11 into the panel, L11^{-1} into linv (at DevFronts::d_off, or
//            one 128 x 128 slot per list entry when d_off is null)
//   trsm   : rows below the diagonal block, X <- X L11^{-T}   (kind 0: DMMA, 1: FMA)
//   update : trailing lower triangle -= P P^T                  (kind 0: DMMA 128-tiles, 1: FMA 64-tiles)
// info_stride 0: the first bad pivot of any front goes to info[0] (atomic min); 1: list slot i's to info[i].
// FP32: the diagonal sub-blocks' pivot chains run in FP32 with an FP64 fallback on a small pivot;
// fallbacks (may be null) counts the sub-blocks redone in FP64.
template <typename T>
// cls (may be null: one launch): four counts splitting the list, in order, into fronts whose
// block needs 4, 3, 2, 1 sub-blocks of 32 columns, each class launched with its own (smaller)
// shared memory and thread count; only for persistent inverse blocks (F.d_off).
void launch_potrf(const DevFronts& F, const int32_t* list, int count, int step, T* panel, T* linv, int32_t* info,
                  cudaStream_t st, bool pdl = false, int info_stride = 0, int32_t* fallbacks = nullptr,
                  const int32_t* cls = nullptr);
// q (FP32 only, may be null): also write the solved rows as packed TF32 operands of the
// tensor-core update (packed_offset below), at q + F.q_off[f].
template <typename T>
void launch_trsm(const DevFronts& F, const int32_t* list, int count, int step, int row_blocks, T* panel,
                 const T* linv, int kind, cudaStream_t st, bool pdl = false, float* q = nullptr);
// Trailing update of step `step` over the tile-column band [blo, bhi) (128-column blocks relative to
// the trailing matrix, bhi < 0: to the end; see select_tile) with updates deferred over groups of
// `defer` steps (update_k_range).  T128 / T64: the largest front's trailing tiles per side.
struct UpdBand {
  int blo = 0, bhi = -1;
};
// Returns the number of kernels launched (0 when the band is empty).
template <typename T>
int launch_update(const DevFronts& F, const int32_t* list, int count, int step, int T128, int T64, T* panel,
                  T* upool, int kind, cudaStream_t st, UpdBand band = {}, int defer = 1, bool pdl = false);
// FP32 trailing update on the tcgen05 tensor cores (update_tc.cu): split = 1 for 3xTF32, 0 for 1xTF32;
// err[0] is raised if a bounded wait expires; err[1] != 0 (read only) asks every CTA to wait on an
// mbarrier nothing arrives at, with a short limit, so that err[0] is raised (a test of the expiry path).
cudaError_t prepare_update_tc();
int launch_update_tc(const DevFronts& F, const int32_t* list, int count, int step, int T128, float* panel,
                     float* upool, int split, int32_t* err, cudaStream_t st, UpdBand band = {}, int defer = 1,
                     bool pdl = false);
// Packed operands of the FP32 tensor-core update, written by the TRSM of a panel step: the
// step's solved rows below the diagonal block, in 128-row blocks rb (rows base + 128 rb ..,
// base = first row below the block), each as 16 K chunks of 8 columns, each chunk a TF32 hi
// block then a lo block (x - hi), 1024 floats each in the canonical K-major no-swizzle UMMA
// layout (8-row x 16-byte core matrices; 16 bytes between the two k-cores, 256 between
// 8-row groups).  Columns past the block width are zero.  Two buffers, by step parity.
constexpr int64_t kPackedBlockElems = 16 * 2 * 1024;   // one 128-row block: 16 chunks x (hi, lo)
#ifdef __CUDACC__
__host__ __device__ constexpr int64_t packed_block_elems() { return kPackedBlockElems; }
__device__ __forceinline__ int64_t packed_offset(int row, int k, int hl) {   // row, k: 0-based within the step
  const int rb = row >> 7, r = row & 127, kc = k >> 3, kk = k & 7;
  return (int64_t)rb * packed_block_elems() + (int64_t)((kc * 2 + hl) * 1024) + (r >> 3) * 64 + (r & 7) * 4 +
         (kk >> 2) * 32 + (kk & 3);
}
#endif
// Trailing update of an FP32 step with deferral depth 1 from the packed operands q (this
// step's parity buffer): warp-specialised tcgen05 pipeline (update_tc.cu).
cudaError_t prepare_update_tcq();
int launch_update_tcq(const DevFronts& F, const int32_t* list, int count, int step, int T128, const float* q,
                      float* panel, float* upool, int split, int32_t* err, cudaStream_t st, UpdBand band = {},
                      bool pdl = false);
// grid size of an update launch over a band of the T x T lower tiles of width tw
int update_grid(int T, int tw, UpdBand band);

// ---- solves --------------------------------------------------------------------
// Small fronts (one size bin, nf <= nf_max <= kSmallFrontMax): one warp per front.
template <typename T>
void launch_fwd_small(const DevFronts& F, const int32_t* list, int count, int nf_max, const T* panel, T* X,
                      int64_t ldx, T* V, int nrhs, cudaStream_t st);
template <typename T>
void launch_bwd_small(const DevFronts& F, const int32_t* list, int count, int nf_max, const T* panel, T* X,
                      int64_t ldx, int nrhs, cudaStream_t st);
// Large fronts: dinv holds the inverted 128 x 128 diagonal blocks the factorization kept (DevFronts::d_off).
// fused: only the gather runs here (single right-hand side; launch_large_fused does the steps)
template <typename T>
void launch_fwd_large(const DevFronts& F, const int32_t* list, int count, int max_nc, int max_nf, const T* panel,
                      const T* dinv, T* X, int64_t ldx, T* V, int32_t* cnt, int nrhs, cudaStream_t st,
                      int64_t* launches, bool pdl, bool fused = false);
// cnt: one zero-initialised ticket per list slot (left zero again on exit)
template <typename T>
void launch_bwd_large(const DevFronts& F, const int32_t* list, int count, int max_nc, int max_nf, const T* panel,
                      const T* dinv, T* X, int64_t ldx, T* V, T* scratch, int32_t* cnt, int nrhs, cudaStream_t st,
                      int64_t* launches, bool pdl, bool fused = false);
// A level's single-RHS large-front sweep as one launch over its task list (4 ints per task:
// front, code, flag base, 0; forward code >= 0: diagonal block, < 0: rest rows chunk -1 - code;
// backward code: column block).  ticket: zero before the launch; flags: zero before the sweep
// (one per front and panel step); expired: raised when a bounded wait gives up.
// test_req (read once per CTA): nonzero makes every wait run out after ~1 ms (a test of the
// expiry path).
// Backward: tasks with code < 0 are partial sums of update-row chunk j (kBwdRestRows rows)
// against column block s (code = -1 - (s << 16 | j)), written to part (front base in the
// task's fourth int) and counted in counters (one per front and step); code >= 0 is the
// column block, which sums its chunks' partials in chunk order.
constexpr int kBwdRestRows = 256;
template <typename T>
void launch_large_fused(const DevFronts& F, const int4* tasks, int ntask, bool backward, int32_t* ticket,
                        int32_t* flags, int32_t* expired, const T* panel, const T* dinv, T* X, T* V, cudaStream_t st,
                        const int32_t* test_req, T* part = nullptr, int32_t* counters = nullptr);
// pdl: the single-RHS step kernels go out with programmatic dependent launch
// (each waits for its predecessor before reading the sweep's vectors)

// ---- vectors, residuals ---------------------------------------------------------
template <typename T>
void launch_permute_in(const double* b, int64_t ldb, const int32_t* perm_global, T* X, int64_t ldx, int64_t n,
                       int nrhs, cudaStream_t st);
template <typename T>
void launch_permute_out(const T* X, int64_t ldx, const int32_t* perm_global, double* b, int64_t ldb, int64_t n,
                        int nrhs, cudaStream_t st);
void launch_gather_values(const double* a, const int32_t* src, double* out, int64_t count, cudaStream_t st);
// r = b - A x (permuted full CSR, FP64), with |A| |x| row sums for the backward error
void launch_residual(const int64_t* rowptr, const int32_t* col, const double* val, const double* x, const double* b,
                     double* r, int64_t n, cudaStream_t st);
// out[0]=max|r|, out[1]=max|x|, out[2]=max|b|, out[3]=sum r^2, out[4]=sum x^2 (per column 0 of nrhs)
void launch_norms(const double* r, const double* x, const double* b, int64_t n, double* out, cudaStream_t st);
// k columns at once (x column-major, ld n; xt: n x k scratch): r = b - A x and
// the per-column norms into out + 8 c
void launch_residual_multi(const int64_t* rowptr, const int32_t* col, const double* val, const double* x,
                           double* xt, const double* b, double* r, int64_t n, int k, double* out, cudaStream_t st);
void launch_row_abs_max(const int64_t* rowptr, const double* val, int64_t n, double* out, cudaStream_t st);
template <typename T>
void launch_to_t(const double* in, T* out, int64_t n, cudaStream_t st);
template <typename T>
void launch_axpy_from_t(const T* d, double* x, int64_t n, cudaStream_t st);
void launch_fill_int(int32_t* p, int32_t v, int64_t n, cudaStream_t st);
// a[i] = map[a[i]] for i < n
void launch_remap_int(const int32_t* map, int32_t* a, int64_t n, cudaStream_t st);

// Device-side refinement control (the FP32 + FP64 refinement loop as a graph
// WHILE node).  State: st_i[0] sweeps done, st_i[1] 1 while refining;
// st_d[0] the worst column's backward error, st_d[1] its residual_ref; prev[c]
// each column's previous backward error.  ir_init resets it; ir_check, after a
// sweep's residual norms (out + 8 c as launch_norms / launch_residual_multi
// write them) and with anorm = max_i sum_j |a_ij|, applies the host loop's test
// -- stop when every column is below tol, or from the fourth sweep on when
// every column above tol has gained less than 10%, or after maxit sweeps --
// and sets the WHILE node's condition.
void launch_ir_init(int32_t* st_i, double* st_d, double* prev, int nrhs, cudaStream_t st);
void launch_ir_check(const double* norms, const double* anorm, int nrhs, double tol, int maxit, double* prev,
                     int32_t* st_i, double* st_d, cudaGraphConditionalHandle cond, cudaStream_t st);

}  // namespace mfd
