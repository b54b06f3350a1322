// sm_100a kernels of the multifrontal numeric phase.
//
// Index maps (built once):      local_index, supernodal_index + assembly map,
//                               block_local_index (reference tiling, export only)
// Factorization, per tree level: fused kernels for small fronts (assembly +
//                               extend-add + partial Cholesky on chip: one warp
//                               per front up to 32 rows, one CTA per front up to
//                               128 with the trailing update on DMMA tiles);
//                               blocked global-memory path for large fronts
//                               (zero, assemble, extend-add per child rank, panel
//                               POTRF+TRSM, trailing SYRK/GEMM on the FP64 tensor
//                               pipe (DMMA), tcgen05 3xTF32 (update_tc.cu) or
//                               FFMA tiles)
// Solves:                       forward/backward per level with the same split
//                               (one warp per small front; 128-column steps with
//                               the kept inverted diagonal blocks for large ones)
// Residual / norms:             FP64 CSR SpMV for iterative refinement.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <type_traits>

#include "kernels.cuh"

namespace mfd {

namespace {

__device__ __forceinline__ int lower_bound_dev(const int32_t* a, int n, int32_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}


template <typename T>
__device__ __forceinline__ T rsqrt_t(T x);
template <>
__device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt(x); }
template <>
__device__ __forceinline__ float rsqrt_t<float>(float x) { return rsqrtf(x); }

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc, bool valid) {

  unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
  int sz = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename T>
__device__ __forceinline__ void cp_async_t(T* dst, const T* src, bool valid) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = valid ? (int)sizeof(T) : 0;
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(src), "r"(sz));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(src), "r"(sz));
}

// Extend-add of one child's lower update triangle into a front held in shared
// memory by `nthreads` threads starting at t0 (a multiple of 32 threads):
// thread (row lane tx, column group ty) takes columns ty, ty + ny, ... and in
// each the rows i >= j of its lane (no division, lower triangle only; the
// unrolled row loop keeps several loads in flight).  The child's local_index
// is first staged in shared memory (sloc, nrc entries) by the caller.
// local_index is injective, so no two entries of one child share a target.
// Packed lower storage (ldS < 0, nf = -ldS): column j starts at
// j nf - j (j + 1) / 2 and holds rows j .. nf-1.
__device__ __forceinline__ int packed_col(int j, int nf) { return j * nf - j * (j + 1) / 2; }

// S(local) += U for one child's update matrix U (nrc x nrc, lower triangle,
// column-major) through its staged local_index sloc: lanes over rows, warps
// over columns, CU columns x RI row passes of loads issued together per
// chunk (predicated, no early exit), then the shared-memory adds.  ldS > 0:
// S column-major with leading dimension ldS; ldS < 0: S packed (nf = -ldS).
template <typename T, int RI, int CU>
__device__ __forceinline__ void extend_add_chunk(T* S, int ldS, const T* __restrict__ U, const int* sloc, int nrc,
                                                 int tx, int ty, int ny) {
  for (int j0 = ty; j0 < nrc; j0 += CU * ny) {
    T u[CU][RI];
#pragma unroll
    for (int c = 0; c < CU; ++c) {
      const int j = j0 + c * ny;
#pragma unroll
      for (int v = 0; v < RI; ++v) {
        const int i = j + tx + 32 * v;
        u[c][v] = (j < nrc && i < nrc) ? U[(size_t)j * nrc + i] : T(0);
      }
    }
#pragma unroll
    for (int c = 0; c < CU; ++c) {
      const int j = j0 + c * ny;
      if (j < nrc) {
        const int lj = sloc[j] - 1;
        const int base = ldS > 0 ? lj * ldS : packed_col(lj, -ldS);
#pragma unroll
        for (int v = 0; v < RI; ++v) {
          const int i = j + tx + 32 * v;
          if (i < nrc) S[base + sloc[i] - 1] += u[c][v];
        }
      }
    }
  }
}
// The same scatter with one column per warp step (lanes over rows): the
// one-CTA-per-front kernel, whose 8 warps already keep 8 columns in flight.
template <typename T>
__device__ __forceinline__ void extend_add_cols(T* S, int ldS, const T* __restrict__ U, const int* sloc, int nrc,
                                                int t0, int nthreads) {
  const int tx = t0 & 31, ty = t0 >> 5, ny = nthreads >> 5;
  for (int j = ty; j < nrc; j += ny) {
    const int lj = sloc[j] - 1;
    const int base = ldS > 0 ? lj * ldS : packed_col(lj, -ldS);
    const T* Uc = U + (size_t)j * nrc;
#pragma unroll 4
    for (int i = j + tx; i < nrc; i += 32) S[base + sloc[i] - 1] += Uc[i];
  }
}
// NB: loads in flight per thread and chunk (register budget)
template <int NB, typename T>
__device__ __forceinline__ void extend_add_smem(T* S, int ldS, const T* __restrict__ U, const int* sloc, int nrc,
                                                int t0, int nthreads) {
  const int tx = t0 & 31, ty = t0 >> 5, ny = nthreads >> 5;
  switch ((nrc + 31) >> 5) {                 // row passes a column needs (nrc <= 128)
    case 0: break;
    case 1: extend_add_chunk<T, 1, NB>(S, ldS, U, sloc, nrc, tx, ty, ny); break;
    case 2: extend_add_chunk<T, 2, (NB / 2 > 0 ? NB / 2 : 1)>(S, ldS, U, sloc, nrc, tx, ty, ny); break;
    case 3: extend_add_chunk<T, 3, (NB / 3 > 0 ? NB / 3 : 1)>(S, ldS, U, sloc, nrc, tx, ty, ny); break;
    default: extend_add_chunk<T, 4, (NB / 4 > 0 ? NB / 4 : 1)>(S, ldS, U, sloc, nrc, tx, ty, ny); break;
  }
}

// A's entries of front f into its shared buffer (entry position pos = row +
// col * nf, row >= col, placed at S[addr(row, col)]), U entries per thread
// with their loads in flight together
template <int UN, typename T, typename Addr>
__device__ __forceinline__ void assemble_smem(const DevFronts& F, int f, int nf, const double* __restrict__ a, T* S,
                                              Addr addr, int t0, int nthreads) {
  const int a0 = F.a_beg[f], a1 = F.a_beg[f + 1];
  for (int k0 = a0 + t0; k0 < a1; k0 += UN * nthreads) {
    int pos[UN], src[UN];
#pragma unroll
    for (int u = 0; u < UN; ++u) {
      const int k = k0 + u * nthreads;
      pos[u] = k < a1 ? F.a_pos[k] : -1;
      src[u] = k < a1 ? F.a_src[k] : 0;
    }
    double v[UN];
#pragma unroll
    for (int u = 0; u < UN; ++u) v[u] = pos[u] >= 0 ? a[src[u]] : 0.0;
#pragma unroll
    for (int u = 0; u < UN; ++u)
      if (pos[u] >= 0) {
        const int c = pos[u] / nf, r = pos[u] - c * nf;
        S[addr(r, c)] = T(v[u]);
      }
  }
}

// Strided element loop (e = threadIdx.x, += blockDim.x, e < total) whose
// global loads are issued kBatch at a time before the matching stores, so a
// thread keeps kBatch independent loads in flight instead of one.
constexpr int kBatch = 16;
template <typename Load, typename Store>
__device__ __forceinline__ void batched_loop(int total, Load&& load, Store&& store) {
  using V = decltype(load(0));
  for (int e0 = threadIdx.x; e0 < total; e0 += blockDim.x * kBatch) {
    V v[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int e = e0 + u * (int)blockDim.x;
      v[u] = e < total ? load(e) : V(0);
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int e = e0 + u * (int)blockDim.x;
      if (e < total) store(e, v[u]);
    }
  }
}
inline int clamp_grid(int64_t g, int64_t cap = 65535) { return (int)std::max<int64_t>(1, std::min<int64_t>(g, cap)); }

// ============================================================================
// index maps
// ============================================================================

// local_index (create_local_index_m.f90:10-45): for every L row r of child c,
// its 1-based position in the parent front: the parent's own column r-first+1,
// or nc_p + (position of r in the parent's sorted L rows).
__global__ void k_local_index(DevFronts F, int32_t* local, int num_front) {
  int c = blockIdx.x;
  if (c >= num_front) return;
  int p = F.parent[c];
  if (p < 0) return;
  int nrc = F.nr[c], off = F.lrow_off[c];
  int fp = F.first[p], ncp = F.nc[p], nrp = F.nr[p];
  const int32_t* lp = F.lrow + F.lrow_off[p];
  for (int i = threadIdx.x; i < nrc; i += blockDim.x) {
    int r = F.lrow[off + i];
    int pos;
    if (r < fp + ncp) {
      pos = r - fp;
    } else {
      int q = lower_bound_dev(lp, nrp, r);
      pos = (q < nrp && lp[q] == r) ? ncp + q : -1;      // -1: structure violation -> 0
    }
    local[off + i] = pos + 1;
  }
}

// supernodal_index (create_supernodal_index_m.f90:10-40) and the assembly map:
// one thread per permuted column; every A entry gets its front position
// (1-based, the reference's value), the source index of its value and its
// offset row + col*nf inside the front's panel.
__global__ void k_assembly_map(DevFronts F, const int32_t* col_front, const int32_t* acol_ptr, const int32_t* arow,
                               const int32_t* ccs_src, int32_t* sidx, int32_t* a_src, int32_t* a_pos, int n_total) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n_total) return;
  int f = col_front[col];
  int first = F.first[f], nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  const int32_t* lr = F.lrow + F.lrow_off[f];
  int jloc = col - first;
  for (int k = acol_ptr[col]; k < acol_ptr[col + 1]; k++) {
    int r = arow[k];
    int pos;
    if (r < first + nc) {
      pos = r - first;
    } else {
      int q = lower_bound_dev(lr, nr, r);
      pos = (q < nr && lr[q] == r) ? nc + q : -1;
    }
    sidx[k] = pos + 1;
    a_src[k] = ccs_src[k];
    a_pos[k] = pos < 0 ? 0 : pos + jloc * nf;
  }
}

// block_local_index (block_local_index_creator_m.f90:13-122): a group is a
// maximal run of a child's local index with constant (parent tile, child tile).
__device__ __forceinline__ void bli_key(int loc, int i, int ncc, int nb, int& pt, int& ct) {
  pt = (loc - 1) / nb + 1;            // get_matrix_num(local(i))
  ct = (ncc + i) / nb + 1;            // get_work_num(i+1, node) = get_matrix_num(nc + i + 1)
}

__global__ void k_bli_count(DevFronts F, const int32_t* fronts, int count, int nb, int32_t* groups) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  int c = fronts[t];
  int g = 0;
  if (F.parent[c] >= 0) {
    int nrc = F.nr[c], ncc = F.nc[c], pp = 0, pc = 0;
    const int32_t* loc = F.local + F.lrow_off[c];
    for (int i = 0; i < nrc; i++) {
      int pt, ct;
      bli_key(loc[i], i, ncc, nb, pt, ct);
      if (pt != pp || ct != pc) { pp = pt; pc = ct; g++; }
    }
  }
  groups[t] = g;
}

__global__ void k_bli_fill(DevFronts F, const int32_t* fronts, int count, int nb, const int32_t* group_base,
                           const int32_t* index_base, int32_t* block_ptr, int32_t* pnum, int32_t* cnum,
                           int32_t* offset, int32_t* rebuilt) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  int c = fronts[t];
  int nrc = F.nr[c], ncc = F.nc[c];
  const int32_t* loc = F.local + F.lrow_off[c];
  int ibase = index_base[t];
  for (int i = 0; i < nrc; i++) rebuilt[ibase + i] = (loc[i] - 1) % nb + 1;        // rebuild_val: mod2(local, nb)
  if (F.parent[c] < 0) return;
  int ss = ncc % nb;                                                                // border_supernode_size
  int ws = min(nb - ss, nrc);                                                       // border_work_size
  int g = group_base[t] - 2, pp = 0, pc = 0;                                       // 0-based, before the first group
  for (int i = 0; i < nrc; i++) {
    int pt, ct;
    bli_key(loc[i], i, ncc, nb, pt, ct);
    if (pt != pp || ct != pc) {
      pp = pt; pc = ct; g++;
      pnum[g] = pt;
      cnum[g] = ct;
      block_ptr[g] = ibase + i + 1;                                                 // 1-based start of the group
      int s = i + 1;                                                                // get_start_row_num
      offset[g] = s <= ws ? s - 1 : (ss + s - 1) % nb;                              // get_block_offset
    }
  }
}

// ============================================================================
// factorization
// ============================================================================

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

constexpr int kSfW = 8;   // panel width of the small-front elimination

// Fused small front: zero, assemble A, extend-add the children in order, partial
// Cholesky of the nc supernode columns and the Schur complement, all in shared
// memory; writes the factor panel and the update matrix once.
// Launched with 128 threads per front.  BIG (fronts of 65..128 rows, the
// upper levels, few fronts per launch): up to 128 registers per thread and the
// children's update columns loaded 16 at a time per thread; otherwise 32
// registers (16 CTAs per SM by registers, shared memory binds first) and one
// child column per warp step.
template <typename T, bool BIG>
__global__ void __launch_bounds__(128, BIG ? 4 : 16) k_small_front(DevFronts F, const int32_t* list, const double* __restrict__ a,
                                                     T* __restrict__ panel, T* __restrict__ upool, int32_t* info) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S = reinterpret_cast<T*>(smem_raw);     // the front's lower triangle, packed by columns
  const int f = list[blockIdx.x];
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  const int tri = nf * (nf + 1) / 2;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;

  // shared memory: the packed front (tri), kSfW pivot scales, a child's
  // local_index (nf ints)
  int* sloc = reinterpret_cast<int*>(S + tri + kSfW);
  for (int i = tid; i < tri; i += nt) S[i] = T(0);
  __syncthreads();
  for (int k = F.a_beg[f] + tid; k < F.a_beg[f + 1]; k += nt) {
    const int pos = F.a_pos[k];
    const int c = pos / nf, r = pos - c * nf;          // r >= c: the lower part of A
    S[packed_col(c, nf) + r] = T(a[F.a_src[k]]);
  }
  __syncthreads();
  for (int t = F.child_ptr[f]; t < F.child_ptr[f + 1]; ++t) {
    const int c = F.child[t];
    const int nrc = F.nr[c];
    const int32_t* loc = F.local + F.lrow_off[c];
    for (int i = tid; i < nrc; i += nt) sloc[i] = loc[i];
    __syncthreads();
    if constexpr (BIG) extend_add_smem<16>(S, -nf, upool + F.u_off[c], sloc, nrc, tid, nt);
    else extend_add_cols(S, -nf, upool + F.u_off[c], sloc, nrc, tid, nt);
    __syncthreads();
  }
  // blocked right-looking elimination, panels of kSfW columns, three barriers
  // per panel: (1) lanes 0..w-1 of warp 0 factor the w x w diagonal block in
  // registers (lane = row, pivots by shuffles); (2) every thread solves rows
  // of the block column below it, l_ip = (a_ip - sum_{p'<p} l_ip' L_pp') y_p;
  // (3) the rank-w update S_ij -= sum_p L_ip L_jp of the trailing triangle
  // (FP64: 8 x 8 tiles on m8n8k4 DMMA, one warp per tile; FP32: warps over
  // columns, lanes over rows)
  T* ys = S + tri;                           // the panel's pivot scales y_p = 1/sqrt(d_p)
  for (int k0 = 0; k0 < nc; k0 += kSfW) {
    const int w = min(kSfW, nc - k0);
    int pc[kSfW];
#pragma unroll
    for (int p = 0; p < kSfW; ++p) pc[p] = packed_col(k0 + min(p, w - 1), nf);
    if (warp == 0) {
      T rv[kSfW];
      const int r = k0 + lane;
#pragma unroll
      for (int p = 0; p < kSfW; ++p) rv[p] = (lane < w && p < w && p <= lane) ? S[pc[p] + r] : T(0);
#pragma unroll
      for (int p = 0; p < kSfW; ++p) {
        if (p < w) {
          T d = __shfl_sync(0xffffffffu, rv[p], p);
          if (!(d > T(0))) {
            if (lane == 0) atomicMin(info, F.first[f] + k0 + p + 1);
            d = T(1);
          }
          const T y = rsqrt_t<T>(d);
          if (lane > p) rv[p] *= y;
          else if (lane == p) { rv[p] = d * y; ys[p] = y; }
#pragma unroll
          for (int p2 = p + 1; p2 < kSfW; ++p2) {
            if (p2 < w) {
              const T lj = __shfl_sync(0xffffffffu, rv[p], p2);
              if (lane >= p2) rv[p2] -= rv[p] * lj;
            }
          }
        }
      }
      if (lane < w) {
#pragma unroll
        for (int p = 0; p < kSfW; ++p)
          if (p <= lane) S[pc[p] + r] = rv[p];
      }
    }
    __syncthreads();
    for (int i = k0 + w + tid; i < nf; i += nt) {
      T x[kSfW];
#pragma unroll
      for (int p = 0; p < kSfW; ++p) x[p] = p < w ? S[pc[p] + i] : T(0);
#pragma unroll
      for (int p = 0; p < kSfW; ++p) {
        if (p < w) {
          T v = x[p];
#pragma unroll
          for (int q = 0; q < p; ++q) v -= x[q] * S[pc[q] + k0 + p];
          x[p] = v * ys[p];
        }
      }
#pragma unroll
      for (int p = 0; p < kSfW; ++p)
        if (p < w) S[pc[p] + i] = x[p];
    }
    __syncthreads();
    const int kb = k0 + w;                   // the trailing triangle: rows and columns [kb, nf)
    if constexpr (std::is_same<T, double>::value) {
      const int t8 = (nf - kb + 7) >> 3, tiles = t8 * (t8 + 1) / 2;
      const int g = lane >> 2, q = lane & 3;
      for (int t = warp; t < tiles; t += nw) {
        int ti = 0;                          // tile (ti, tj), ti >= tj, row-major over the lower triangle
        while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
        const int tj = t - ti * (ti + 1) / 2;
        const int i0 = kb + 8 * ti, j0 = kb + 8 * tj;
        const int ia = i0 + g, jb = j0 + g;  // the row of A and the column of B this lane feeds
        double c[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = j0 + 2 * q + e;
          c[e] = (ia < nf && j < nf && ia >= j) ? S[packed_col(j, nf) + ia] : 0.0;
        }
#pragma unroll
        for (int s4 = 0; s4 < kSfW; s4 += 4) {
          const int p = s4 + q;
          const double av = (p < w && ia < nf) ? -S[pc[p] + ia] : 0.0;
          const double bv = (p < w && jb < nf) ? S[pc[p] + jb] : 0.0;
          dmma(c[0], c[1], av, bv);
        }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = j0 + 2 * q + e;
          if (ia < nf && j < nf && ia >= j) S[packed_col(j, nf) + ia] = c[e];
        }
      }
    } else {
      for (int j = kb + warp; j < nf; j += nw) {
        T lj[kSfW];
#pragma unroll
        for (int p = 0; p < kSfW; ++p) lj[p] = p < w ? S[pc[p] + j] : T(0);
        T* colj = S + packed_col(j, nf);
        for (int i = j + lane; i < nf; i += 32) {
          T acc = colj[i];
#pragma unroll
          for (int p = 0; p < kSfW; ++p)
            if (p < w) acc -= S[pc[p] + i] * lj[p];
          colj[i] = acc;
        }
      }
    }
    __syncthreads();
  }
  T* P = panel + F.panel_off[f];
  for (int j = warp; j < nc; j += nw)
    for (int i = j + lane; i < nf; i += 32) P[i + (size_t)j * nf] = S[packed_col(j, nf) + i];
  T* U = upool + F.u_off[f];
  for (int j = warp; j < nr; j += nw)
    for (int i = j + lane; i < nr; i += 32) U[i + (size_t)j * nr] = S[packed_col(nc + j, nf) + nc + i];
}

// Zero the lower triangles of a large front's panel (nf x nc) and update
// matrix (nr x nr): one warp per column, grid-stride over columns.
template <typename T>
__global__ void k_zero_large(DevFronts F, const int32_t* list, T* panel, T* upool) {
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  T* P = panel + F.panel_off[f];
  T* U = upool + F.u_off[f];
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = blockIdx.x * nw + (threadIdx.x >> 5); j < nc + nr; j += gridDim.x * nw) {
    if (j < nc) {
      T* col = P + (size_t)j * nf;
      for (int i = j + lane; i < nf; i += 32) col[i] = T(0);
    } else {
      const int jj = j - nc;
      T* col = U + (size_t)jj * nr;
      for (int i = jj + lane; i < nr; i += 32) col[i] = T(0);
    }
  }
}

template <typename T>
__global__ void k_assemble_large(DevFronts F, const int32_t* list, const double* __restrict__ a, T* panel) {
  const int f = list[blockIdx.y];
  T* P = panel + F.panel_off[f];
  for (int k = F.a_beg[f] + blockIdx.x * blockDim.x + threadIdx.x; k < F.a_beg[f + 1]; k += gridDim.x * blockDim.x)
    P[F.a_pos[k]] = T(a[F.a_src[k]]);
}

// Extend-add of one child per parent (children of one rank, so no two CTAs of a
// launch write the same parent entry): warp per child column, lanes over rows.
template <typename T>
__global__ void __launch_bounds__(256) k_extend_add(DevFronts F, const int32_t* list, T* panel, T* upool) {
  const int c = list[blockIdx.y];
  const int p = F.parent[c];
  const int nrc = F.nr[c];
  const int ncp = F.nc[p], nrp = F.nr[p], nfp = ncp + nrp;
  const T* __restrict__ Uc = upool + F.u_off[c];
  T* Pp = panel + F.panel_off[p];
  T* Up = upool + F.u_off[p];
  const int32_t* __restrict__ loc = F.local + F.lrow_off[c];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = blockIdx.x * nw + warp; j < nrc; j += gridDim.x * nw) {
    const int lj = loc[j] - 1;
    const T* src = Uc + (size_t)j * nrc;
    if (lj < ncp) {
      T* dst = Pp + (size_t)lj * nfp;
      for (int i = j + lane; i < nrc; i += 32) dst[loc[i] - 1] += src[i];
    } else {
      T* dst = Up + (size_t)(lj - ncp) * nrp - ncp;
      for (int i = j + lane; i < nrc; i += 32) dst[loc[i] - 1] += src[i];
    }
  }
}

// FP32 form: warps take column pairs (j, nrc-1-j), nrc + 1 entries per pair,
// lanes over rows with four rows per lane in flight (the source and
// local-index reads, then the parent reads, then the stores).  Measured on the
// 64^3 Laplacian: FP32 4.1 -> 2.9 ms per factorization; for FP64 (twice the
// bytes per entry, already near the bandwidth the scatter reaches) the same
// scheme was slower (5.0 -> 5.6 ms), so FP64 keeps the kernel above.
template <typename T>
__global__ void __launch_bounds__(256) k_extend_add_ilp(DevFronts F, const int32_t* list, T* panel, T* upool) {
  const int c = list[blockIdx.y];
  const int p = F.parent[c];
  const int nrc = F.nr[c];
  const int ncp = F.nc[p], nrp = F.nr[p], nfp = ncp + nrp;
  const T* __restrict__ Uc = upool + F.u_off[c];
  T* Pp = panel + F.panel_off[p];
  T* Up = upool + F.u_off[p];
  const int32_t* __restrict__ loc = F.local + F.lrow_off[c];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int ntask = (nrc + 1) / 2;
  for (int q = blockIdx.x * nw + warp; q < ntask; q += gridDim.x * nw) {
#pragma unroll 1
    for (int hh = 0; hh < 2; ++hh) {
      const int j = hh ? nrc - 1 - q : q;
      if (hh && j == q) break;
      const int lj = __ldg(&loc[j]) - 1;
      const T* src = Uc + (size_t)j * nrc;
      T* dst = lj < ncp ? Pp + (size_t)lj * nfp : Up + (size_t)(lj - ncp) * nrp - ncp;
      for (int i0 = j + lane; i0 < nrc; i0 += 128) {
        int li[4];
        T v[4], d[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = i0 + 32 * u;
          v[u] = i < nrc ? src[i] : T(0);
          li[u] = i < nrc ? __ldg(&loc[i]) - 1 : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) d[u] = li[u] >= 0 ? dst[li[u]] : T(0);
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (li[u] >= 0) dst[li[u]] = d[u] + v[u];
      }
    }
  }
}

// ---- blocked large-front factorization: per panel step s (columns c0 = s*128) ----
//   k_potrf : one CTA per front: Cholesky of the w x w diagonal block in shared
//             memory, written back as L11, then inverted in place (lower
//             triangular) and stored as L11^{-1} in per-front scratch
//   k_trsm  : the rows below, X <- A L11^{-T} = A (L11^{-1})^T, a GEMM with K = w
//   k_update: trailing C(lower) -= P P^T with P the solved panel rows

// Diagonal-block POTRF + inverse, one CTA (8 warps) per front, w <= 128.  The
// block lives in shared memory in FP64 whatever the storage type.  FP64
// factorization: every step in FP64.  FP32 factorization: the serial pivot
// chain of each 32 x 32 diagonal sub-block (and its inverse) runs in FP32,
// with a fallback to the FP64 chain when a pivot is small (warp_chol32_f32;
// the `fallbacks` counter counts them); the sub-panel TRSM, the trailing SYRK
// and the block inverse stay on FP64 DMMA.
//
// The block (zero-padded to wp = 32 * ceil(w / 32), identity on the padded
// diagonal) sits in shared memory S, column-major, ld kPLd.  Right-looking
// over 32-wide sub-blocks b:
//   1. warp 0: Cholesky of the 32 x 32 diagonal sub-block, one row per lane,
//      pivots by shuffle, 1/sqrt by rsqrt (no division), the next column
//      updated ahead of the rest (one shuffle) so the next pivot's 1/sqrt
//      overlaps the rank-1 update, whose column broadcast goes through a
//      double-buffered shared vector; then the sub-block's inverse D_b by
//      forward substitution, one column per lane;
//   2. sub-panel below: L_ib = A_ib D_b^T, one 32-row tile per warp (DMMA);
//   3. trailing update S_ij -= L_ib L_jb^T, 32 x 32 lower tiles over the warps
//      (DMMA).
// Then the full inverse X = L^{-1}: X_bb = D_b and, per block row r,
// X_rc = -D_r (sum_{k=c}^{r-1} L_rk X_kc), two warps per block column c; the
// off-diagonal X blocks are kept in the strict upper part of S (block (c, r) holds X_rc).
// L goes to the panel, X (column-major, ld 128, zero outside the lower w x w;
// persistent blocks are zeroed at allocation and written on that part only)
// to linv.  A non-positive pivot records its 1-based column in info (atomic
// min) and continues with pivot 1.
constexpr int kPSub = 32;
constexpr int kPLd = kFactB + 4;   // 132: ld = 4 mod 16 doubles keeps DMMA fragment loads conflict-free
constexpr int kDLd = kPSub + 4;    // 36
// The kernel is instantiated per number of 32-wide sub-blocks NSB (the block
// width w <= 32 NSB): shared memory for 32 NSB columns of S (ld kPLd), NSB
// inverse blocks and NSB - 1 scratch blocks; 32 x {1, 2, 4, 8} threads, the
// most any phase uses (sub-panel TRSM: NSB - 1 warps, trailing tiles, inverse:
// 2 (NSB - 1) warps), so narrow panels fit many fronts per SM.
// scratch blocks Yv: NSB - 1 for the inverse, at least one (the FP32 pivot chain's
// 32 x 33 float copy of the sub-block lives there)
template <int NSB>
__host__ __device__ constexpr int potrf_yblocks() {
  return NSB > 1 ? NSB - 1 : 1;
}
template <int NSB>
__host__ __device__ constexpr size_t potrf_smem() {
  return sizeof(double) * ((size_t)kPSub * NSB * kPLd + (size_t)NSB * kPSub * kDLd +
                           (size_t)potrf_yblocks<NSB>() * kPSub * kDLd + kFactB + 2 * kPSub);
}
template <int NSB>
__host__ __device__ constexpr int potrf_threads() {
  return NSB == 1 ? 32 : NSB == 2 ? 64 : NSB == 3 ? 128 : 256;
}


// One warp: acc(8 MF x 32) += A(8 MF x K) B(K x 32), K a multiple of 4, operands
// in shared memory addressed as A(i, k) = A[i * ai + k * ak] and
// B(k, j) = B[k * bk + j * bj].  acc[m][n][e] holds C(8m + g, 8n + 2q + e)
// with g = lane / 4, q = lane % 4 (the m8n8k4 accumulator layout).
template <int MF>
__device__ __forceinline__ void warp_mm32(double (&acc)[MF][4][2], const double* A, int ai, int ak, const double* B,
                                          int bk, int bj, int K, int lane) {
  const int g = lane >> 2, q = lane & 3;
  for (int k = 0; k < K; k += 4) {
    double a[MF], b[4];
#pragma unroll
    for (int m = 0; m < MF; ++m) a[m] = A[(8 * m + g) * ai + (k + q) * ak];
#pragma unroll
    for (int n = 0; n < 4; ++n) b[n] = B[(k + q) * bk + (8 * n + g) * bj];
#pragma unroll
    for (int m = 0; m < MF; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n) dmma(acc[m][n][0], acc[m][n][1], a[m], b[n]);
  }
}

template <int MF>
__device__ __forceinline__ void acc_zero(double (&acc)[MF][4][2]) {
#pragma unroll
  for (int m = 0; m < MF; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n) acc[m][n][0] = acc[m][n][1] = 0.0;
}

// store s * acc at C(i, j) = C[i * ci + j * cj]
template <int MF>
__device__ __forceinline__ void acc_store(const double (&acc)[MF][4][2], double* C, int ci, int cj, double s,
                                          int lane) {
  const int g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int m = 0; m < MF; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int e = 0; e < 2; ++e) C[(8 * m + g) * ci + (8 * n + 2 * q + e) * cj] = s * acc[m][n][e];
}

// warp 0 of the CTA: Cholesky of S(o:o+32, o:o+32) in place, rsqrt of the
// pivots into rq[o..o+31], inverse of the factor into D (column-major, ld kDLd,
// zero above the diagonal).  Returns the 1-based sub-block pivot that failed, or 0.
__device__ int warp_chol32(double* S, int o, double* D, double* rq, double* cbuf, int lane) {
  double a[kPSub];
#pragma unroll
  for (int j = 0; j < kPSub; ++j) a[j] = S[(o + lane) + (o + j) * kPLd];
  int bad = 0;
  // pivot k's scale y and column l = L(lane, k) are formed one step ahead: at
  // step k the next column is updated first (one shuffle), so pivot k+1's
  // 1/sqrt overlaps the rest of step k's rank-1 update
  double d = __shfl_sync(0xffffffffu, a[0], 0);
  if (!(d > 0.0)) { bad = 1; d = 1.0; }
  double y = rsqrt(d);
  double l = a[0] * y;
#pragma unroll
  for (int k = 0; k < kPSub; ++k) {
    double* cb = cbuf + (k & 1) * kPSub;
    cb[lane] = l;
    if (lane == 0) rq[o + k] = y;
    a[k] = lane == k ? d * y : l;
    double dn = 1.0, yn = 1.0, ln = 0.0;
    if (k + 1 < kPSub) {
      a[k + 1] = fma(-l, __shfl_sync(0xffffffffu, l, k + 1), a[k + 1]);
      dn = __shfl_sync(0xffffffffu, a[k + 1], k + 1);
      if (!(dn > 0.0)) {               // uniform: every lane holds the same pivot
        if (!bad) bad = k + 2;
        dn = 1.0;
      }
      yn = rsqrt(dn);
      ln = a[k + 1] * yn;
    }
    __syncwarp();
#pragma unroll
    for (int j = k + 2; j < kPSub; ++j) a[j] = fma(-l, cb[j], a[j]);
    d = dn;
    y = yn;
    l = ln;
  }
#pragma unroll
  for (int j = 0; j < kPSub; ++j)
    if (j <= lane) S[(o + lane) + (o + j) * kPLd] = a[j];
  __syncwarp();
  // inverse: lane j owns column j of X = L^{-1}; forward substitution on e_j
  double x[kPSub];
#pragma unroll
  for (int i = 0; i < kPSub; ++i) x[i] = i == lane ? 1.0 : 0.0;
#pragma unroll
  for (int k = 0; k < kPSub; ++k) {
    x[k] *= rq[o + k];
#pragma unroll
    for (int i = k + 1; i < kPSub; ++i) x[i] = fma(-S[(o + i) + (o + k) * kPLd], x[k], x[i]);
  }
#pragma unroll
  for (int i = 0; i < kPSub; ++i) D[i + lane * kDLd] = x[i];
  return bad;
}

// The FP64 chain as the FP32 path's fallback, out of line so that its
// registers do not add to the FP32 chain's.
__device__ __noinline__ int warp_chol32_fallback(double* S, int o, double* D, double* rq, double* cbuf, int lane) {
  return warp_chol32(S, o, D, rq, cbuf, lane);
}

// FP32 form of warp_chol32 for the FP32 factorization: the pivot chain runs
// in FP32 (rsqrtf, FP32 FMAs) on the block's values as stored; the factor
// goes back to S widened to FP64 and, as FP32, to Fb (32 x 33 floats), from
// which the inverse is formed in FP32 and written to D in FP64.  A pivot is
// "small" when it is not positive or below kSmallPivot times the diagonal
// entry it started from (more than 12 of FP32's 24 significand bits
// cancelled): the function then returns -1 before writing S or D, and the
// caller redoes the sub-block with the FP64 warp_chol32 (the fallback).  The
// test is uniform across the warp (the pivot comes from a shuffle, the
// diagonal entry from shared memory).
constexpr float kSmallPivot = 1.0f / 4096.0f;
constexpr int kFbLd = kPSub + 1;
__device__ int warp_chol32_f32(double* S, int o, double* D, double* rq, float* cbuf, float* Fb, int lane) {
  float a[kPSub], dg[kPSub];
#pragma unroll
  for (int j = 0; j < kPSub; ++j) a[j] = (float)S[(o + lane) + (o + j) * kPLd];
#pragma unroll
  for (int j = 0; j < kPSub; ++j) dg[j] = __shfl_sync(0xffffffffu, a[j], j) * kSmallPivot;   // small-pivot bounds
  float d = __shfl_sync(0xffffffffu, a[0], 0);
  if (!(d > dg[0])) return -1;
  float y = rsqrtf(d);
  float l = a[0] * y;
#pragma unroll
  for (int k = 0; k < kPSub; ++k) {
    float* cb = cbuf + (k & 1) * kPSub;
    cb[lane] = l;
    if (lane == 0) rq[o + k] = (double)y;              // the FP64 fallback rewrites rq if it runs
    a[k] = lane == k ? d * y : l;
    float dn = 1.0f, yn = 1.0f, ln = 0.0f;
    if (k + 1 < kPSub) {
      a[k + 1] = fmaf(-l, __shfl_sync(0xffffffffu, l, k + 1), a[k + 1]);
      dn = __shfl_sync(0xffffffffu, a[k + 1], k + 1);
      if (!(dn > dg[k + 1])) return -1;                  // uniform: small pivot, FP64 fallback
      yn = rsqrtf(dn);
      ln = a[k + 1] * yn;
    }
    __syncwarp();
#pragma unroll
    for (int j = k + 2; j < kPSub; ++j) a[j] = fmaf(-l, cb[j], a[j]);
    d = dn;
    y = yn;
    l = ln;
  }
#pragma unroll
  for (int j = 0; j < kPSub; ++j) {
    Fb[lane + j * kFbLd] = a[j];
    if (j <= lane) S[(o + lane) + (o + j) * kPLd] = (double)a[j];
  }
  __syncwarp();
  // inverse: lane j owns column j of X = L^{-1}; forward substitution on e_j (FP32)
  float x[kPSub];
#pragma unroll
  for (int i = 0; i < kPSub; ++i) x[i] = i == lane ? 1.0f : 0.0f;
#pragma unroll
  for (int k = 0; k < kPSub; ++k) {
    x[k] *= (float)rq[o + k];
#pragma unroll
    for (int i = k + 1; i < kPSub; ++i) x[i] = fmaf(-Fb[i + k * kFbLd], x[k], x[i]);
  }
#pragma unroll
  for (int i = 0; i < kPSub; ++i) D[i + lane * kDLd] = (double)x[i];
  return 0;
}

// Inverted diagonal block of panel step `step` of front f: persistent per front
// when the plan provides d_off (kept for the solves), else one slot per list
// entry of the launch.
template <typename T>
__device__ __forceinline__ T* inv_block(const DevFronts& F, T* linv, int f, int step, int slot) {
  return F.d_off ? linv + F.d_off[f] + (size_t)step * kFactB * kFactB : linv + (size_t)slot * kFactB * kFactB;
}

// info_stride 0: every front reports into info[0]; 1: list slot i reports into info[i].
// fallbacks (may be null): counts the FP32 sub-blocks redone in FP64.
template <typename T, int NSB>
__global__ void __launch_bounds__(potrf_threads<NSB>(), 1) k_potrf(DevFronts F, const int32_t* list, int step,
                                                                   T* panel, T* linv, int32_t* info, int info_stride,
                                                                   int32_t* fallbacks) {
  constexpr int B = kPSub * NSB;                             // the block's capacity (w <= B)
  constexpr int NT = potrf_threads<NSB>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* S = reinterpret_cast<double*>(smem_raw);
  double* Dv = S + (size_t)B * kPLd;                         // NSB blocks of kPSub x kDLd
  double* Yv = Dv + (size_t)NSB * kPSub * kDLd;               // potrf_yblocks<NSB>() blocks
  double* rq = Yv + (size_t)potrf_yblocks<NSB>() * kPSub * kDLd;   // kFactB
  double* cbuf = rq + kFactB;                                 // 2 x kPSub
  const int f = list[blockIdx.x];
  const int nc = F.nc[f], nf = nc + F.nr[f];
  const int c0 = step * kFactB;
  if (c0 >= nc) return;
  const int w = min(kFactB, nc - c0);                       // <= B by the launch's choice of NSB
  const int nsb = (w + kPSub - 1) / kPSub, wp = nsb * kPSub;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  T* P = panel + F.panel_off[f];
  pdl_wait();
  pdl_trigger();          // after the wait: every kernel before this one has completed
  // ---- load the lower w x w block, identity on the padding ----
  if constexpr (sizeof(T) == 8) {
    // asynchronous 8-byte copies, all in flight at once; out-of-block entries zero-filled
    for (int e = tid; e < B * B; e += NT) {
      const int i = e % B, j = e / B;
      if (i < wp && j < wp) {
        if (i == j && i >= w) {
          S[i + j * kPLd] = 1.0;              // identity on the padded diagonal
        } else {
          const bool v = i < w && j < w && i >= j;
          cp_async8(&S[i + j * kPLd], v ? (const void*)&P[(c0 + i) + (size_t)(c0 + j) * nf] : (const void*)P, v);
        }
      }
    }
    cp_async_commit();
    cp_async_wait<0>();
  } else {
    // FP32 storage: 4-byte copies into a float staging block (the D / Y / rq /
    // cbuf area, larger than B x B floats, is free until the first sub-block),
    // then widened into S
    float* Fs = reinterpret_cast<float*>(Dv);
    for (int e = tid; e < B * B; e += NT) {
      const int i = e % B, j = e / B;
      if (i < w && j < w && i >= j) cp_async_t(&Fs[e], (const float*)&P[(c0 + i) + (size_t)(c0 + j) * nf], true);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    for (int e = tid; e < B * B; e += NT) {
      const int i = e % B, j = e / B;
      if (i < wp && j < wp) S[i + j * kPLd] = (i < w && j < w) ? (i >= j ? (double)Fs[e] : 0.0) : (i == j ? 1.0 : 0.0);
    }
  }
  __syncthreads();
  // ---- right-looking over 32-wide sub-blocks ----
  for (int b = 0; b < nsb; ++b) {
    const int o = b * kPSub;
    double* Db = Dv + (size_t)b * kPSub * kDLd;
    if (warp == 0) {
      int bad;
      if constexpr (sizeof(T) == 4) {
        // Yv (the inverse phase's scratch) is free here: the sub-block's FP32 copy
        bad = warp_chol32_f32(S, o, Db, rq, reinterpret_cast<float*>(cbuf), reinterpret_cast<float*>(Yv), lane);
        if (bad < 0) {                                   // small pivot: the FP64 chain
          if (lane == 0 && fallbacks) atomicAdd(fallbacks, 1);
          bad = warp_chol32_fallback(S, o, Db, rq, cbuf, lane);
        }
      } else {
        bad = warp_chol32(S, o, Db, rq, cbuf, lane);
      }
      if (bad && lane == 0 && o + bad <= w) atomicMin(info + (size_t)info_stride * blockIdx.x, F.first[f] + c0 + o + bad);
    }
    __syncthreads();
    const int rt = nsb - b - 1;                 // 32-row tiles below the sub-block
    if (rt == 0) break;
    if (warp < rt) {                            // L_ib = A_ib D_b^T, in place
      const int r0 = o + kPSub + warp * kPSub;
      double acc[4][4][2];
      acc_zero(acc);
      warp_mm32(acc, S + r0 + o * kPLd, 1, kPLd, Db, kDLd, 1, kPSub, lane);
      __syncwarp();
      acc_store(acc, S + r0 + o * kPLd, 1, kPLd, 1.0, lane);
    }
    __syncthreads();
    for (int t = warp; t < rt * (rt + 1) / 2; t += NT / 32) {   // trailing lower tiles
      int ti = 0;
      while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
      const int tj = t - ti * (ti + 1) / 2;
      const int r0 = o + kPSub + ti * kPSub, q0 = o + kPSub + tj * kPSub;
      double acc[4][4][2];
      acc_zero(acc);
      warp_mm32(acc, S + r0 + o * kPLd, 1, kPLd, S + q0 + o * kPLd, kPLd, 1, kPSub, lane);
      const int g = lane >> 2, q = lane & 3;
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
          for (int e = 0; e < 2; ++e) S[(r0 + 8 * m + g) + (q0 + 8 * n + 2 * q + e) * kPLd] -= acc[m][n][e];
    }
    __syncthreads();
  }
  // ---- inverse: X_rc = -D_r sum_{k=c}^{r-1} L_rk X_kc, X_rc(i, j) stored at S(32c + i, 32r + j) (the
  //      free block above the diagonal, not transposed, so the write-out below reads it conflict-free);
  //      two warps per block column c, 16 rows each ----
  for (int r = 1; r < nsb; ++r) {
    const int c = warp >> 1, h = warp & 1;
    double* Y = Yv + (size_t)c * kPSub * kDLd;
    if (c < r) {
      double acc[2][4][2];
      acc_zero(acc);
      // k = c: X_cc = D_c, B(k', j) = D_c(k', j)
      warp_mm32(acc, S + r * kPSub + 16 * h + c * kPSub * kPLd, 1, kPLd, Dv + (size_t)c * kPSub * kDLd, 1, kDLd,
                kPSub, lane);
      for (int k = c + 1; k < r; ++k)   // B(k', j) = X_kc(k', j) = S(32c + k', 32k + j)
        warp_mm32(acc, S + r * kPSub + 16 * h + k * kPSub * kPLd, 1, kPLd, S + c * kPSub + k * kPSub * kPLd, 1,
                  kPLd, kPSub, lane);
      acc_store(acc, Y + 16 * h, 1, kDLd, 1.0, lane);
    }
    __syncthreads();
    if (c < r) {
      double acc[2][4][2];
      acc_zero(acc);
      warp_mm32(acc, Dv + (size_t)r * kPSub * kDLd + 16 * h, 1, kDLd, Y, 1, kDLd, kPSub, lane);
      acc_store(acc, S + c * kPSub + 16 * h + r * kPSub * kPLd, 1, kPLd, -1.0, lane);
    }
    __syncthreads();
  }
  // ---- write L11 to the panel and X to linv ----
  for (int e = tid; e < B * B; e += NT) {
    const int i = e % B, j = e / B;
    if (i < w && j < w && i >= j) P[(c0 + i) + (size_t)(c0 + j) * nf] = (T)S[i + j * kPLd];
  }
  // persistent blocks (d_off) were zeroed once: only their lower w x w part is written
  T* Li = inv_block(F, linv, f, step, blockIdx.x);
  const bool full = F.d_off == nullptr;                      // scratch blocks: the whole 128 x 128 block written
  const int EB = full ? kFactB : B;
  for (int e = tid; e < EB * EB; e += NT) {
    const int i = e % EB, j = e / EB;
    const bool in = i < w && j < w && i >= j;
    if (!in && !full) continue;
    double v = 0.0;
    if (in) {
      const int bi = i / kPSub, bj = j / kPSub;
      v = bi == bj ? Dv[(size_t)bi * kPSub * kDLd + (i - bi * kPSub) + (j - bj * kPSub) * kDLd]
                   : S[(bj * kPSub + i - bi * kPSub) + (bi * kPSub + j - bj * kPSub) * kPLd];
    }
    Li[i + (size_t)j * kFactB] = (T)v;
  }
}



template <typename T>
__device__ __forceinline__ T* trailing_addr(T* P, T* U, int nc, int nr, int nf, int gi, int gj) {
  return gj < nc ? P + gi + (size_t)gj * nf : U + (gi - nc) + (size_t)(gj - nc) * nr;
}

// Trailing update on the FP64 tensor pipe: one 128x128 tile of the trailing
// lower triangle per CTA, C -= P_i P_j^T over the K range of the step's
// deferred group (update_k_range: up to defer x 128 panel columns) in chunks
// of 32, double-buffered with cp.async.  16 warps as 4 (rows) x 4 (columns) of 32x32,
// each 2 x 4 mma.m16n8k16.f64 per K step of 16.  Shared-memory operands are
// k-major with a row stride of 132 doubles (= 4 mod 16): every fragment load of
// a half-warp hits 16 distinct 8-byte bank pairs.  The accumulators are loaded
// with C itself (8 rows x 4 column pairs per warp access: full 32-byte
// sectors) while the first operand chunk is in flight, the A fragments enter
// negated, and the epilogue only stores.
constexpr int kUT = 128, kUK = 32, kULD = 132;
constexpr int kUThreads = 512;              // 16 warps: 4 (rows) x 4 (columns) of 32 x 32
constexpr int kUMF = kUT / (kUThreads / 32 / 4) / 16;   // m16 fragments per warp (2)

__device__ __forceinline__ void dmma16(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Panel TRSM X = A Li^T (Li = L11^{-1}, lower): one CTA per 32 rows of X and
// all its w <= 128 columns (the TRSM is in place, so a CTA must read its rows
// of A before any CTA writes them: rows are never split across CTAs), so a
// panel step of nrem rows runs on nrem / 32 CTAs.  Operands arrive by
// cp.async (all in flight at once).  FP64: 8 warps as 2 x 4 of 16 x 32
// (m16n8k16 DMMA); FP32: 256 threads of 2 rows x 8 columns (FFMA).
constexpr int kTr2Rows = 32;
constexpr int kTr2LdA = kTr2Rows + 4, kTr2LdB = kFactB + 4;   // = 4 mod 16 doubles
template <typename T>
constexpr size_t trsm2_smem() {
  return ((size_t)kFactB * kTr2LdA + (size_t)kFactB * kTr2LdB) * sizeof(T);
}


template <typename T>
__global__ void __launch_bounds__(256) k_trsm2(DevFronts F, const int32_t* list, int step, T* panel, const T* linv,
                                               float* q) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);            // [k][row]
  T* Bs = As + kFactB * kTr2LdA;                      // [k][n]: Li(n, k)
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nf = nc + F.nr[f];
  const int c0 = step * kFactB;
  if (c0 >= nc) return;
  const int w = min(kFactB, nc - c0);
  const int r0 = c0 + w + blockIdx.x * kTr2Rows;
  if (r0 >= nf) return;
  T* P = panel + F.panel_off[f];
  const T* Li = inv_block(F, linv, f, step, blockIdx.y);
  const int kp = (w + 15) & ~15;
  // the rows below the diagonal block do not depend on the POTRF that precedes this kernel
  // (no event wait sits between the two launches)
  for (int e = threadIdx.x; e < kTr2Rows * kp; e += blockDim.x) {
    const int k = e / kTr2Rows, r = e - k * kTr2Rows;
    const bool v = k < w && r0 + r < nf;
    cp_async_t(&As[k * kTr2LdA + r], v ? P + (r0 + r) + (size_t)(c0 + k) * nf : P, v);
  }
  pdl_wait();
  pdl_trigger();
  // Li in 16-byte copies: the block is 16-byte aligned, rows of 128 elements, and zero
  // outside its lower w x w part (so the rows k < kp copy whole)
  constexpr int kVec = 16 / (int)sizeof(T);
  for (int e = threadIdx.x; e < kFactB / kVec * kp; e += blockDim.x) {
    const int k = e / (kFactB / kVec), n = (e - k * (kFactB / kVec)) * kVec;
    const unsigned sa = (unsigned)__cvta_generic_to_shared(&Bs[k * kTr2LdB + n]);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(Li + n + (size_t)k * kFactB));
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  if constexpr (sizeof(T) == 8) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 2, wn = warp & 3;            // 16-row band, 32-column band
    const int g = lane >> 2, q = lane & 3;
    double acc[4][4] = {};
    for (int kk = 0; kk < kp; kk += 16) {
      double av[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) av[i] = As[(kk + q + 4 * (i >> 1)) * kTr2LdA + wm * 16 + g + 8 * (i & 1)];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        double bv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) bv[i] = Bs[(kk + q + 4 * i) * kTr2LdB + wn * 32 + ni * 8 + g];
        dmma16(acc[ni], av, bv);
      }
    }
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int gi = r0 + wm * 16 + g + 8 * (e >> 1);
        const int n = wn * 32 + ni * 8 + 2 * q + (e & 1);
        if (gi < nf && n < w) P[gi + (size_t)(c0 + n) * nf] = acc[ni][e];
      }
  } else {
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // columns tx + 16 m, rows ty + 16 l
    T acc[2][8] = {};
    for (int k = 0; k < w; ++k) {
      T av[2], bv[8];
#pragma unroll
      for (int l = 0; l < 2; ++l) av[l] = As[k * kTr2LdA + ty + 16 * l];
#pragma unroll
      for (int m = 0; m < 8; ++m) bv[m] = Bs[k * kTr2LdB + tx + 16 * m];
#pragma unroll
      for (int l = 0; l < 2; ++l)
#pragma unroll
        for (int m = 0; m < 8; ++m) acc[l][m] = fmaf(av[l], bv[m], acc[l][m]);
    }
#pragma unroll
    for (int l = 0; l < 2; ++l)
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const int gi = r0 + ty + 16 * l, n = tx + 16 * m;
        if (gi < nf && n < w) P[gi + (size_t)(c0 + n) * nf] = acc[l][m];
      }
    if (q != nullptr) {     // the same rows as packed TF32 hi / lo operands of the tensor-core update
      float* Q = q + F.q_off[f];
      const int rrel = blockIdx.x * kTr2Rows;                 // first row of the CTA relative to c0 + w
#pragma unroll
      for (int l = 0; l < 2; ++l)
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const int rr = rrel + ty + 16 * l, n = tx + 16 * m;
          const float v = (r0 + ty + 16 * l < nf && n < w) ? (float)acc[l][m] : 0.0f;
          uint32_t hb;
          asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"(v));
          const float hi = __uint_as_float(hb);
          Q[packed_offset(rr, n, 0)] = hi;
          Q[packed_offset(rr, n, 1)] = v - hi;
        }
    }
  }
}

__global__ void __launch_bounds__(kUThreads, 1) k_update_dmma(DevFronts F, const int32_t* list, int step, double* panel,
                                                        double* upool, int blo, int bhi, int defer) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sm = reinterpret_cast<double*>(smem_raw);     // [stage][operand][k][row]
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  const int c0 = step * kFactB;
  if (c0 >= nc) return;
  const int w = min(kFactB, nc - c0);
  const int base = c0 + w;
  const int nrem = nf - base;
  if (nrem <= 0) return;
  const int T = (nrem + kUT - 1) / kUT;
  int ti, tj, kbeg, kend;
  if (!select_tile(T, kUT, blo, bhi, blockIdx.x, ti, tj)) return;
  if (!update_k_range(nc, step, defer, tj, kUT, kbeg, kend)) return;
  const int K = kend - kbeg;                            // panel columns [kbeg, kend) of the front
  const int i0 = base + ti * kUT, j0 = base + tj * kUT;
  double* P = panel + F.panel_off[f];
  double* U = upool + F.u_off[f];
  const int nchunks = (K + kUK - 1) / kUK;
  const bool diag = ti == tj;
  auto load = [&](int stage, int kc) {
    double* dst = sm + stage * (2 * kUK * kULD);
    const int ops = diag ? 1 : 2;                       // a diagonal tile's B is its A
    for (int e = threadIdx.x; e < ops * kUK * kUT; e += blockDim.x) {
      const int op = e / (kUK * kUT), rem = e - op * (kUK * kUT);
      const int k = rem / kUT, r = rem - k * kUT;
      const int row = (op == 0 ? i0 : j0) + r, col = kc * kUK + k;
      const bool valid = row < nf && col < K;
      const double* src = valid ? P + row + (size_t)(kbeg + col) * nf : P;
      cp_async8(dst + op * (kUK * kULD) + k * kULD + r, src, valid);
    }
    cp_async_commit();
  };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;
  const int g = lane >> 2, q = lane & 3;
  // the accumulators start as C (loads in flight with the first operand chunk) and the
  // A fragments enter negated, so the tile ends as C - P_i P_j^T and the epilogue only stores
  const int rbase = i0 + wm * (16 * kUMF) + g, cbase = j0 + wn * 32 + 2 * q;
  // C may be written by a kernel this one waits on through an event (the
  // lookahead's side stream): everything is read after the wait
  pdl_wait();
  pdl_trigger();
  double acc[kUMF][4][4];
#pragma unroll
  for (int mi = 0; mi < kUMF; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int gi = rbase + mi * 16 + 8 * (e >> 1), gj = cbase + ni * 8 + (e & 1);
        acc[mi][ni][e] = (gi < nf && gj < nf && gi >= gj) ? *trailing_addr(P, U, nc, nr, nf, gi, gj) : 0.0;
      }
  load(0, 0);
  for (int kc = 0; kc < nchunks; ++kc) {
    if (kc + 1 < nchunks) {
      load((kc + 1) & 1, kc + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* As = sm + (kc & 1) * (2 * kUK * kULD);
    const double* Bs = diag ? As : As + kUK * kULD;
#pragma unroll
    for (int kk = 0; kk < kUK; kk += 16) {
      double bv[4][4];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int i = 0; i < 4; ++i) bv[ni][i] = Bs[(kk + q + 4 * i) * kULD + wn * 32 + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < kUMF; ++mi) {
        double av[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) av[i] = -As[(kk + q + 4 * (i >> 1)) * kULD + wm * (16 * kUMF) + mi * 16 + g + 8 * (i & 1)];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma16(acc[mi][ni], av, bv[ni]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < kUMF; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int gi = rbase + mi * 16 + 8 * (e >> 1), gj = cbase + ni * 8 + (e & 1);
        if (gi < nf && gj < nf && gi >= gj) *trailing_addr(P, U, nc, nr, nf, gi, gj) = acc[mi][ni][e];
      }
}

// FP64 trailing update in 128 x 64 halves: CTA x computes columns
// 64 h .. 64 h + 63 (h = x & 1) of square tile x >> 1 of the band (the same
// tiles, bands and K ranges as k_update_dmma).  256 threads: 8 warps as 4
// (rows) x 2 (columns) of 32 x 32, each 2 x 4 mma.m16n8k16.f64 per K step of
// 16, so 128 registers and 102 KB of shared memory per CTA and two CTAs per
// SM: one CTA's C loads and stores overlap the other's MMAs.  Operands come
// in K chunks of 32 by cp.async (16-byte row pairs where aligned),
// double-buffered; a diagonal tile's B is rows 64 h .. of its A.  C is loaded into the accumulators (the A fragments enter
// negated) and stored back; tiles wholly inside the trailing matrix, below
// the diagonal and inside the panel or the update matrix take an unchecked
// path.  In a diagonal tile's right half the warps whose 32 rows all lie
// above the diagonal skip the MMAs.
constexpr int kU2Threads = 256;
constexpr int kU2N = 64;
constexpr int kU2LdB = kU2N + 4;                             // 68 = 4 mod 16 doubles: conflict-free fragments
constexpr int kU2Stage = kUK * kULD + kUK * kU2LdB;           // doubles per pipeline stage
constexpr size_t kU2Smem = 2 * (size_t)kU2Stage * sizeof(double);

__global__ void __launch_bounds__(kU2Threads, 2) k_update_dmma2(DevFronts F, const int32_t* list, int step,
                                                              double* panel, double* upool, int blo, int bhi,
                                                              int defer) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sm = reinterpret_cast<double*>(smem_raw);     // per stage: A [k][kULD] (128 rows), B [k][kU2LdB] (64 rows)
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  const int c0 = step * kFactB;
  if (c0 >= nc) return;
  const int w = min(kFactB, nc - c0);
  const int base = c0 + w;
  const int nrem = nf - base;
  if (nrem <= 0) return;
  const int T = (nrem + kUT - 1) / kUT;
  const int hf = blockIdx.x & 1;
  int ti, tj, kbeg, kend;
  if (!select_tile(T, kUT, blo, bhi, blockIdx.x >> 1, ti, tj)) return;
  if (!update_k_range(nc, step, defer, tj, kUT, kbeg, kend)) return;
  const int i0 = base + ti * kUT, j0 = base + tj * kUT + hf * kU2N;
  if (j0 >= nf) return;                                 // the right half lies beyond the matrix
  const int K = kend - kbeg;                            // panel columns [kbeg, kend) of the front
  const bool diag = ti == tj;
  double* P = panel + F.panel_off[f];
  double* U = upool + F.u_off[f];
  const int nchunks = (K + kUK - 1) / kUK;
  // Copies: thread t moves row pairs -- A rows i0 + 2 (t & 63) (+1) at columns
  // (t >> 6) + 4 v, v < 8; B rows j0 + 2 (t & 31) (+1) at columns (t >> 5) +
  // 8 v, v < 4 (a diagonal tile's B is in A) -- 16 bytes per copy when the
  // pair's source is 16-byte aligned.  A thread's copies are 4 or 8 columns
  // apart, so the alignment is the same for all of them (and, the lanes of a
  // warp sharing the column, the same across the warp); otherwise two 8-byte
  // copies.  Rows past the matrix and columns past K are zero-filled.
  auto copy = [&](double* d, const double* src, int bytes, bool al) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(d);
    if (al) {
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(bytes ? src : P), "r"(bytes));
    } else {
      const int b0 = bytes >= 8 ? 8 : 0, b1 = bytes >= 16 ? 8 : 0;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(b0 ? src : P), "r"(b0));
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa + 8), "l"(b1 ? src + 1 : P), "r"(b1));
    }
  };
  auto load = [&](int stage, int kc) {
    // the per-thread quantities are recomputed here (kept live they would spill)
    const int pa = threadIdx.x & 63, ka = threadIdx.x >> 6;
    const int ra = i0 + 2 * pa;
    const int na = ra < nf ? (ra + 1 < nf ? 16 : 8) : 0;          // bytes of the A pair inside the matrix
    const bool ala = ((ra + (long long)(kbeg + ka) * nf) & 1) == 0; // panel offsets are multiples of 32 elements
    double* dst = sm + stage * kU2Stage;
    const int k0 = kc * kUK;
    const double* sa = P + ra + (size_t)(kbeg + k0 + ka) * nf;
    double* da = dst + ka * kULD + 2 * pa;
#pragma unroll 1
    for (int v = 0; v < 8; ++v) {                   // rolled: unrolled, the copies' addresses would be kept live
      const int k = k0 + ka + 4 * v;
      copy(da + v * 4 * kULD, sa + (size_t)(4 * v) * nf, k < K ? na : 0, ala);
    }
    if (diag) return;
    const int pb = threadIdx.x & 31, kb = threadIdx.x >> 5;
    const int rb = j0 + 2 * pb;
    const int nbb = rb < nf ? (rb + 1 < nf ? 16 : 8) : 0;
    const bool alb = ((rb + (long long)(kbeg + kb) * nf) & 1) == 0;
    const double* sb = P + rb + (size_t)(kbeg + k0 + kb) * nf;
    double* db = dst + kUK * kULD + kb * kU2LdB + 2 * pb;
#pragma unroll 1
    for (int v = 0; v < 4; ++v) {
      const int k = k0 + kb + 8 * v;
      copy(db + v * 8 * kU2LdB, sb + (size_t)(8 * v) * nf, k < K ? nbb : 0, alb);
    }
  };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, q = lane & 3;
  const int rbase = i0 + wm * 32 + g, cbase = j0 + wn * 32 + 2 * q;
  // warps of a diagonal tile's right half whose rows all lie above the diagonal
  const bool idle = i0 + wm * 32 + 31 < j0 + wn * 32;
  // unchecked path: the tile is inside the trailing matrix, wholly below the
  // diagonal and wholly in the panel or wholly in the update matrix (formed
  // again for the epilogue rather than kept live through the K loop)
  auto full_tile = [&]() { return i0 + kUT <= nf && j0 + kU2N <= nf && i0 >= j0 + kU2N && (j0 + kU2N <= nc || j0 >= nc); };
  auto c_base = [&]() { return j0 < nc ? P + (size_t)j0 * nf : U + (size_t)(j0 - nc) * nr - nc; };   // C(gi, gj) = Cb[gi + (gj - j0) ldc]
  pdl_wait();
  pdl_trigger();
  load(0, 0);
  cp_async_commit();
  double acc[2][4][4];
  {
  const bool full = full_tile();
  const int ldc = j0 < nc ? nf : nr;
  double* Cb = c_base();
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int gi = rbase + mi * 16 + 8 * (e >> 1), gj = cbase + ni * 8 + (e & 1);
        if (full)
          acc[mi][ni][e] = Cb[gi + (size_t)(gj - j0) * ldc];
        else
          acc[mi][ni][e] = (!idle && gi < nf && gj < nf && gi >= gj) ? *trailing_addr(P, U, nc, nr, nf, gi, gj) : 0.0;
      }
  }
  for (int kc = 0; kc < nchunks; ++kc) {
    if (kc + 1 < nchunks) {
      load((kc + 1) & 1, kc + 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (!idle) {
      const double* As = sm + (kc & 1) * kU2Stage;
      const double* Bs = diag ? As + hf * kU2N : As + kUK * kULD;
      const int ldb = diag ? kULD : kU2LdB;
#pragma unroll
      for (int kk = 0; kk < kUK; kk += 16) {
        double bv[4][4];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
          for (int i = 0; i < 4; ++i) bv[ni][i] = Bs[(kk + q + 4 * i) * ldb + wn * 32 + ni * 8 + g];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
          double av[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) av[i] = -As[(kk + q + 4 * (i >> 1)) * kULD + wm * 32 + mi * 16 + g + 8 * (i & 1)];
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) dmma16(acc[mi][ni], av, bv[ni]);
        }
      }
    }
    __syncthreads();
  }
  if (idle) return;
  const bool full = full_tile();
  const int ldc = j0 < nc ? nf : nr;
  double* Cb = c_base();
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int gi = rbase + mi * 16 + 8 * (e >> 1), gj = cbase + ni * 8 + (e & 1);
        if (full)
          Cb[gi + (size_t)(gj - j0) * ldc] = acc[mi][ni][e];
        else if (gi < nf && gj < nf && gi >= gj)
          *trailing_addr(P, U, nc, nr, nf, gi, gj) = acc[mi][ni][e];
      }
}

// Trailing update on the FMA pipes (any T): 64x64 tiles, K in chunks of 64,
// 256 threads each 4x4 outputs (rows ty+16m, columns tx+16n).
constexpr int kSimtTile = 64, kSimtK = 64;
template <typename T>
__global__ void __launch_bounds__(256) k_update_simt(DevFronts F, const int32_t* list, int step, T* panel, T* upool,
                                                     int blo, int bhi, int defer) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int LDK = kSimtTile + 4;
  T* As = reinterpret_cast<T*>(smem_raw);
  T* Bs = As + kSimtK * LDK;
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  const int c0 = step * kFactB;
  if (c0 >= nc) return;
  const int w = min(kFactB, nc - c0);
  const int base = c0 + w;
  const int nrem = nf - base;
  if (nrem <= 0) return;
  const int Tn = (nrem + kSimtTile - 1) / kSimtTile;
  int ti, tj, kbeg, kend;
  if (!select_tile(Tn, kSimtTile, blo, bhi, blockIdx.x, ti, tj)) return;
  if (!update_k_range(nc, step, defer, tj, kSimtTile, kbeg, kend)) return;
  const int K = kend - kbeg;
  const int i0 = base + ti * kSimtTile, j0 = base + tj * kSimtTile;
  T* P = panel + F.panel_off[f];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n) acc[m][n] = T(0);
  for (int k0 = 0; k0 < K; k0 += kSimtK) {
    const int kw = min(kSimtK, K - k0);
    __syncthreads();
    batched_loop(
        2 * kSimtTile * kw,
        [&](int e) {
          const int op = e / (kSimtTile * kw), rem = e - op * (kSimtTile * kw);
          const int k = rem / kSimtTile, g = (op ? j0 : i0) + rem % kSimtTile;
          return g < nf ? P[g + (size_t)(kbeg + k0 + k) * nf] : T(0);
        },
        [&](int e, T v) {
          const int op = e / (kSimtTile * kw), rem = e - op * (kSimtTile * kw);
          (op ? Bs : As)[(rem / kSimtTile) * LDK + rem % kSimtTile] = v;
        });
    __syncthreads();
    for (int k = 0; k < kw; ++k) {
      T av[4], bv[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) av[m] = As[k * LDK + ty + 16 * m];
#pragma unroll
      for (int n = 0; n < 4; ++n) bv[n] = Bs[k * LDK + tx + 16 * n];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n) acc[m][n] += av[m] * bv[n];
    }
  }
  T* U = upool + F.u_off[f];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      int gi = i0 + ty + 16 * m, gj = j0 + tx + 16 * n;
      if (gi < nf && gj < nf && gi >= gj) *trailing_addr(P, U, nc, nr, nf, gi, gj) -= acc[m][n];
    }
}

// ============================================================================
// solves
// ============================================================================

// ---- fronts with nf <= 32: one warp per front ---------------------------------
// Four fronts per 128-thread CTA.  The front is assembled in a per-warp
// shared buffer (A entries, then the children's update matrices through
// local_index), loaded one row per lane into registers and partially
// factored there (nc pivots: shuffle for the pivot, rsqrt, rank-1 update with
// the column broadcast through a double-buffered shared vector); the panel
// columns and the update matrix are written back one column per step, lanes
// over rows (coalesced).  No CTA-wide barrier: many more fronts in flight per
// SM than the one-CTA-per-front kernel.
constexpr int kWF = 32;          // front capacity of a warp
constexpr int kWFLd = kWF + 1;
constexpr int kWFWarps = 4;


template <typename T>
__global__ void __launch_bounds__(kWFWarps * 32) k_small_warp(DevFronts F, const int32_t* list, int count,
                                                              const double* __restrict__ a, T* __restrict__ panel,
                                                              T* __restrict__ upool, int32_t* info) {
  __shared__ T sbuf[kWFWarps][kWF * kWFLd];
  __shared__ T cbuf[kWFWarps][2][kWF];
  __shared__ int slocbuf[kWFWarps][kWF];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = blockIdx.x * kWFWarps + warp;
  if (slot >= count) return;
  const int f = list[slot];
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  T* S = sbuf[warp];
  // children's metadata one per lane (broadcast by shuffles), loaded while
  // the front is zeroed and assembled
  const int cp0 = F.child_ptr[f], nch = F.child_ptr[f + 1] - cp0;
  int cnr = 0, clo = 0;
  long long cuo = 0;
  if (lane < nch) {
    const int c = F.child[cp0 + lane];
    cnr = F.nr[c]; clo = F.lrow_off[c]; cuo = F.u_off[c];
  }
  for (int e = lane; e < kWF * kWFLd; e += 32) S[e] = T(0);
  __syncwarp();
  assemble_smem<4>(F, f, nf, a, S, [](int r, int c) { return r + c * kWFLd; }, lane, 32);
  __syncwarp();
  int* sloc = slocbuf[warp];
  for (int cb = 0; cb < nch; cb += 32) {
    if (cb > 0) {
      cnr = 0; clo = 0; cuo = 0;
      if (cb + lane < nch) {
        const int c = F.child[cp0 + cb + lane];
        cnr = F.nr[c]; clo = F.lrow_off[c]; cuo = F.u_off[c];
      }
    }
    const int m = min(32, nch - cb);
    for (int t = 0; t < m; ++t) {
      const int nrc = __shfl_sync(0xffffffffu, cnr, t), lo = __shfl_sync(0xffffffffu, clo, t);
      const long long uo = __shfl_sync(0xffffffffu, cuo, t);
      if (lane < nrc) sloc[lane] = F.local[lo + lane];
      __syncwarp();
      extend_add_smem<8>(S, kWFLd, upool + uo, sloc, nrc, lane, 32);
      __syncwarp();
    }
  }
  T row[kWF];
#pragma unroll
  for (int j = 0; j < kWF; ++j) row[j] = S[lane + j * kWFLd];
  int bad = 0;
#pragma unroll
  for (int k = 0; k < kWF; ++k) {
    if (k >= nc) break;
    T d = __shfl_sync(0xffffffffu, row[k], k);
    if (!(d > T(0))) {                    // uniform across the warp
      if (!bad) bad = k + 1;
      d = T(1);
    }
    const T y = rsqrt_t<T>(d);
    const T l = row[k] * y;
    T* cb = cbuf[warp][k & 1];
    cb[lane] = l;
    __syncwarp();
    row[k] = lane == k ? d * y : l;
#pragma unroll
    for (int j = k + 1; j < kWF; ++j) row[j] -= l * cb[j];
  }
  if (bad && lane == 0) atomicMin(info, F.first[f] + bad);
  T* P = panel + F.panel_off[f];
  T* Uf = upool + F.u_off[f];
#pragma unroll
  for (int j = 0; j < kWF; ++j) {
    if (j >= nf) break;
    if (lane >= j && lane < nf) {
      if (j < nc) P[lane + (size_t)j * nf] = row[j];
      else Uf[(lane - nc) + (size_t)(j - nc) * nr] = row[j];
    }
  }
}

// ---- small-front solves: one warp per front (nf <= 32 R) ----------------------
// Four fronts per 128-thread CTA, no CTA-wide barrier, so many fronts are in
// flight per SM and their panel reads overlap.  The front's solve vector is
// staged in a per-warp shared vector (the children's update vectors are
// scattered into it through local_index).
//   forward : lane l holds rows l + 32 q (q < R); column k of the panel is
//             read lanes over rows (coalesced), y_k = v_k / L_kk is formed by
//             the lane holding row k and broadcast by a shuffle, and every row
//             below k takes v_i -= L_ik y_k.
//   backward: 32-column blocks from the last: the rows below the block's
//             triangle give t_k -= sum_i L_ik x_i as per-lane partial sums
//             over rows (coalesced) reduced through a transposing per-warp
//             tile; the 32 x 32 triangle is read lanes over rows, transposed
//             through the same tile (lane k then holds column k) and solved
//             by shuffles.
constexpr int kSWarps = 4;
constexpr int kTileLd = 33;

template <typename T, int R>
__device__ __forceinline__ T pick(const T (&a)[R], int q) {
  T r = a[0];
#pragma unroll
  for (int p = 1; p < R; ++p)
    if (p == q) r = a[p];
  return r;
}
template <typename T, int R>
__device__ __forceinline__ void put(T (&a)[R], int q, T v) {
#pragma unroll
  for (int p = 0; p < R; ++p)
    if (p == q) a[p] = v;
}

// v += the children's update vectors of front f (right-hand side r), child
// metadata loaded one child per lane so the per-child chain is one load deep
template <typename T, int R>
__device__ __forceinline__ void gather_children(const DevFronts& F, int f, const T* V, int nrhs, int r, T* vs,
                                                int lane) {
  const int c0 = F.child_ptr[f], nch = F.child_ptr[f + 1] - c0;
  for (int cb = 0; cb < nch; cb += 32) {
    int cnc = 0, cnr = 0, clo = 0;
    long long cvo = 0;
    if (cb + lane < nch) {
      const int c = F.child[c0 + cb + lane];
      cnc = F.nc[c]; cnr = F.nr[c]; clo = F.lrow_off[c]; cvo = F.v_off[c];
    }
    const int m = min(32, nch - cb);
    for (int t = 0; t < m; ++t) {
      const int ncc = __shfl_sync(0xffffffffu, cnc, t), nrc = __shfl_sync(0xffffffffu, cnr, t);
      const int lo = __shfl_sync(0xffffffffu, clo, t);
      const long long vo = __shfl_sync(0xffffffffu, cvo, t);
      const T* Vc = V + vo * nrhs + (int64_t)r * (ncc + nrc) + ncc;
      const int32_t* loc = F.local + lo;
      int li[R];
      T vv[R];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int i = lane + 32 * q;
        li[q] = i < nrc ? loc[i] - 1 : -1;
        vv[q] = i < nrc ? Vc[i] : T(0);
      }
#pragma unroll
      for (int q = 0; q < R; ++q)
        if (li[q] >= 0) vs[li[q]] += vv[q];
      __syncwarp();
    }
  }
}

// L2 prefetch of a front's panel (nf x nc, contiguous, 16-byte aligned; the
// size is rounded up into the pool's alignment padding)
template <typename T>
__device__ __forceinline__ void prefetch_panel(const T* P, int nf, int nc) {
  const unsigned bytes = ((unsigned)((size_t)nf * nc * sizeof(T)) + 15u) & ~15u;
  if (bytes) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(P), "r"(bytes) : "memory");
}

template <typename T, int R>
__device__ __forceinline__ void fwd_small_front(const DevFronts& F, int f, const T* __restrict__ panel, T* X,
                                                int64_t ldx, T* V, int nrhs, T* vs, int lane) {
  const int nc = F.nc[f], nf = nc + F.nr[f], first = F.first[f];
  const T* P = panel + F.panel_off[f];
  if (lane == 0) prefetch_panel(P, nf, nc);
  T dinv[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int i = lane + 32 * q;
    dinv[q] = i < nc ? T(1) / P[i + (size_t)i * nf] : T(1);
  }
  T* Vf = V + F.v_off[f] * nrhs;
  const int rb = gridDim.y > 1 ? (int)blockIdx.y : 0, re = gridDim.y > 1 ? rb + 1 : nrhs;   // one RHS per CTA row
  for (int r = rb; r < re; ++r) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int i = lane + 32 * q;
      vs[i] = i < nc ? X[first + i + r * ldx] : T(0);
    }
    __syncwarp();
    gather_children<T, R>(F, f, V, nrhs, r, vs, lane);
    T v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = vs[lane + 32 * q];
    __syncwarp();
    // columns in groups of G with predicated (not early-exited) steps, so the
    // group's loads issue together: one memory latency per group
    constexpr int G = 8;
    for (int k0 = 0; k0 < nc; k0 += 32) {
      const int qb = k0 >> 5, kn = min(32, nc - k0);
      const T dk = pick(dinv, qb);
      for (int g = 0; g < kn; g += G) {
        T l[G][R];
#pragma unroll
        for (int u = 0; u < G; ++u) {
          const int k = k0 + g + u;
          const T* Pk = P + (size_t)k * nf;
#pragma unroll
          for (int q = 0; q < R; ++q) {
            const int i = lane + 32 * q;
            l[u][q] = (g + u < kn && i > k && i < nf) ? Pk[i] : T(0);
          }
        }
#pragma unroll
        for (int u = 0; u < G; ++u) {
          if (g + u < kn) {
            const int kk = g + u, k = k0 + kk;
            const T yk = __shfl_sync(0xffffffffu, pick(v, qb) * dk, kk);
#pragma unroll
            for (int q = 0; q < R; ++q)
              if (lane + 32 * q > k) v[q] -= l[u][q] * yk;
            if (lane == kk) put(v, qb, yk);
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int i = lane + 32 * q;
      if (i < nc) X[first + i + r * ldx] = v[q];
      else if (i < nf) Vf[(int64_t)r * nf + i] = v[q];
    }
  }
}

template <typename T, int R>
__global__ void __launch_bounds__(kSWarps * 32) k_fwd_small(DevFronts F, const int32_t* list, int count,
                                                            const T* __restrict__ panel, T* X, int64_t ldx, T* V,
                                                            int nrhs) {
  __shared__ T vbuf[kSWarps][32 * R];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = blockIdx.x * kSWarps + warp;
  if (slot >= count) return;
  fwd_small_front<T, R>(F, list[slot], panel, X, ldx, V, nrhs, vbuf[warp], lane);
}

template <typename T, int R>
__device__ __forceinline__ void bwd_small_front(const DevFronts& F, int f, const T* __restrict__ panel, T* X,
                                                int64_t ldx, int nrhs, T* xs, T* tile, int lane) {
  const int nc = F.nc[f], nf = nc + F.nr[f], first = F.first[f];
  const int32_t* lr = F.lrow + F.lrow_off[f];
  const T* P = panel + F.panel_off[f];
  if (lane == 0) prefetch_panel(P, nf, nc);
  const int rb = gridDim.y > 1 ? (int)blockIdx.y : 0, re = gridDim.y > 1 ? rb + 1 : nrhs;   // one RHS per CTA row
  for (int r = rb; r < re; ++r) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int i = lane + 32 * q;
      xs[i] = i < nc ? X[first + i + r * ldx] : (i < nf ? X[lr[i - nc] + r * ldx] : T(0));
    }
    __syncwarp();
    for (int b = (nc - 1) >> 5; b >= 0; --b) {
      const int j0 = 32 * b, e = min(j0 + 32, nc), kn = e - j0;   // the block's columns [j0, e)
      T s = T(0);
      if constexpr (R == 1) {
        // nf <= 32: the whole panel in one pass, lanes over rows (one memory
        // latency): triangle rows raw and lower, rows below nc as products
        // with x, summed per column in row order
        const int i = lane;
        const bool tri = i < nc, ok = i < nf;
        const T xi = (!tri && ok) ? xs[i] : T(0);
        T l[32];
#pragma unroll
        for (int kk = 0; kk < 32; ++kk) l[kk] = (ok && kk < nc && (!tri || kk <= i)) ? P[i + (size_t)kk * nf] : T(0);
#pragma unroll
        for (int kk = 0; kk < 32; ++kk) tile[lane * kTileLd + kk] = tri ? l[kk] : l[kk] * xi;
        __syncwarp();
#pragma unroll
        for (int ii = 0; ii < 32; ++ii) {
          const T v = tile[ii * kTileLd + lane];
          if (ii >= nc && ii < nf) s += v;
        }
      } else {
        // rows below the triangle [e, nf), lanes over rows, 8 columns at a time:
        // tile(lane, kk) = sum over the lane's rows i of L(i, j0+kk) x_i
        for (int g = 0; g < kn; g += 8) {
          T acc[8];
#pragma unroll
          for (int kk = 0; kk < 8; ++kk) acc[kk] = T(0);
          for (int i0 = e; i0 < nf; i0 += 32) {
            const int i = i0 + lane;
            const bool ok = i < nf;
            const T xi = ok ? xs[i] : T(0);
            const T* Pi = P + i + (size_t)(j0 + g) * nf;
            T l[8];
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) l[kk] = (ok && g + kk < kn) ? Pi[(size_t)kk * nf] : T(0);
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) acc[kk] += l[kk] * xi;
          }
#pragma unroll
          for (int kk = 0; kk < 8; ++kk) tile[lane * kTileLd + g + kk] = acc[kk];
        }
        __syncwarp();
        // columns >= kn of the tile are not written: unused
#pragma unroll
        for (int j = 0; j < 32; ++j) s += tile[j * kTileLd + lane];
        __syncwarp();
        // the triangle, read lanes over rows (row j0 + lane, columns j0 .. row)
        // into the tile; lane k then reads column k from it
        {
          const int i = j0 + lane;
          const T* Pi = P + i + (size_t)j0 * nf;
#pragma unroll
          for (int h = 0; h < 32; h += 16) {
            T l[16];
#pragma unroll
            for (int kk = 0; kk < 16; ++kk) l[kk] = (h + kk <= lane && lane < kn) ? Pi[(size_t)(h + kk) * nf] : T(0);
#pragma unroll
            for (int kk = 0; kk < 16; ++kk) tile[lane * kTileLd + h + kk] = l[kk];
          }
        }
      }
      __syncwarp();
      const T dk = lane < kn ? T(1) / tile[lane * kTileLd + lane] : T(1);
      T t = lane < kn ? xs[j0 + lane] - s : T(0);
#pragma unroll 8
      for (int ii = 31; ii >= 0; --ii) {
        if (ii >= kn) continue;
        const T lv = tile[ii * kTileLd + lane];    // L(j0 + ii, j0 + lane)
        const T xi = __shfl_sync(0xffffffffu, t * dk, ii);
        if (lane == ii) t = xi;
        else if (lane < ii) t -= lv * xi;
      }
      __syncwarp();
      if (lane < kn) xs[j0 + lane] = t;
      __syncwarp();
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int i = lane + 32 * q;
      if (i < nc) X[first + i + r * ldx] = xs[i];
    }
    __syncwarp();
  }
}

template <typename T, int R>
__global__ void __launch_bounds__(kSWarps * 32, 6) k_bwd_small(DevFronts F, const int32_t* list, int count,
                                                            const T* __restrict__ panel, T* X, int64_t ldx, int nrhs) {
  __shared__ T xbuf[kSWarps][32 * R];
  __shared__ T tbuf[kSWarps][32 * kTileLd];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = blockIdx.x * kSWarps + warp;
  if (slot >= count) return;
  bwd_small_front<T, R>(F, list[slot], panel, X, ldx, nrhs, xbuf[warp], tbuf[warp], lane);
}

// ---- large fronts: the solve vector of front f lives in V (nf per RHS) --------
// Panel steps of kSolveB = 128 columns use the inverted diagonal blocks kept
// from the factorization (Li = L_ss^{-1}), one launch per step:
//   forward : v_rest -= L_rest,s y_s over 32-row chunks (k_fwd_large_rest);
//             the last CTA of the front to finish (ticket) then forms the next
//             step's y_{s+1} = Li v_{s+1}; y_0 is formed by the gather kernel
//   backward: t_s = v_s - L_rest,s^T x_rest, partial sums per 64-row chunk;
//             the last CTA sums them in chunk order (deterministic) and forms
//             x_s = Li^T t_s (k_bwd_large_step)
// The diagonal solves write the front's own entries of X directly.
constexpr int kRhsG = 8;      // right-hand sides per pass
constexpr int kMrhsMin = 8;   // from this many right-hand sides on, GEMM-shaped large-front steps
constexpr int kFwdRows = 32;  // rows per CTA of k_fwd_large_rest

// y_s = Li v_s by one CTA of 256 threads: thread (row i, half h) sums k in
// [64h, 64h + 64) for a group of 8 right-hand sides (Li is zero above its
// diagonal and outside w x w, so the loops have fixed trip counts and the
// loads pipeline); halves meet in shared memory.  v is read past L1: other
// CTAs wrote it.
template <typename T>
__device__ void fwd_diag_cta(const DevFronts& F, int f, int step, int slot, const T* __restrict__ dinv, T* X,
                             int64_t ldx, T* Vf, int nf, int nrhs, T* vs, T* hs) {
  const int nc = F.nc[f];
  const int c0 = step * kSolveB;
  const int w = min(kSolveB, nc - c0);
  const T* Li = inv_block(F, dinv, f, step, slot);
  const int first = F.first[f];
  const int tid = threadIdx.x, i = tid & (kSolveB - 1), h = tid >> 7;
  for (int r0 = 0; r0 < nrhs; r0 += kRhsG) {
    const int g = min(kRhsG, nrhs - r0);
    __syncthreads();
    for (int e = tid; e < kSolveB * kRhsG; e += blockDim.x) {
      const int k = e % kSolveB, r = e / kSolveB;
      vs[k * kRhsG + r] = (k < w && r < g) ? __ldcg(&Vf[(int64_t)(r0 + r) * nf + c0 + k]) : T(0);
    }
    __syncthreads();
    T acc[kRhsG];
#pragma unroll
    for (int u = 0; u < kRhsG; ++u) acc[u] = T(0);
#pragma unroll 16
    for (int kk = 0; kk < kSolveB / 2; ++kk) {
      const int k = h * (kSolveB / 2) + kk;
      const T l = Li[i + k * kSolveB];
#pragma unroll
      for (int u = 0; u < kRhsG; ++u) acc[u] += l * vs[k * kRhsG + u];
    }
    if (h == 1)
#pragma unroll
      for (int u = 0; u < kRhsG; ++u) hs[i * kRhsG + u] = acc[u];
    __syncthreads();
    if (h == 0 && i < w) {
#pragma unroll
      for (int u = 0; u < kRhsG; ++u) {
        if (u < g) {
          const T y = acc[u] + hs[i * kRhsG + u];
          const int r = r0 + u;
          Vf[(int64_t)r * nf + c0 + i] = y;
          X[first + c0 + i + r * ldx] = y;
        }
      }
    }
  }
}

// gather v (own X entries + the children's update vectors), then y_0
template <typename T>
__global__ void __launch_bounds__(256) k_fwd_large_gather(DevFronts F, const int32_t* list,
                                                          const T* __restrict__ dinv, T* X, int64_t ldx, T* V,
                                                          int nrhs, int diag0) {
  __shared__ T vs[kSolveB * kRhsG];
  __shared__ T hs[kSolveB * kRhsG];
  const int f = list[blockIdx.x];
  const int nc = F.nc[f], nf = nc + F.nr[f], first = F.first[f];
  T* Vbase = V + F.v_off[f] * nrhs;
  // one right-hand side per CTA when the grid has a y extent (many RHS)
  const int rb = gridDim.y > 1 ? (int)blockIdx.y : 0, re = gridDim.y > 1 ? rb + 1 : nrhs;
  // loads batched kGU per thread (in flight together); each entry takes one
  // add per child, children in order
  constexpr int kGU = 4;
  const int nt = blockDim.x;
  for (int r = rb; r < re; ++r) {
    T* Vf = Vbase + (int64_t)r * nf;
    for (int i0 = threadIdx.x; i0 < nf; i0 += kGU * nt) {
      T xv[kGU];
#pragma unroll
      for (int u = 0; u < kGU; ++u) {
        const int i = i0 + u * nt;
        xv[u] = i < nc ? X[first + i + r * ldx] : T(0);
      }
#pragma unroll
      for (int u = 0; u < kGU; ++u)
        if (i0 + u * nt < nf) Vf[i0 + u * nt] = xv[u];
    }
    __syncthreads();
    for (int t = F.child_ptr[f]; t < F.child_ptr[f + 1]; ++t) {
      const int c = F.child[t];
      const int ncc = F.nc[c], nrc = F.nr[c];
      const T* Vc = V + F.v_off[c] * nrhs + (int64_t)r * (ncc + nrc) + ncc;
      const int32_t* loc = F.local + F.lrow_off[c];
      for (int i0 = threadIdx.x; i0 < nrc; i0 += kGU * nt) {
        int li[kGU];
        T cv[kGU], ov[kGU];
#pragma unroll
        for (int u = 0; u < kGU; ++u) {
          const int i = i0 + u * nt;
          li[u] = i < nrc ? loc[i] - 1 : -1;
          cv[u] = i < nrc ? Vc[i] : T(0);
        }
#pragma unroll
        for (int u = 0; u < kGU; ++u) ov[u] = li[u] >= 0 ? Vf[li[u]] : T(0);
#pragma unroll
        for (int u = 0; u < kGU; ++u)
          if (li[u] >= 0) Vf[li[u]] = ov[u] + cv[u];
      }
      __syncthreads();
    }
  }
  if (nrhs >= kMrhsMin || gridDim.y > 1 || !diag0) return;   // the GEMM-shaped diagonal kernel (or the fused sweep) follows
  __threadfence_block();
  fwd_diag_cta(F, f, 0, blockIdx.x, dinv, X, ldx, Vbase, nf, nrhs, vs, hs);
}

// v_rest -= L_rest,s y_s: 32 rows per CTA (lane = row), warp q takes panel
// columns 16q .. 16q+15 (held in registers), partial sums reduced in shared
// memory; the front's last CTA then forms y_{s+1}
template <typename T>
__global__ void __launch_bounds__(256) k_fwd_large_rest(DevFronts F, const int32_t* list, int step,
                                                        const T* __restrict__ panel, const T* __restrict__ dinv,
                                                        T* X, int64_t ldx, T* V, int32_t* cnt, int nrhs) {
  __shared__ T part[8][kRhsG][32];
  __shared__ T vs[kSolveB * kRhsG];
  __shared__ T hs[kSolveB * kRhsG];
  __shared__ int last;
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nf = nc + F.nr[f];
  pdl_wait();            // the previous step (or gather) of the sweep has completed
  pdl_trigger();
  const int c0 = step * kSolveB;
  if (c0 >= nc) return;
  const int w = min(kSolveB, nc - c0);
  const int rs0 = c0 + w;
  const int rbase = rs0 + blockIdx.x * kFwdRows;
  if (rbase >= nf) return;
  const int nchunks = (nf - rs0 + kFwdRows - 1) / kFwdRows;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i = rbase + lane;
  const bool valid = i < nf;
  const T* P = panel + F.panel_off[f];
  T* Vf = V + F.v_off[f] * nrhs;
  T lr[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int col = warp * 16 + k;
    lr[k] = (valid && col < w) ? P[i + (size_t)(c0 + col) * nf] : T(0);
  }
  for (int r0 = 0; r0 < nrhs; r0 += kRhsG) {
    const int g = min(kRhsG, nrhs - r0);
#pragma unroll
    for (int u = 0; u < kRhsG; ++u) {
      T s = T(0);
      if (u < g) {
        const T* y = Vf + (int64_t)(r0 + u) * nf + c0 + warp * 16;
#pragma unroll
        for (int k = 0; k < 16; ++k)
          if (warp * 16 + k < w) s += lr[k] * y[k];
      }
      part[warp][u][lane] = s;
    }
    __syncthreads();
    {
      const int u = threadIdx.x >> 5;
      if (u < g && valid) {
        T s = T(0);
#pragma unroll
        for (int q = 0; q < 8; ++q) s += part[q][u][lane];
        Vf[(int64_t)(r0 + u) * nf + i] -= s;
      }
    }
    __syncthreads();
  }
  if (rs0 >= nc) return;                                 // no next step for this front
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&cnt[blockIdx.y], 1) == nchunks - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  fwd_diag_cta(F, f, step + 1, blockIdx.y, dinv, X, ldx, Vf, nf, nrhs, vs, hs);
  if (threadIdx.x == 0) cnt[blockIdx.y] = 0;
}

// ---- single right-hand side: a level's large-front sweep in one launch ----------
// The sweep is a list of tasks in dependency order: forward, for each panel step
// s the diagonal-block task (f, s) of every front (y_s = Li (v_s - sum_{t<s}
// L_st y_t)), then the rest-row tasks (128 rows below the front's columns each,
// v_rest -= sum_t L_rest,t y_t); backward, for s from the last step down the
// column-block task (f, s) of every front (x_s = Li^T (v_s - L_below,s^T
// x_below)).  A CTA takes the next task from a ticket counter, so a task only
// waits (on the per-front, per-step flags the producing tasks release) for
// tasks that CTAs already running have taken: the sweep always progresses.
// Every wait is bounded (~1 s); on expiry the CTA raises `expired` and stops
// (the solve reports MFD_E_TIMEOUT).  Each task's sums have a fixed order, so
// the sweep is deterministic.
constexpr int kFuseRows = 128;                // rows of a forward rest task
constexpr long long kSolveWaitLimit = 1ll << 31;

__device__ __forceinline__ int ld_acquire_i32(const int32_t* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_i32(int32_t* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
constexpr long long kSolveProbeLimit = 1ll << 21;   // the test request's wait (~1 ms)
// thread 0 waits for *flag >= need (bounded; gives up at once when another
// CTA's wait expired); the result is the CTA's.  probe (a test request): the
// wait is for a value no producer writes, with a ~1 ms limit, so it expires.
__device__ __forceinline__ bool cta_wait_flag(const int32_t* flag, int32_t* expired, int* sh_ok, bool probe,
                                              int need = 1) {
  if (threadIdx.x == 0) {
    int ok = 1;
    if (probe) need = INT_MAX;
    const long long limit = probe ? kSolveProbeLimit : kSolveWaitLimit;
    if (ld_acquire_i32(flag) < need) {
      const long long t0 = clock64();
      while (ld_acquire_i32(flag) < need) {
        if (clock64() - t0 > limit || ld_acquire_i32(expired) != 0) {
          ok = 0;
          atomicExch(expired, 1);
          break;
        }
        __nanosleep(32);
      }
    }
    *sh_ok = ok;
  }
  __syncthreads();
  return *sh_ok != 0;
}

// forward: thread (row r0 + (t mod 128), half t / 128) sums its half of each
// step's 128 columns; the step's 64 panel entries are loaded before the wait on
// y_s (they do not depend on it)
template <typename T>
__global__ void __launch_bounds__(256) k_fwd_large_fused(DevFronts F, const int4* __restrict__ tasks, int ntask,
                                                         int32_t* ticket, int32_t* flags, int32_t* expired,
                                                         const T* __restrict__ panel, const T* __restrict__ dinv,
                                                         T* X, T* V, const int32_t* test_req) {
  __shared__ int sh_t, sh_ok;
  __shared__ T ys[kSolveB];
  __shared__ T part[kFuseRows];
  if (threadIdx.x == 0) sh_t = atomicAdd(ticket, 1);
  __syncthreads();
  const int t = sh_t;
  if (t >= ntask) return;
  const int4 tk = tasks[t];
  const int f = tk.x, code = tk.y;
  int32_t* fl = flags + tk.z;
  const bool probe = *test_req != 0;
  const int nc = F.nc[f], nf = nc + F.nr[f];
  const int r0 = code >= 0 ? code * kSolveB : nc + (-1 - code) * kFuseRows;
  const int r1 = code >= 0 ? min(nc, r0 + kSolveB) : min(nf, r0 + kFuseRows);
  const int nsteps = code >= 0 ? code : (nc + kSolveB - 1) / kSolveB;   // steps whose y this task consumes
  const T* P = panel + F.panel_off[f];
  T* Vf = V + F.v_off[f];
  const int tid = threadIdx.x, ri = tid & (kFuseRows - 1), h = tid >> 7;
  const int i = r0 + ri;
  const bool valid = i < r1;
  T acc = T(0);
  for (int s = 0; s < nsteps; ++s) {
    const int c0 = s * kSolveB, w = min(kSolveB, nc - c0);
    T l[64];
    const T* pc = P + (valid ? i : 0) + (size_t)(c0 + 64 * h) * nf;
#pragma unroll
    for (int k = 0; k < 64; ++k) l[k] = (valid && 64 * h + k < w) ? pc[(size_t)k * nf] : T(0);
    if (!cta_wait_flag(fl + s, expired, &sh_ok, probe)) return;
    if (tid < kSolveB) ys[tid] = tid < w ? __ldcg(&Vf[c0 + tid]) : T(0);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 64; ++k) acc += l[k] * ys[64 * h + k];
    __syncthreads();
  }
  if (h == 1) part[ri] = acc;
  __syncthreads();
  T v = T(0);
  if (h == 0 && valid) v = Vf[i] - (acc + part[ri]);
  if (code < 0) {
    if (h == 0 && valid) Vf[i] = v;
    return;
  }
  if (h == 0) ys[ri] = valid ? v : T(0);
  __syncthreads();
  const T* Li = inv_block(F, dinv, f, code, 0);    // zero outside its w x w part
  T y = T(0);
#pragma unroll 16
  for (int k = 0; k < 64; ++k) y += Li[ri + (size_t)(64 * h + k) * kSolveB] * ys[64 * h + k];
  if (h == 1) part[ri] = y;
  __syncthreads();
  if (h == 0 && valid) {
    const T yy = y + part[ri];
    Vf[i] = yy;
    X[F.first[f] + i] = yy;
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    st_release_i32(fl + code, 1);
  }
}

// backward: warp w takes columns 16 w .. 16 w + 15 of the block, lanes rows;
// the rows below the block in the update part (their x known from the gather)
// first, then the later diagonal blocks of the front from the last one down,
// each after its flag (its panel entries loaded before the wait); a butterfly
// transpose-reduce leaves column 16 w + (l mod 16)'s sum in lane l.
template <typename T>
__device__ __forceinline__ void bwd_rows_acc(const T* P, int nf, int c0, int w, int ra, int rb, const T* Vf, bool cg,
                                             int wc, int lane, T (&acc)[16]) {
  for (int rr = ra; rr < rb; rr += 32) {
    const int r = rr + lane;
    const bool ok = r < rb;
    const T xv = ok ? (cg ? __ldcg(&Vf[r]) : Vf[r]) : T(0);
    const T* pr = P + (ok ? r : ra) + (size_t)(c0 + wc) * nf;
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[j] += (ok && wc + j < w ? pr[(size_t)j * nf] : T(0)) * xv;
  }
}

// butterfly transpose-reduce of 16 per-lane column sums: lane l ends with column (l mod 16)'s sum
template <typename T>
__device__ __forceinline__ T transpose_reduce16(T (&acc)[16], int lane) {
#pragma unroll
  for (int sft = 8; sft >= 1; sft >>= 1) {
    const bool up = (lane & sft) != 0;
#pragma unroll
    for (int j = 0; j < sft; ++j) {
      const T send = up ? acc[j] : acc[j + sft];
      const T keep = up ? acc[j + sft] : acc[j];
      acc[j] = keep + __shfl_xor_sync(0xffffffffu, send, sft);
    }
  }
  return acc[0] + __shfl_xor_sync(0xffffffffu, acc[0], 16);
}

template <typename T>
__global__ void __launch_bounds__(256) k_bwd_large_fused(DevFronts F, const int4* __restrict__ tasks, int ntask,
                                                         int32_t* ticket, int32_t* flags, int32_t* expired,
                                                         const T* __restrict__ panel, const T* __restrict__ dinv,
                                                         T* X, T* V, T* part, int32_t* counters,
                                                         const int32_t* test_req) {
  __shared__ int sh_t, sh_ok;
  __shared__ T ts[kSolveB];
  if (threadIdx.x == 0) sh_t = atomicAdd(ticket, 1);
  __syncthreads();
  const int t = sh_t;
  if (t >= ntask) return;
  const int4 tk = tasks[t];
  const int f = tk.x;
  int32_t* fl = flags + tk.z;
  const bool probe = *test_req != 0;
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  const int nsteps = (nc + kSolveB - 1) / kSolveB;
  const int nch = (nr + kBwdRestRows - 1) / kBwdRestRows;
  const T* P = panel + F.panel_off[f];
  T* Vf = V + F.v_off[f];
  T* Pt = part + tk.w;                        // the front's partial sums: [step][chunk][128]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wc = 16 * warp;
  T acc[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) acc[j] = T(0);
  if (tk.y < 0) {                             // update-row chunk j against column block s (x gathered)
    const int code = -1 - tk.y, s = code >> 16, j = code & 0xffff;
    const int c0 = s * kSolveB, w = min(kSolveB, nc - c0);
    const int ra = nc + j * kBwdRestRows;
    bwd_rows_acc(P, nf, c0, w, ra, min(nf, ra + kBwdRestRows), Vf, false, wc, lane, acc);
    const T sum = transpose_reduce16(acc, lane);
    if (lane < 16) Pt[((size_t)s * nch + j) * kSolveB + wc + lane] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&counters[tk.z + s], 1);
    }
    return;
  }
  const int s = tk.y;
  const int c0 = s * kSolveB, w = min(kSolveB, nc - c0);
  for (int b = nsteps - 1; b > s; --b) {                                   // later diagonal blocks
    const int ra = b * kSolveB, rb = min(nc, ra + kSolveB);
    T l[4][16];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ra + lane + 32 * q;
      const T* pr = P + (r < rb ? r : ra) + (size_t)(c0 + wc) * nf;
#pragma unroll
      for (int j = 0; j < 16; ++j) l[q][j] = (r < rb && wc + j < w) ? pr[(size_t)j * nf] : T(0);
    }
    if (!cta_wait_flag(fl + b, expired, &sh_ok, probe)) return;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ra + lane + 32 * q;
      const T xv = r < rb ? __ldcg(&Vf[r]) : T(0);
#pragma unroll
      for (int j = 0; j < 16; ++j) acc[j] += l[q][j] * xv;
    }
  }
  const T dsum = transpose_reduce16(acc, lane);           // lane l: column wc + (l mod 16), diagonal blocks
  // the update rows' partial sums, chunk by chunk in order, once every chunk task has counted in
  if (nch > 0 && !cta_wait_flag(counters + tk.z + s, expired, &sh_ok, probe, nch)) return;
  if (lane < 16) {
    const int c = wc + lane;
    T rsum = T(0);
    for (int j = 0; j < nch; ++j) rsum += __ldcg(&Pt[((size_t)s * nch + j) * kSolveB + c]);
    ts[c] = c < w ? Vf[c0 + c] - (rsum + dsum) : T(0);
  }
  __syncthreads();
  // x = Li^T t: column i of Li against t, lanes over k (coalesced), 16 columns per warp
  const T* Li = inv_block(F, dinv, f, s, 0);
  T tv[kSolveB / 32];
#pragma unroll
  for (int q = 0; q < kSolveB / 32; ++q) tv[q] = ts[lane + 32 * q];
  const int first = F.first[f];
#pragma unroll 4
  for (int cc = 0; cc < 16; ++cc) {
    const int i = wc + cc;
    const T* lcol = Li + (size_t)i * kSolveB + lane;
    T sum = T(0);
#pragma unroll
    for (int q = 0; q < kSolveB / 32; ++q) sum += lcol[32 * q] * tv[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0 && i < w) {
      Vf[c0 + i] = sum;
      X[first + c0 + i] = sum;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release_i32(fl + s, 1);
  }
}

template <typename T>
__global__ void k_bwd_large_gather(DevFronts F, const int32_t* list, const T* X, int64_t ldx, T* V, int nrhs) {
  const int f = list[blockIdx.x];
  const int nc = F.nc[f], nf = nc + F.nr[f], first = F.first[f];
  const int32_t* lr = F.lrow + F.lrow_off[f];
  const int rb = gridDim.y > 1 ? (int)blockIdx.y : 0, re = gridDim.y > 1 ? rb + 1 : nrhs;
  constexpr int kGU = 4;                     // loads in flight per thread
  const int nt = blockDim.x;
  for (int r = rb; r < re; ++r) {
    T* Vf = V + F.v_off[f] * nrhs + (int64_t)r * nf;
    for (int i0 = threadIdx.x; i0 < nf; i0 += kGU * nt) {
      int gi[kGU];
#pragma unroll
      for (int u = 0; u < kGU; ++u) {
        const int i = i0 + u * nt;
        gi[u] = i < nc ? first + i : (i < nf ? lr[i - nc] : -1);
      }
      T xv[kGU];
#pragma unroll
      for (int u = 0; u < kGU; ++u) xv[u] = gi[u] >= 0 ? X[gi[u] + r * ldx] : T(0);
#pragma unroll
      for (int u = 0; u < kGU; ++u)
        if (gi[u] >= 0) Vf[i0 + u * nt] = xv[u];
    }
  }
}

constexpr int kBwdG = 4;   // right-hand sides per pass of the backward partial sums

// ---- fused backward step (one launch per panel step) -------------------------
// Backward, any number of right-hand sides: every CTA writes its chunk's
// partial sums (64 rows; warp (g, q) takes rows 32g .. 32g+31 against the
// block's columns 32q .. 32q+31, lane = row, coalesced column reads, 16
// columns at a time, then a butterfly transpose-reduce leaves column kb +
// (l mod 16)'s sum in lane l); the last CTA of the front to finish (ticket on cnt[slot])
// sums them in chunk order (deterministic), forms x_s = Li^T t_s, writes V_s
// and X, and resets the ticket.  A front without rows below the block is
// finished by CTA 0 alone.  The finish reads Li straight from memory rather
// than caching a slice per thread, so the whole kernel fits 80 registers and
// three CTAs per SM (measured: 64^3 Laplacian FP64 solve 5.7 -> 5.1 ms).
template <typename T>
__global__ void __launch_bounds__(256, 3) k_bwd_large_step(DevFronts F, const int32_t* list, int step,
                                                        const T* __restrict__ panel, const T* __restrict__ dinv,
                                                        T* X, int64_t ldx, T* V, T* scratch, int32_t* cnt,
                                                        int nrhs) {
  constexpr int CW = kSolveB / 8;
  __shared__ T part[2][kBwdG][kSolveB];
  __shared__ T ts[kSolveB];
  __shared__ int last;
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nf = nc + F.nr[f];
  pdl_wait();            // the previous step (or gather) of the sweep has completed
  pdl_trigger();
  const int c0 = step * kSolveB;
  if (c0 >= nc) return;
  const int w = min(kSolveB, nc - c0);
  const int rs0 = c0 + w;
  const int nchunks = nf > rs0 ? (nf - rs0 + kSolveRows - 1) / kSolveRows : 0;
  const int rbase = rs0 + blockIdx.x * kSolveRows;
  if ((int)blockIdx.x >= max(nchunks, 1)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T* P = panel + F.panel_off[f];
  T* Vf = V + F.v_off[f] * nrhs;
  if (nchunks > 0) {
    const int rg = warp & 1, cq = warp >> 1;
    const int i = rbase + rg * 32 + lane;
    const bool valid = i < nf;
    for (int r0 = 0; r0 < nrhs; r0 += kBwdG) {
      const int g = min(kBwdG, nrhs - r0);
      T xi[kBwdG];
#pragma unroll
      for (int u = 0; u < kBwdG; ++u) xi[u] = (valid && u < g) ? Vf[(int64_t)(r0 + u) * nf + i] : T(0);
#pragma unroll 1
      for (int kb = 32 * cq; kb < 32 * cq + 32; kb += 16) {
        T pv[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) pv[j] = (valid && kb + j < w) ? P[i + (size_t)(c0 + kb + j) * nf] : T(0);
#pragma unroll
        for (int u = 0; u < kBwdG; ++u) {
          if (u >= g) break;
          T v[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = pv[j] * xi[u];
#pragma unroll
          for (int s = 8; s >= 1; s >>= 1) {
            const bool up = (lane & s) != 0;
#pragma unroll
            for (int j = 0; j < s; ++j) {
              const T send = up ? v[j] : v[j + s];
              const T keep = up ? v[j + s] : v[j];
              v[j] = keep + __shfl_xor_sync(0xffffffffu, send, s);
            }
          }
          v[0] += __shfl_xor_sync(0xffffffffu, v[0], 16);
          if (lane < 16) part[rg][u][kb + lane] = v[0];
        }
      }
      __syncthreads();
      for (int e = threadIdx.x; e < g * kSolveB; e += blockDim.x) {
        const int u = e / kSolveB, k = e % kSolveB;
        const T s = part[0][u][k] + part[1][u][k];
        scratch[F.s_off[f] * nrhs + ((int64_t)(r0 + u) * nchunks + blockIdx.x) * kSolveB + k] = s;
      }
      __syncthreads();
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&cnt[blockIdx.y], 1) == nchunks - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
  }
  // finish: x_s = Li^T (v_s - sum of partials)
  const T* Li = inv_block(F, dinv, f, step, blockIdx.y);
  const int first = F.first[f];
  for (int r = 0; r < nrhs; ++r) {
    __syncthreads();
    if (threadIdx.x < kSolveB) {
      T s = T(0);
      if (threadIdx.x < w) {
        s = Vf[(int64_t)r * nf + c0 + threadIdx.x];
        const T* pr = scratch + F.s_off[f] * nrhs + (int64_t)r * nchunks * kSolveB + threadIdx.x;
        for (int q0 = 0; q0 < nchunks; q0 += 8) {   // other CTAs' partials (read past L1), 8 loads in flight,
          T pv[8];                                   // subtracted in chunk order
#pragma unroll
          for (int q = 0; q < 8; ++q) pv[q] = q0 + q < nchunks ? __ldcg(pr + (int64_t)(q0 + q) * kSolveB) : T(0);
#pragma unroll
          for (int q = 0; q < 8; ++q) s -= pv[q];
        }
      }
      ts[threadIdx.x] = s;
    }
    __syncthreads();
    T tv[kSolveB / 32];
#pragma unroll
    for (int q = 0; q < kSolveB / 32; ++q) tv[q] = ts[lane + 32 * q];
#pragma unroll 4
    for (int cc = 0; cc < CW; ++cc) {   // Li(lane + 32q, warp*CW + cc), read here (registers for the partial phase)
      const T* lcol = Li + (size_t)(warp * CW + cc) * kSolveB + lane;
      T s = T(0);
#pragma unroll
      for (int q = 0; q < kSolveB / 32; ++q) s += lcol[32 * q] * tv[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      const int i = warp * CW + cc;
      if (lane == 0 && i < w) {
        Vf[(int64_t)r * nf + c0 + i] = s;
        X[first + c0 + i + r * ldx] = s;
      }
    }
  }
  if (nchunks > 0 && threadIdx.x == 0) cnt[blockIdx.y] = 0;
}

// ---- many right-hand sides (nrhs >= kMrhsMin): GEMM-shaped large-front steps --
// V of a front is an nf x nrhs column-major block (ld nf).  GEMMs over 64-wide
// RHS tiles, on m8n8k4 DMMA in FP64 (one 32 x 32 or 16 x 32 block per warp)
// and register-tiled FFMA in FP32; operands stream through shared memory in
// K chunks with cp.async double buffering (the next chunk's copies are in
// flight while the current one is multiplied):
//   forward step s : Y = Li V_s (k_mrhs_diag), V_rest -= L_rest,s Y (k_mrhs_fwd_rest)
//   backward step s: partial(chunk) = L_chunk,s^T X_chunk (k_mrhs_bwd_part, 64-row chunks),
//                    V_s -= sum of partials in chunk order (k_mrhs_bwd_reduce),
//                    X_s = Li^T V_s (k_mrhs_diag, transposed)
constexpr int kMT = 64;          // RHS tile
constexpr int kMKc = 16;         // K chunk

// FP64: one warp accumulates an (8 MF) x 32 block of C += A B over a K chunk
// of KC (a multiple of 4) on m8n8k4 DMMA, operands in shared memory as
// A(i, k) = As[k * lda + i], B(k, j) = Bs[k * ldb + j]; acc[m][n][e] holds
// C(wr + 8m + g, wc + 8n + 2q + e), g = lane / 4, q = lane % 4
template <int MF, int KC>
__device__ __forceinline__ void warp_mma_chunk(double (&acc)[MF][4][2], const double* As, int lda, const double* Bs,
                                               int ldb, int wr, int wc, int lane) {
  const int g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int k0 = 0; k0 < KC; k0 += 4) {
    double a[MF], b[4];
#pragma unroll
    for (int m = 0; m < MF; ++m) a[m] = As[(k0 + q) * lda + wr + 8 * m + g];
#pragma unroll
    for (int n = 0; n < 4; ++n) b[n] = Bs[(k0 + q) * ldb + wc + 8 * n + g];
#pragma unroll
    for (int m = 0; m < MF; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n) dmma(acc[m][n][0], acc[m][n][1], a[m], b[n]);
  }
}

// Y (128 x 64 RHS tile) = op(Li) V_s, op = identity or transpose; writes V_s and X
template <typename T>
__global__ void __launch_bounds__(256) k_mrhs_diag(DevFronts F, const int32_t* list, int step,
                                                   const T* __restrict__ dinv, T* X, int64_t ldx, T* V, int nrhs,
                                                   int transposed) {
  constexpr int KC = sizeof(T) == 8 ? 8 : 16;   // K chunk: two 128-wide stages under 48 KB
  __shared__ __align__(16) T As[2][KC][kSolveB + 4];   // op(Li)(i, k), [k][i]
  __shared__ __align__(16) T Bs[2][KC][kMT + 4];       // V_s(k, r)
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nf = nc + F.nr[f];
  const int c0 = step * kSolveB;
  if (c0 >= nc) return;
  const int w = min(kSolveB, nc - c0);
  const int r0 = blockIdx.x * kMT;
  if (r0 >= nrhs) return;
  const int rt = min(kMT, nrhs - r0);
  const T* Li = inv_block(F, dinv, f, step, blockIdx.y);
  T* Vf = V + F.v_off[f] * nrhs;
  auto load = [&](int buf, int k0) {
    for (int e = threadIdx.x; e < KC * kSolveB; e += blockDim.x) {
      int i, k;
      if (transposed) { k = e % KC; i = e / KC; }   // Li(k0 + k, i): k contiguous in global
      else { i = e % kSolveB; k = e / kSolveB; }         // Li(i, k0 + k): i contiguous
      const bool v = k0 + k < w && i < w;
      const T* src = transposed ? Li + (k0 + k) + (size_t)i * kSolveB : Li + i + (size_t)(k0 + k) * kSolveB;
      cp_async_t(&As[buf][k][i], v ? src : Li, v);
    }
    for (int e = threadIdx.x; e < KC * kMT; e += blockDim.x) {
      const int k = e % KC, r = e / KC;
      const bool v = k0 + k < w && r < rt;
      cp_async_t(&Bs[buf][k][r], v ? Vf + (int64_t)(r0 + r) * nf + c0 + k0 + k : Vf, v);
    }
    cp_async_commit();
  };
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // rows ty + 16 m (8), RHS tx + 16 n (4)
  T acc[8][4] = {};
  // FP64: DMMA, warp (warp % 4, warp / 4) owns rows 32 (warp % 4) .. +32, RHS 32 (warp / 4) .. +32
  double dacc[4][4][2] = {};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = 32 * (warp & 3), wc = 32 * (warp >> 2);
  const int nch = (w + KC - 1) / KC;
  load(0, 0);
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) {
      load((c + 1) & 1, (c + 1) * KC);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int b = c & 1;
    if constexpr (std::is_same<T, double>::value) {
      warp_mma_chunk<4, KC>(dacc, &As[b][0][0], kSolveB + 4, &Bs[b][0][0], kMT + 4, wr, wc, lane);
    } else {
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        T a[8], bv[4];
#pragma unroll
        for (int m = 0; m < 8; ++m) a[m] = As[b][k][ty + 16 * m];
#pragma unroll
        for (int n = 0; n < 4; ++n) bv[n] = Bs[b][k][tx + 16 * n];
#pragma unroll
        for (int m = 0; m < 8; ++m)
#pragma unroll
          for (int n = 0; n < 4; ++n) acc[m][n] += a[m] * bv[n];
      }
    }
    __syncthreads();
  }
  const int first = F.first[f];
  if constexpr (std::is_same<T, double>::value) {
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int i = wr + 8 * m + g, r = wc + 8 * n + 2 * q + e;
          if (i < w && r < rt) {
            Vf[(int64_t)(r0 + r) * nf + c0 + i] = dacc[m][n][e];
            X[first + c0 + i + (int64_t)(r0 + r) * ldx] = dacc[m][n][e];
          }
        }
  } else {
#pragma unroll
    for (int m = 0; m < 8; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const int i = ty + 16 * m, r = tx + 16 * n;
        if (i < w && r < rt) {
          Vf[(int64_t)(r0 + r) * nf + c0 + i] = acc[m][n];
          X[first + c0 + i + (int64_t)(r0 + r) * ldx] = acc[m][n];
        }
      }
  }
}

// V_rest(64-row tile, 64 RHS) -= L(rows, step columns) Y_s
template <typename T>
__global__ void __launch_bounds__(256) k_mrhs_fwd_rest(DevFronts F, const int32_t* list, int step,
                                                       const T* __restrict__ panel, T* V, int nrhs) {
  __shared__ __align__(16) T As[2][kMKc][kMT + 4];   // L(row, k), [k][row]
  __shared__ __align__(16) T Bs[2][kMKc][kMT + 4];   // Y(k, r)
  const int f = list[blockIdx.z];
  const int nc = F.nc[f], nf = nc + F.nr[f];
  const int c0 = step * kSolveB;
  if (c0 >= nc) return;
  const int w = min(kSolveB, nc - c0);
  const int i0 = c0 + w + blockIdx.x * kMT;
  if (i0 >= nf) return;
  const int r0 = blockIdx.y * kMT;
  if (r0 >= nrhs) return;
  const int rt = min(kMT, nrhs - r0);
  const T* P = panel + F.panel_off[f];
  T* Vf = V + F.v_off[f] * nrhs;
  auto load = [&](int buf, int k0) {
    for (int e = threadIdx.x; e < kMKc * kMT; e += blockDim.x) {
      const int i = e % kMT, k = e / kMT;
      const bool v = i0 + i < nf && k0 + k < w;
      cp_async_t(&As[buf][k][i], v ? P + (i0 + i) + (size_t)(c0 + k0 + k) * nf : P, v);
    }
    for (int e = threadIdx.x; e < kMKc * kMT; e += blockDim.x) {
      const int k = e % kMKc, r = e / kMKc;
      const bool v = k0 + k < w && r < rt;
      cp_async_t(&Bs[buf][k][r], v ? Vf + (int64_t)(r0 + r) * nf + c0 + k0 + k : Vf, v);
    }
    cp_async_commit();
  };
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // rows ty + 16 m (4), RHS tx + 16 n (4)
  T acc[4][4] = {};
  // FP64: DMMA, warp (warp % 4, warp / 4) owns rows 16 (warp % 4) .. +16, RHS 32 (warp / 4) .. +32
  double dacc[2][4][2] = {};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = 16 * (warp & 3), wc = 32 * (warp >> 2);
  const int nch = (w + kMKc - 1) / kMKc;
  load(0, 0);
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) {
      load((c + 1) & 1, (c + 1) * kMKc);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int b = c & 1;
    if constexpr (std::is_same<T, double>::value) {
      warp_mma_chunk<2, kMKc>(dacc, &As[b][0][0], kMT + 4, &Bs[b][0][0], kMT + 4, wr, wc, lane);
    } else {
#pragma unroll
      for (int k = 0; k < kMKc; ++k) {
        T a[4], bv[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) a[m] = As[b][k][ty + 16 * m];
#pragma unroll
        for (int n = 0; n < 4; ++n) bv[n] = Bs[b][k][tx + 16 * n];
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int n = 0; n < 4; ++n) acc[m][n] += a[m] * bv[n];
      }
    }
    __syncthreads();
  }
  if constexpr (std::is_same<T, double>::value) {
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int i = i0 + wr + 8 * m + g, r = wc + 8 * n + 2 * q + e;
          if (i < nf && r < rt) Vf[(int64_t)(r0 + r) * nf + i] -= dacc[m][n][e];
        }
  } else {
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const int i = i0 + ty + 16 * m, r = tx + 16 * n;
        if (i < nf && r < rt) Vf[(int64_t)(r0 + r) * nf + i] -= acc[m][n];
      }
  }
}

// partial(chunk)(128 columns, 64 RHS) = L(chunk rows, step columns)^T X(chunk rows), 64-row chunks
template <typename T>
__global__ void __launch_bounds__(256) k_mrhs_bwd_part(DevFronts F, const int32_t* list, int step,
                                                       const T* __restrict__ panel, const T* V, T* scratch,
                                                       int nrhs) {
  constexpr int KC = sizeof(T) == 8 ? 8 : 16;   // K chunk: two 128-wide stages under 48 KB
  __shared__ __align__(16) T As[2][KC][kSolveB + 4];   // L(row, col), [row][col]
  __shared__ __align__(16) T Bs[2][KC][kMT + 4];       // X(row, r)
  const int f = list[blockIdx.z];
  const int nc = F.nc[f], nf = nc + F.nr[f];
  const int c0 = step * kSolveB;
  if (c0 >= nc) return;
  const int w = min(kSolveB, nc - c0);
  const int rs0 = c0 + w;
  const int rbase = rs0 + blockIdx.x * kMrhsRows;
  if (rbase >= nf) return;
  const int nchunks = (nf - rs0 + kMrhsRows - 1) / kMrhsRows;
  const int r0 = blockIdx.y * kMT;
  if (r0 >= nrhs) return;
  const int rt = min(kMT, nrhs - r0);
  const int rend = min(nf, rbase + kMrhsRows);
  const T* P = panel + F.panel_off[f];
  const T* Vf = V + F.v_off[f] * nrhs;
  auto load = [&](int buf, int k0) {
    for (int e = threadIdx.x; e < KC * kSolveB; e += blockDim.x) {
      const int k = e % KC, col = e / KC;     // rows contiguous in global
      const bool v = k0 + k < rend && col < w;
      cp_async_t(&As[buf][k][col], v ? P + (k0 + k) + (size_t)(c0 + col) * nf : P, v);
    }
    for (int e = threadIdx.x; e < KC * kMT; e += blockDim.x) {
      const int k = e % KC, r = e / KC;
      const bool v = k0 + k < rend && r < rt;
      cp_async_t(&Bs[buf][k][r], v ? Vf + (int64_t)(r0 + r) * nf + k0 + k : Vf, v);
    }
    cp_async_commit();
  };
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // columns ty + 16 m (8), RHS tx + 16 n (4)
  T acc[8][4] = {};
  // FP64: DMMA, warp (warp % 4, warp / 4) owns rows 32 (warp % 4) .. +32, RHS 32 (warp / 4) .. +32
  double dacc[4][4][2] = {};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = 32 * (warp & 3), wc = 32 * (warp >> 2);
  const int nch = (rend - rbase + KC - 1) / KC;
  load(0, rbase);
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) {
      load((c + 1) & 1, rbase + (c + 1) * KC);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int b = c & 1;
    if constexpr (std::is_same<T, double>::value) {
      warp_mma_chunk<4, KC>(dacc, &As[b][0][0], kSolveB + 4, &Bs[b][0][0], kMT + 4, wr, wc, lane);
    } else {
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        T a[8], bv[4];
#pragma unroll
        for (int m = 0; m < 8; ++m) a[m] = As[b][k][ty + 16 * m];
#pragma unroll
        for (int n = 0; n < 4; ++n) bv[n] = Bs[b][k][tx + 16 * n];
#pragma unroll
        for (int m = 0; m < 8; ++m)
#pragma unroll
          for (int n = 0; n < 4; ++n) acc[m][n] += a[m] * bv[n];
      }
    }
    __syncthreads();
  }
  if constexpr (std::is_same<T, double>::value) {
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = wr + 8 * m + g, r = wc + 8 * n + 2 * q + e;
          if (col < w && r < rt)
            scratch[F.s_off[f] * nrhs + ((int64_t)(r0 + r) * nchunks + blockIdx.x) * kSolveB + col] = dacc[m][n][e];
        }
  } else {
#pragma unroll
    for (int m = 0; m < 8; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const int col = ty + 16 * m, r = tx + 16 * n;
        if (col < w && r < rt)
          scratch[F.s_off[f] * nrhs + ((int64_t)(r0 + r) * nchunks + blockIdx.x) * kSolveB + col] = acc[m][n];
      }
  }
}

// V_s(k, r) -= sum over chunks of partial (chunk order), one thread per entry
template <typename T>
__global__ void __launch_bounds__(256) k_mrhs_bwd_reduce(DevFronts F, const int32_t* list, int step, T* V,
                                                         const T* scratch, int nrhs) {
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nf = nc + F.nr[f];
  const int c0 = step * kSolveB;
  if (c0 >= nc) return;
  const int w = min(kSolveB, nc - c0);
  const int rs0 = c0 + w;
  const int nchunks = nf > rs0 ? (nf - rs0 + kMrhsRows - 1) / kMrhsRows : 0;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = e % kSolveB, r = e / kSolveB;
  if (nchunks == 0 || r >= nrhs || k >= w) return;
  T s = V[F.v_off[f] * nrhs + (int64_t)r * nf + c0 + k];
  for (int q = 0; q < nchunks; ++q) s -= scratch[F.s_off[f] * nrhs + ((int64_t)r * nchunks + q) * kSolveB + k];
  V[F.v_off[f] * nrhs + (int64_t)r * nf + c0 + k] = s;
}

// ============================================================================
// vectors
// ============================================================================
template <typename T>
__global__ void k_permute_in(const double* b, int64_t ldb, const int32_t* perm, T* X, int64_t ldx, int64_t n, int nrhs) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t src = perm[i];
    for (int r = 0; r < nrhs; ++r) X[i + r * ldx] = T(b[src + r * ldb]);
  }
}
template <typename T>
__global__ void k_permute_out(const T* X, int64_t ldx, const int32_t* perm, double* b, int64_t ldb, int64_t n, int nrhs) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t dst = perm[i];
    for (int r = 0; r < nrhs; ++r) b[dst + r * ldb] = double(X[i + r * ldx]);
  }
}
__global__ void k_gather_values(const double* a, const int32_t* src, double* out, int64_t count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = a[src[i]];
}
__global__ void k_residual(const int64_t* rowptr, const int32_t* col, const double* val, const double* x,
                           const double* b, double* r, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) s += val[e] * x[col[e]];
    r[i] = b[i] - s;
  }
}
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), __double_as_longlong(v));
}
// r = b - A x for k columns at once (x row-major: xt[i * k + c]): one warp per
// row, lanes over columns (32 at a time), the row's entries loaded 32 at a
// time and broadcast by shuffles; A is read once for all columns and the
// lanes' reads of a row of x are contiguous.  Entries are summed in row order,
// as in k_residual.
__global__ void k_residual_multi(const int64_t* rowptr, const int32_t* col, const double* val, const double* xt,
                                 const double* b, double* r, int64_t n, int k) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = w0; i < n; i += nw) {
    const int64_t e0 = rowptr[i], e1 = rowptr[i + 1];
    for (int c0 = 0; c0 < k; c0 += 32) {
      const int c = c0 + lane;
      double s = 0.0;
      for (int64_t eb = e0; eb < e1; eb += 32) {
        const int m = (int)min((int64_t)32, e1 - eb);
        int cj = 0;
        double av = 0.0;
        if (lane < m) {
          cj = col[eb + lane];
          av = val[eb + lane];
        }
        for (int t = 0; t < m; ++t) {
          const int j = __shfl_sync(0xffffffffu, cj, t);
          const double a = __shfl_sync(0xffffffffu, av, t);
          if (c < k) s += a * xt[(int64_t)j * k + c];
        }
      }
      if (c < k) r[i + (int64_t)c * n] = b[i + (int64_t)c * n] - s;
    }
  }
}
// column-major n x k (ld n) -> row-major, 32 x 32 tiles through shared memory
__global__ void k_to_rows(const double* x, double* xt, int64_t n, int k) {
  __shared__ double t[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int c = ty; c < 32; c += 8) t[c][tx] = (i0 + tx < n && c0 + c < k) ? x[i0 + tx + (int64_t)(c0 + c) * n] : 0.0;
  __syncthreads();
  for (int q = ty; q < 32; q += 8)
    if (i0 + q < n && c0 + tx < k) xt[(i0 + q) * k + c0 + tx] = t[tx][q];
}
// per column (grid y): out + 8 c gets max|r|, max|x|, max|b|, sum r^2, sum x^2
__global__ void k_norms(const double* r, const double* x, const double* b, int64_t n, double* out) {
  r += (int64_t)blockIdx.y * n;
  x += (int64_t)blockIdx.y * n;
  b += (int64_t)blockIdx.y * n;
  out += 8 * blockIdx.y;
  double mr = 0, mx = 0, mb = 0, sr = 0, sx = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double a = fabs(r[i]), c = fabs(x[i]), d = fabs(b[i]);
    mr = fmax(mr, a); mx = fmax(mx, c); mb = fmax(mb, d);
    sr += r[i] * r[i]; sx += x[i] * x[i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(out + 0, mr);
    atomic_max_nonneg(out + 1, mx);
    atomic_max_nonneg(out + 2, mb);
    atomicAdd(out + 3, sr);
    atomicAdd(out + 4, sx);
  }
}
__global__ void k_row_abs_max(const int64_t* rowptr, const double* val, int64_t n, double* out) {
  double m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0;
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) s += fabs(val[e]);
    m = fmax(m, s);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}
template <typename T>
__global__ void k_to_t(const double* in, T* out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = T(in[i]);
}
template <typename T>
__global__ void k_axpy_from_t(const T* d, double* x, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += double(d[i]);
}
__global__ void k_fill_int(int32_t* p, int32_t v, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

inline int grid_1d(int64_t n, int threads = 256) { return clamp_grid(ceil_div(n, threads), 148 * 16); }

template <typename T>
size_t small_front_smem(int nf_max) {   // packed front, kSfW pivot scales, a staged local_index
  return ((size_t)nf_max * (nf_max + 1) / 2 + kSfW) * sizeof(T) + (size_t)nf_max * sizeof(int);
}

// Dynamic shared memory above 48 KB is opted into once per kernel at handle
// creation (prepare_kernels), never inside a stream capture.
constexpr int kMaxDynSmem = 227 * 1024;
template <typename KernelT>
cudaError_t opt_in(KernelT k) {
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
}
template <typename KernelT>
void set_smem(KernelT, size_t) {}

}  // namespace

// ============================================================================
// launch wrappers
// ============================================================================
cudaError_t prepare_kernels() {
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) { if (r != cudaSuccess && e == cudaSuccess) e = r; };
  chk(opt_in(k_small_front<double, false>)); chk(opt_in(k_small_front<float, false>));
  chk(opt_in(k_small_front<double, true>)); chk(opt_in(k_small_front<float, true>));
  chk(opt_in(k_trsm2<double>)); chk(opt_in(k_trsm2<float>));
  chk(opt_in(k_update_dmma));
  chk(opt_in(k_potrf<double, 4>)); chk(opt_in(k_potrf<float, 4>));
  chk(opt_in(k_potrf<double, 3>)); chk(opt_in(k_potrf<float, 3>));
  chk(opt_in(k_potrf<double, 2>)); chk(opt_in(k_potrf<float, 2>));
  chk(opt_in(k_potrf<double, 1>)); chk(opt_in(k_potrf<float, 1>));
  chk(prepare_update_tc());
  chk(prepare_update_tcq());
  chk(opt_in(k_update_simt<double>)); chk(opt_in(k_update_simt<float>));
  chk(opt_in(k_update_dmma2));
  return e;
}

void launch_local_index(const DevFronts& F, int32_t* local, int num_front, cudaStream_t st) {
  if (num_front > 0) k_local_index<<<num_front, 128, 0, st>>>(F, local, num_front);
}
void launch_assembly_map(const DevFronts& F, const int32_t* col_front, const int32_t* acol_ptr, const int32_t* arow,
                         const int32_t* ccs_src, int32_t* sidx, int32_t* a_src, int32_t* a_pos, int n_total,
                         cudaStream_t st) {
  if (n_total > 0)
    k_assembly_map<<<ceil_div(n_total, 256), 256, 0, st>>>(F, col_front, acol_ptr, arow, ccs_src, sidx, a_src, a_pos,
                                                           n_total);
}
void launch_bli_count(const DevFronts& F, const int32_t* fronts, int count, int nb, int32_t* groups, cudaStream_t st) {
  if (count > 0) k_bli_count<<<ceil_div(count, 128), 128, 0, st>>>(F, fronts, count, nb, groups);
}
void launch_bli_fill(const DevFronts& F, const int32_t* fronts, int count, int nb, const int32_t* group_base,
                     const int32_t* index_base, int32_t* block_ptr, int32_t* pnum, int32_t* cnum, int32_t* offset,
                     int32_t* rebuilt, cudaStream_t st) {
  if (count > 0)
    k_bli_fill<<<ceil_div(count, 128), 128, 0, st>>>(F, fronts, count, nb, group_base, index_base, block_ptr, pnum,
                                                     cnum, offset, rebuilt);
}

template <typename T>
void launch_small_fronts(const DevFronts& F, const int32_t* list, int count, int nf_max, const double* a, T* panel,
                         T* upool, int32_t* info, cudaStream_t st) {
  if (count <= 0) return;
  if (nf_max <= kWF) {
    k_small_warp<T><<<ceil_div(count, kWFWarps), kWFWarps * 32, 0, st>>>(F, list, count, a, panel, upool, info);
    return;
  }
  size_t sm = small_front_smem<T>(nf_max);
  // 128 threads per front, so that shared memory and registers (not the
  // thread count) bound the fronts in flight per SM (measured faster than 256
  // on the 2,000-system batch, both variants)
  if (nf_max > 64) k_small_front<T, true><<<count, 128, sm, st>>>(F, list, a, panel, upool, info);
  else k_small_front<T, false><<<count, 128, sm, st>>>(F, list, a, panel, upool, info);
}
template <typename T>
void launch_zero_large(const DevFronts& F, const int32_t* list, int count, int64_t max_cols, T* panel, T* upool,
                       cudaStream_t st) {
  if (count <= 0) return;
  dim3 grid(clamp_grid(ceil_div(max_cols, 8), 512), count);
  k_zero_large<T><<<grid, 256, 0, st>>>(F, list, panel, upool);
}
template <typename T>
void launch_assemble_large(const DevFronts& F, const int32_t* list, int count, int max_entries, const double* a,
                           T* panel, cudaStream_t st) {
  if (count <= 0) return;
  dim3 grid(clamp_grid(ceil_div(max_entries, 256), 256), count);
  k_assemble_large<T><<<grid, 256, 0, st>>>(F, list, a, panel);
}
template <typename T>
void launch_extend_add(const DevFronts& F, const int32_t* list, int count, int max_nr, T* panel, T* upool,
                       cudaStream_t st) {
  if (count <= 0) return;
  if constexpr (sizeof(T) == 4) {   // one warp per column pair of the largest child, at most 1,024 CTAs per child
    const int gx = std::max(1, std::min(ceil_div((max_nr + 1) / 2, 8), 1024));
    k_extend_add_ilp<T><<<dim3(gx, count), 256, 0, st>>>(F, list, panel, upool);
    return;
  }
  dim3 grid(clamp_grid(ceil_div(max_nr, 8), 1024), count);
  k_extend_add<T><<<grid, 256, 0, st>>>(F, list, panel, upool);
}
template <typename T>
void launch_potrf(const DevFronts& F, const int32_t* list, int count, int step, T* panel, T* linv, int32_t* info,
                  cudaStream_t st, bool pdl, int info_stride, int32_t* fallbacks, const int32_t* cls) {
  if (count <= 0) return;
  if (cls == nullptr) {                   // one launch, any block width
    launch_k(k_potrf<T, 4>, dim3(count), dim3(potrf_threads<4>()), potrf_smem<4>(), st, pdl, F, list, step, panel,
             linv, info, info_stride, fallbacks);
    return;
  }
  // cls[k]: fronts of the list (in order, block widths non-increasing) whose block needs 4 - k sub-blocks;
  // the list slots of a launch are offset, so this form is for persistent inverse blocks (F.d_off)
  int off = 0;
  auto go = [&](auto kern, int nt, size_t smem, int cnt) {
    if (cnt > 0)
      launch_k(kern, dim3(cnt), dim3(nt), smem, st, pdl, F, list + off, step, panel, linv, info, info_stride,
               fallbacks);
    off += cnt;
  };
  go(k_potrf<T, 4>, potrf_threads<4>(), potrf_smem<4>(), cls[0]);
  go(k_potrf<T, 3>, potrf_threads<3>(), potrf_smem<3>(), cls[1]);
  go(k_potrf<T, 2>, potrf_threads<2>(), potrf_smem<2>(), cls[2]);
  go(k_potrf<T, 1>, potrf_threads<1>(), potrf_smem<1>(), cls[3]);
}
template <typename T>
void launch_trsm(const DevFronts& F, const int32_t* list, int count, int step, int row_blocks, T* panel,
                 const T* linv, int kind, cudaStream_t st, bool pdl, float* q) {
  if (count <= 0 || row_blocks <= 0) return;
  (void)kind;
  // row_blocks counts 64-row blocks
  dim3 grid(row_blocks * 2, count);
  launch_k(k_trsm2<T>, grid, dim3(256), trsm2_smem<T>(), st, pdl, F, list, step, panel, linv,
           sizeof(T) == 4 ? q : nullptr);
}
int update_grid(int T, int tw, UpdBand band) {
  const int c1 = kFactB / tw, jlo = band.blo * c1;
  if (T <= 0 || jlo >= T) return 0;
  if (band.bhi < 0) return (T - jlo) * (T - jlo + 1) / 2;
  return (T - jlo) * ((band.bhi - band.blo) * c1);
}

template <typename T>
int launch_update(const DevFronts& F, const int32_t* list, int count, int step, int T128, int T64, T* panel,
                  T* upool, int kind, cudaStream_t st, UpdBand band, int defer, bool pdl) {
  if (count <= 0) return 0;
  if constexpr (sizeof(T) == 8) {
    if (kind == 0) {                                   // 128 x 64 halves, two CTAs per SM
      const int g = update_grid(T128, kUT, band);
      if (g <= 0) return 0;
      launch_k(k_update_dmma2, dim3(2 * g, count), dim3(kU2Threads), kU2Smem, st, pdl, F, list, step,
               reinterpret_cast<double*>(panel), reinterpret_cast<double*>(upool), band.blo, band.bhi, defer);
      return 1;
    }
    if (kind == 3) {                                   // whole 128 x 128 tiles, one CTA per SM
      const int g = update_grid(T128, kUT, band);
      if (g <= 0) return 0;
      size_t sm = 2 * 2 * (size_t)kUK * kULD * sizeof(double);
      launch_k(k_update_dmma, dim3(g, count), dim3(kUThreads), sm, st, pdl, F, list, step, reinterpret_cast<double*>(panel),
               reinterpret_cast<double*>(upool), band.blo, band.bhi, defer);
      return 1;
    }
  }
  const int g = update_grid(T64, kSimtTile, band);
  if (g <= 0) return 0;
  size_t sm = 2 * (size_t)kSimtK * (kSimtTile + 4) * sizeof(T);
  k_update_simt<T><<<dim3(g, count), 256, sm, st>>>(F, list, step, panel, upool, band.blo, band.bhi, defer);
  return 1;
}

// one launch per size bin (nf_max <= 32 R, R <= kSmallFrontMax / 32 = 4)
template <typename T>
void launch_fwd_small(const DevFronts& F, const int32_t* list, int count, int nf_max, const T* panel, T* X,
                      int64_t ldx, T* V, int nrhs, cudaStream_t st) {
  if (count <= 0) return;
  const dim3 grid(ceil_div(count, kSWarps), nrhs >= kMrhsMin ? nrhs : 1), block(kSWarps * 32);
  switch (ceil_div(nf_max, 32)) {
    case 1: k_fwd_small<T, 1><<<grid, block, 0, st>>>(F, list, count, panel, X, ldx, V, nrhs); break;
    case 2: k_fwd_small<T, 2><<<grid, block, 0, st>>>(F, list, count, panel, X, ldx, V, nrhs); break;
    case 3: k_fwd_small<T, 3><<<grid, block, 0, st>>>(F, list, count, panel, X, ldx, V, nrhs); break;
    default: k_fwd_small<T, 4><<<grid, block, 0, st>>>(F, list, count, panel, X, ldx, V, nrhs); break;
  }
}
template <typename T>
void launch_bwd_small(const DevFronts& F, const int32_t* list, int count, int nf_max, const T* panel, T* X,
                      int64_t ldx, int nrhs, cudaStream_t st) {
  if (count <= 0) return;
  const dim3 grid(ceil_div(count, kSWarps), nrhs >= kMrhsMin ? nrhs : 1), block(kSWarps * 32);
  switch (ceil_div(nf_max, 32)) {
    case 1: k_bwd_small<T, 1><<<grid, block, 0, st>>>(F, list, count, panel, X, ldx, nrhs); break;
    case 2: k_bwd_small<T, 2><<<grid, block, 0, st>>>(F, list, count, panel, X, ldx, nrhs); break;
    case 3: k_bwd_small<T, 3><<<grid, block, 0, st>>>(F, list, count, panel, X, ldx, nrhs); break;
    default: k_bwd_small<T, 4><<<grid, block, 0, st>>>(F, list, count, panel, X, ldx, nrhs); break;
  }
}
template <typename T>
void launch_fwd_large(const DevFronts& F, const int32_t* list, int count, int max_nc, int max_nf, const T* panel,
                      const T* dinv, T* X, int64_t ldx, T* V, int32_t* cnt, int nrhs, cudaStream_t st,
                      int64_t* launches, bool pdl, bool fused) {
  if (count <= 0) return;
  k_fwd_large_gather<T><<<dim3(count, nrhs >= kMrhsMin ? nrhs : 1), 256, 0, st>>>(F, list, dinv, X, ldx, V, nrhs,
                                                                                    fused ? 0 : 1);
  if (fused) {                    // the level's steps as one launch (single right-hand side)
    if (launches) *launches += 1;
    return;
  }
  const int steps = ceil_div(max_nc, kSolveB);
  if (nrhs >= kMrhsMin) {
    const int rtiles = ceil_div(nrhs, kMT), rows = std::max(1, ceil_div(max_nf, kMT));
    for (int s = 0; s < steps; ++s) {
      k_mrhs_diag<T><<<dim3(rtiles, count), 256, 0, st>>>(F, list, s, dinv, X, ldx, V, nrhs, 0);
      k_mrhs_fwd_rest<T><<<dim3(rows, rtiles, count), 256, 0, st>>>(F, list, s, panel, V, nrhs);
    }
    if (launches) *launches += 1 + 2 * steps;
    return;
  }
  const int chunks = std::max(1, ceil_div(max_nf, kFwdRows));
  for (int s = 0; s < steps; ++s)
    launch_k(k_fwd_large_rest<T>, dim3(chunks, count), dim3(256), 0, st, pdl, F, list, s, panel, dinv, X, ldx, V, cnt,
             nrhs);
  if (launches) *launches += 1 + steps;
}
template <typename T>
void launch_bwd_large(const DevFronts& F, const int32_t* list, int count, int max_nc, int max_nf, const T* panel,
                      const T* dinv, T* X, int64_t ldx, T* V, T* scratch, int32_t* cnt, int nrhs, cudaStream_t st,
                      int64_t* launches, bool pdl, bool fused) {
  if (count <= 0) return;
  k_bwd_large_gather<T><<<dim3(count, nrhs >= kMrhsMin ? nrhs : 1), 256, 0, st>>>(F, list, X, ldx, V, nrhs);
  if (fused) {
    if (launches) *launches += 1;
    return;
  }
  const int steps = ceil_div(max_nc, kSolveB);
  const int chunks = std::max(1, ceil_div(max_nf, kSolveRows));
  if (nrhs >= kMrhsMin) {
    const int rtiles = ceil_div(nrhs, kMT);
    for (int s = steps - 1; s >= 0; --s) {
      k_mrhs_bwd_part<T><<<dim3(std::max(1, ceil_div(max_nf, kMrhsRows)), rtiles, count), 256, 0, st>>>(
          F, list, s, panel, V, scratch, nrhs);
      k_mrhs_bwd_reduce<T><<<dim3(ceil_div((int64_t)kSolveB * nrhs, 256), count), 256, 0, st>>>(F, list, s, V, scratch,
                                                                                                nrhs);
      k_mrhs_diag<T><<<dim3(rtiles, count), 256, 0, st>>>(F, list, s, dinv, X, ldx, V, nrhs, 1);
    }
    if (launches) *launches += 1 + 3 * steps;
    return;
  }
  for (int s = steps - 1; s >= 0; --s)
    launch_k(k_bwd_large_step<T>, dim3(chunks, count), dim3(256), 0, st, pdl, F, list, s, panel, dinv, X, ldx, V,
             scratch, cnt, nrhs);
  if (launches) *launches += 1 + steps;
}
template <typename T>
void launch_large_fused(const DevFronts& F, const int4* tasks, int ntask, bool backward, int32_t* ticket,
                        int32_t* flags, int32_t* expired, const T* panel, const T* dinv, T* X, T* V, cudaStream_t st,
                        const int32_t* test_req, T* part, int32_t* counters) {
  if (ntask <= 0) return;
  if (backward)
    k_bwd_large_fused<T><<<ntask, 256, 0, st>>>(F, tasks, ntask, ticket, flags, expired, panel, dinv, X, V, part,
                                                counters, test_req);
  else
    k_fwd_large_fused<T><<<ntask, 256, 0, st>>>(F, tasks, ntask, ticket, flags, expired, panel, dinv, X, V,
                                                test_req);
}

template <typename T>
void launch_permute_in(const double* b, int64_t ldb, const int32_t* perm, T* X, int64_t ldx, int64_t n, int nrhs,
                       cudaStream_t st) {
  k_permute_in<T><<<grid_1d(n), 256, 0, st>>>(b, ldb, perm, X, ldx, n, nrhs);
}
template <typename T>
void launch_permute_out(const T* X, int64_t ldx, const int32_t* perm, double* b, int64_t ldb, int64_t n, int nrhs,
                        cudaStream_t st) {
  k_permute_out<T><<<grid_1d(n), 256, 0, st>>>(X, ldx, perm, b, ldb, n, nrhs);
}
void launch_gather_values(const double* a, const int32_t* src, double* out, int64_t count, cudaStream_t st) {
  if (count > 0) k_gather_values<<<grid_1d(count), 256, 0, st>>>(a, src, out, count);
}
void launch_residual(const int64_t* rowptr, const int32_t* col, const double* val, const double* x, const double* b,
                     double* r, int64_t n, cudaStream_t st) {
  k_residual<<<grid_1d(n), 256, 0, st>>>(rowptr, col, val, x, b, r, n);
}
void launch_norms(const double* r, const double* x, const double* b, int64_t n, double* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, 5 * sizeof(double), st);
  k_norms<<<grid_1d(n), 256, 0, st>>>(r, x, b, n, out);
}
void launch_residual_multi(const int64_t* rowptr, const int32_t* col, const double* val, const double* x,
                           double* xt, const double* b, double* r, int64_t n, int k, double* out, cudaStream_t st) {
  if (n <= 0 || k <= 0) return;
  k_to_rows<<<dim3((unsigned)ceil_div(n, 32), (unsigned)ceil_div(k, 32)), 256, 0, st>>>(x, xt, n, k);
  k_residual_multi<<<grid_1d(n * 32), 256, 0, st>>>(rowptr, col, val, xt, b, r, n, k);
  cudaMemsetAsync(out, 0, 8 * sizeof(double) * k, st);
  k_norms<<<dim3(grid_1d(n), k), 256, 0, st>>>(r, x, b, n, out);
}
void launch_row_abs_max(const int64_t* rowptr, const double* val, int64_t n, double* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, sizeof(double), st);
  k_row_abs_max<<<grid_1d(n), 256, 0, st>>>(rowptr, val, n, out);
}
template <typename T>
void launch_to_t(const double* in, T* out, int64_t n, cudaStream_t st) {
  k_to_t<T><<<grid_1d(n), 256, 0, st>>>(in, out, n);
}
template <typename T>
void launch_axpy_from_t(const T* d, double* x, int64_t n, cudaStream_t st) {
  k_axpy_from_t<T><<<grid_1d(n), 256, 0, st>>>(d, x, n);
}
void launch_fill_int(int32_t* p, int32_t v, int64_t n, cudaStream_t st) {
  if (n > 0) k_fill_int<<<grid_1d(n), 256, 0, st>>>(p, v, n);
}
__global__ void k_ir_init(int32_t* st_i, double* st_d, double* prev, int nrhs) {
  for (int c = threadIdx.x; c < nrhs; c += blockDim.x) prev[c] = 1e300;
  if (threadIdx.x == 0) {
    st_i[0] = 0;
    st_i[1] = 1;
    st_d[0] = st_d[1] = 0.0;
  }
}
void launch_ir_init(int32_t* st_i, double* st_d, double* prev, int nrhs, cudaStream_t st) {
  k_ir_init<<<1, 128, 0, st>>>(st_i, st_d, prev, nrhs);
}
// one thread: the per-column test in column order, as the host loop does it
__global__ void k_ir_check(const double* norms, const double* anorm, int nrhs, double tol, int maxit, double* prev,
                           int32_t* st_i, double* st_d, cudaGraphConditionalHandle cond) {
  if (threadIdx.x != 0) return;
  const int it = st_i[0];                 // 0-based index of the sweep just done
  bool all_ok = true, all_stalled = it > 2;
  double worst = 0.0, worst_ref = 0.0;
  for (int c = 0; c < nrhs; ++c) {
    const double* v = norms + 8 * c;
    const double denom = anorm[0] * v[1] + v[2];
    const double cur = denom > 0 ? v[0] / denom : v[0];
    if (cur > tol) {
      all_ok = false;
      if (cur <= 0.9 * prev[c]) all_stalled = false;
    }
    if (cur >= worst) {
      worst = cur;
      worst_ref = v[4] > 0 ? sqrt(v[3]) / sqrt(v[4]) : sqrt(v[3]);
    }
    prev[c] = cur;
  }
  st_i[0] = it + 1;
  st_d[0] = worst;
  st_d[1] = worst_ref;
  const bool more = !(all_ok || all_stalled) && it + 1 < maxit;
  st_i[1] = more ? 1 : 0;
  cudaGraphSetConditional(cond, more ? 1u : 0u);
}
void launch_ir_check(const double* norms, const double* anorm, int nrhs, double tol, int maxit, double* prev,
                     int32_t* st_i, double* st_d, cudaGraphConditionalHandle cond, cudaStream_t st) {
  k_ir_check<<<1, 32, 0, st>>>(norms, anorm, nrhs, tol, maxit, prev, st_i, st_d, cond);
}

__global__ void k_remap_int(const int32_t* map, int32_t* a, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = map[a[i]];
}
void launch_remap_int(const int32_t* map, int32_t* a, int64_t n, cudaStream_t st) {
  if (n > 0) k_remap_int<<<grid_1d(n), 256, 0, st>>>(map, a, n);
}

#define MFD_INSTANTIATE(T)                                                                                          \
  template void launch_small_fronts<T>(const DevFronts&, const int32_t*, int, int, const double*, T*, T*, int32_t*, \
                                       cudaStream_t);                                                              \
  template void launch_zero_large<T>(const DevFronts&, const int32_t*, int, int64_t, T*, T*, cudaStream_t);         \
  template void launch_assemble_large<T>(const DevFronts&, const int32_t*, int, int, const double*, T*,             \
                                         cudaStream_t);                                                            \
  template void launch_extend_add<T>(const DevFronts&, const int32_t*, int, int, T*, T*, cudaStream_t);             \
  template void launch_potrf<T>(const DevFronts&, const int32_t*, int, int, T*, T*, int32_t*, cudaStream_t, bool,  \
                                int, int32_t*, const int32_t*);                                                    \
  template void launch_trsm<T>(const DevFronts&, const int32_t*, int, int, int, T*, const T*, int, cudaStream_t,   \
                               bool, float*);                                                                           \
  template int launch_update<T>(const DevFronts&, const int32_t*, int, int, int, int, T*, T*, int, cudaStream_t,    \
                                 UpdBand, int, bool);                                                              \
  template void launch_fwd_small<T>(const DevFronts&, const int32_t*, int, int, const T*, T*, int64_t, T*, int,    \
                                    cudaStream_t);                                                                 \
  template void launch_bwd_small<T>(const DevFronts&, const int32_t*, int, int, const T*, T*, int64_t, int,         \
                                    cudaStream_t);                                                                 \
  template void launch_fwd_large<T>(const DevFronts&, const int32_t*, int, int, int, const T*, const T*, T*,       \
                                    int64_t, T*, int32_t*, int, cudaStream_t, int64_t*, bool, bool);               \
  template void launch_bwd_large<T>(const DevFronts&, const int32_t*, int, int, int, const T*, const T*, T*,       \
                                    int64_t, T*, T*, int32_t*, int, cudaStream_t, int64_t*, bool, bool);           \
  template void launch_large_fused<T>(const DevFronts&, const int4*, int, bool, int32_t*, int32_t*, int32_t*,      \
                                      const T*, const T*, T*, T*, cudaStream_t, const int32_t*, T*, int32_t*);     \
  template void launch_permute_in<T>(const double*, int64_t, const int32_t*, T*, int64_t, int64_t, int,            \
                                     cudaStream_t);                                                                \
  template void launch_permute_out<T>(const T*, int64_t, const int32_t*, double*, int64_t, int64_t, int,           \
                                      cudaStream_t);                                                               \
  template void launch_to_t<T>(const double*, T*, int64_t, cudaStream_t);                                          \
  template void launch_axpy_from_t<T>(const T*, double*, int64_t, cudaStream_t);

MFD_INSTANTIATE(double)
MFD_INSTANTIATE(float)

}  // namespace mfd
