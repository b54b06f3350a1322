// Host side of the C ABI (include/mfdag.h): handle, static plan, graph-captured
// launch sequences, iterative refinement, exports, and the reference-named
// hppllt_* entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mfdag.h"
#include "analysis.hpp"
#include "kernels.cuh"
#include "plan.hpp"

namespace mfd {
namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? MFD_E_NOMEM : MFD_E_CUDA,                \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

constexpr int64_t kAlign = 32;  // elements; keeps every front 256-byte aligned in FP64
constexpr int kResMulti = 4;     // from this many right-hand sides on, one multi-column residual per IR sweep
constexpr int kPotrfSplitMin = 148;   // fronts in a panel step above which POTRF launches per width class
// panel steps per deferred trailing update: FP64 2 (64^3 Laplacian 38.1 -> 37.7 ms: K = 256 per pass
// halves the C traffic of the DMMA update); FP32 1 (the packed-operand tensor-core update needs it)
constexpr int kDeferDefaultFp64 = 2, kDeferDefaultFp32 = 1;
int64_t align_up(int64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    release();
    n = count;
    return cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
  }
  cudaError_t upload(const std::vector<T>& v, cudaStream_t st) {
    cudaError_t e = alloc(v.size());
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
  }
};

// best-fit allocator over a simulated address space (static memory plan):
// free blocks indexed by address (for coalescing) and by (size, address) (for
// the search; erasing one block is O(log F) even when thousands of blocks have
// the same size, as in a batch of equal systems), so a plan over millions of
// fronts stays O(F log F)
struct BestFit {
  std::map<int64_t, int64_t> by_addr;            // offset -> size
  std::set<std::pair<int64_t, int64_t>> by_size; // (size, offset)
  int64_t top = 0;
  void insert(int64_t off, int64_t size) {
    by_addr[off] = size;
    by_size.emplace(size, off);
  }
  int64_t alloc(int64_t size) {
    size = align_up(std::max<int64_t>(size, 1));
    auto it = by_size.lower_bound({size, INT64_MIN});
    if (it != by_size.end()) {
      int64_t have = it->first, off = it->second;
      by_size.erase(it);
      by_addr.erase(off);
      if (have > size) insert(off + size, have - size);
      return off;
    }
    // extend the top, reusing a free block that ends there
    if (!by_addr.empty()) {
      auto last = std::prev(by_addr.end());
      if (last->first + last->second == top) {
        int64_t off = last->first;
        by_size.erase({last->second, off});
        by_addr.erase(last);
        top = off + size;
        return off;
      }
    }
    int64_t off = top;
    top += size;
    return off;
  }
  void release(int64_t off, int64_t size) {
    size = align_up(std::max<int64_t>(size, 1));
    auto nx = by_addr.lower_bound(off);
    if (nx != by_addr.end() && off + size == nx->first) {
      size += nx->second;
      by_size.erase({nx->second, nx->first});
      nx = by_addr.erase(nx);
    }
    if (nx != by_addr.begin()) {
      auto pv = std::prev(nx);
      if (pv->first + pv->second == off) {
        off = pv->first;
        size += pv->second;
        by_size.erase({pv->second, pv->first});
        by_addr.erase(pv);
      }
    }
    insert(off, size);
  }
};

struct SmallBin {
  int nf_max;
};

}  // namespace
}  // namespace mfd

namespace mfd {
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace mfd

using namespace mfd;

struct mfd_handle {
  int device = 0;
  mfd_options opt{};
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;                       // lookahead: trailing updates off the panel critical path
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // deferred trailing updates: a bulk update on st2 in column bands, one event per band
  static constexpr int kMaxDefer = 8;
  cudaEvent_t ev_part[kMaxDefer] = {};
  int defer = 2;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // a level's independent launches (small-front size bins) on side streams,
  // forked from st at the level's start and joined back at its end
  static constexpr int kSide = 4;
  cudaStream_t sst[kSide] = {};
  cudaEvent_t ev_lvl = nullptr, ev_side[kSide] = {};

  // systems
  std::vector<Symbolic> sys;
  std::vector<int64_t> col_base, a_base;
  std::vector<int32_t> front_base;
  int64_t n_total = 0, nnz_total = 0;
  int64_t a_len = 0;                                // length of the caller's value array (CSR input: its nnz)
  int32_t num_front = 0;

  // host tables
  std::vector<HostFront> fronts;
  std::vector<int32_t> h_child_ptr, h_child, h_lrow_off, h_a_beg;
  std::vector<LevelPlan> levels;
  std::vector<int32_t> h_lists;
  std::vector<int32_t> h_stasks;                    // fused single-RHS solve tasks, 4 ints each
  int32_t solve_flags = 0;                          // per front and panel step, one sweep's worth
  int64_t bw_part_elems = 0;                        // backward sweep partial sums, largest level
  void* d_bwpart = nullptr;                         // T, the backward sweep's partial sums
  std::vector<int> small_bins;
  int64_t panel_elems = 0, upool_elems = 0, v_elems = 0, s_elems = 0, dinv_elems = 0;
  int64_t q_elems = 0;                              // packed FP32 update operands of one step parity
  int32_t max_large_count = 0, max_nf = 0;
  int64_t cost = 0, nonzero = 0;

  // device tables
  DBuf<int32_t> d_nc, d_nr, d_first, d_parent, d_child_ptr, d_child, d_lrow_off, d_lrow, d_local, d_a_beg, d_a_src,
      d_a_pos, d_sidx, d_lists, d_perm, d_info, d_cnt;
  // fused solve: the tasks, and [0] expiry flag, [1 + 2 l] / [2 + 2 l] level l's forward /
  // backward tickets, then forward and backward step flags (zeroed before every solve)
  DBuf<int32_t> d_stasks, d_ssync;
  DBuf<int64_t> d_panel_off, d_u_off, d_v_off, d_s_off, d_d_off, d_q_off;
  DevFronts F{};

  // CSR of the permuted full matrix (residuals)
  DBuf<int64_t> d_csr_ptr;
  DBuf<int32_t> d_csr_col, d_csr_src;
  DBuf<double> d_csr_val;

  // numeric storage
  bool fp32 = false;
  void* d_panel = nullptr;
  void* d_upool = nullptr;
  void* d_diag = nullptr;
  float* d_q = nullptr;                             // FP32: packed update operands, two step parities
  DBuf<double> d_a, d_b, d_xp, d_bp, d_r, d_norms, d_cnorms, d_xt;
  void* d_X = nullptr;   // T, n_total x nrhs
  void* d_V = nullptr;   // T
  void* d_S = nullptr;   // T
  int nrhs_cap = 0;

  // block-local index export (per system)
  std::vector<std::vector<int32_t>> bli_node_ptr, bli_block_ptr, bli_pnum, bli_cnum, bli_off, bli_val, local_sys,
      sidx_sys;

  bool factored = false;
  bool expire_waits = false;                        // test request (mfd_test_expire_waits)
  int64_t pivot_fallbacks = 0;                      // FP32 diagonal sub-blocks redone in FP64, last factorize
  int64_t launches_factor = 0, launches_solve = 0;
  double factor_ms = 0, solve_ms = 0, anorm = 0;
  double time_info[7] = {0, 0, 0, 0, 0, 0, 0};
  double setup_s[4] = {0, 0, 0, 0};                 // analysis, plan, device index maps + exports, CSR + storage
  cudaGraphExec_t g_factor = nullptr;
  std::map<int, cudaGraphExec_t> g_solve;
  std::map<int, cudaGraphExec_t> g_ir;              // FP32 + FP64 refinement, whole loop per RHS count
  cudaStream_t bst = nullptr;                       // captures the refinement loop's body
  DBuf<int32_t> d_ir_i;                             // refinement state (launch_ir_init / launch_ir_check)
  DBuf<double> d_ir_d, d_ir_prev;

  // per-kernel-class profiling (graphs off while enabled)
  bool profiling = false;
  mfd_kernel_profile prof[MFD_K_COUNT]{};
  struct PendingLaunch { int kind; double flops, bytes; cudaEvent_t a, b; };
  std::vector<PendingLaunch> pending;
  std::vector<cudaEvent_t> event_pool;

  ~mfd_handle() {
    if (st) cudaStreamSynchronize(st);
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    if (g_factor) cudaGraphExecDestroy(g_factor);
    for (auto& kv : g_solve) cudaGraphExecDestroy(kv.second);
    for (auto& kv : g_ir) cudaGraphExecDestroy(kv.second);
    if (bst) cudaStreamDestroy(bst);
    for (void* p : {d_panel, d_upool, d_diag, d_X, d_V, d_S, static_cast<void*>(d_q), d_bwpart})
      if (p) cudaFree(p);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    for (cudaEvent_t e : ev_part)
      if (e) cudaEventDestroy(e);
    if (ev_lvl) cudaEventDestroy(ev_lvl);
    for (int b = 0; b < kSide; ++b) {
      if (ev_side[b]) cudaEventDestroy(ev_side[b]);
      if (sst[b]) cudaStreamDestroy(sst[b]);
    }
    if (st2) cudaStreamDestroy(st2);
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

int small_front_max(const mfd_handle* h) {
  // fronts above 128 go to the blocked path: measured on the 64^3 Laplacian,
  // 128 is as fast as 160 (FP64) and 1.3 ms faster than 224 (FP32)
  int lim = kSmallFrontMax;
  if (h->opt.small_front_max > 0) lim = std::min(lim, h->opt.small_front_max);
  return lim;
}

int32_t push_list(mfd_handle* h, const std::vector<int32_t>& ids) {
  int32_t off = (int32_t)h->h_lists.size();
  h->h_lists.insert(h->h_lists.end(), ids.begin(), ids.end());
  return off;
}

// ---- plan construction --------------------------------------------------------
int build_plan(mfd_handle* h) {
  const int nsys = (int)h->sys.size();
  h->col_base.assign(nsys + 1, 0);
  h->a_base.assign(nsys + 1, 0);
  h->front_base.assign(nsys + 1, 0);
  for (int s = 0; s < nsys; ++s) {
    h->col_base[s + 1] = h->col_base[s] + h->sys[s].n;
    h->a_base[s + 1] = h->a_base[s] + h->sys[s].nnz;
    h->front_base[s + 1] = h->front_base[s] + h->sys[s].num_node;
  }
  h->n_total = h->col_base[nsys];
  h->nnz_total = h->a_base[nsys];
  h->num_front = h->front_base[nsys];
  if (h->n_total >= INT32_MAX || h->nnz_total >= INT32_MAX) return fail(MFD_E_ARG, "system too large for int32 indices");
  const int32_t nfr = h->num_front;
  h->fronts.assign(nfr, HostFront{});
  std::vector<int32_t> lrow_glob;
  h->h_lrow_off.assign(nfr + 1, 0);
  h->h_a_beg.assign(nfr + 1, 0);
  h->cost = h->nonzero = 0;
  for (int s = 0; s < nsys; ++s) {
    const Symbolic& S = h->sys[s];
    for (int node = 0; node < S.num_node; ++node) {
      int32_t g = h->front_base[s] + node;
      HostFront& fr = h->fronts[g];
      fr.nc = S.node_ptr[node + 1] - S.node_ptr[node];
      fr.nr = S.lrow_ptr[node + 1] - S.lrow_ptr[node];
      fr.first = (int32_t)(h->col_base[s] + S.node_ptr[node] - 1);
      fr.parent = S.parent[node] > 0 ? h->front_base[s] + S.parent[node] - 1 : -1;
      fr.sys = s;
      fr.node = node;
      h->h_lrow_off[g] = (int32_t)lrow_glob.size();
      for (int32_t k = S.lrow_ptr[node] - 1; k < S.lrow_ptr[node + 1] - 1; ++k)
        lrow_glob.push_back((int32_t)(h->col_base[s] + S.lrow[k] - 1));
      h->h_a_beg[g] = (int32_t)(h->a_base[s] + S.acol_ptr[S.node_ptr[node] - 1] - 1);
      for (int64_t k = fr.nr + 1; k <= fr.nr + fr.nc; ++k) {
        h->cost += k * k;
        h->nonzero += k;
      }
    }
  }
  h->h_lrow_off[nfr] = (int32_t)lrow_glob.size();
  h->h_a_beg[nfr] = (int32_t)h->nnz_total;
  // children lists (ascending node order == the reference's tree_child order)
  std::vector<int32_t> cnt(nfr, 0);
  for (int32_t g = 0; g < nfr; ++g)
    if (h->fronts[g].parent >= 0) cnt[h->fronts[g].parent]++;
  h->h_child_ptr.assign(nfr + 1, 0);
  for (int32_t g = 0; g < nfr; ++g) h->h_child_ptr[g + 1] = h->h_child_ptr[g] + cnt[g];
  h->h_child.assign(h->h_child_ptr[nfr], 0);
  {
    std::vector<int32_t> fill(h->h_child_ptr.begin(), h->h_child_ptr.end() - 1);
    for (int32_t g = 0; g < nfr; ++g)
      if (h->fronts[g].parent >= 0) h->h_child[fill[h->fronts[g].parent]++] = g;
  }
  // levels: height above the leaves (children precede parents in the numbering)
  int32_t nlev = 0;
  for (int32_t g = 0; g < nfr; ++g) {
    HostFront& fr = h->fronts[g];
    int lv = 0;
    for (int32_t t = h->h_child_ptr[g]; t < h->h_child_ptr[g + 1]; ++t)
      lv = std::max(lv, h->fronts[h->h_child[t]].level + 1);
    fr.level = lv;
    nlev = std::max(nlev, lv + 1);
  }
  // panel offsets, solve vector offsets, large-front solve scratch
  const int sfm = small_front_max(h);
  h->panel_elems = h->v_elems = h->s_elems = h->dinv_elems = 0;
  h->q_elems = 0;
  h->max_nf = 0;
  for (int32_t g = 0; g < nfr; ++g) {
    HostFront& fr = h->fronts[g];
    int nf = fr.nc + fr.nr;
    h->max_nf = std::max(h->max_nf, nf);
    fr.panel_off = h->panel_elems;
    h->panel_elems += align_up((int64_t)nf * fr.nc);
    fr.v_off = h->v_elems;
    h->v_elems += nf;
    fr.d_off = h->dinv_elems;
    if (nf > sfm) h->dinv_elems += (int64_t)((fr.nc + kFactB - 1) / kFactB) * kFactB * kFactB;   // kept for the solves
  }
  // large-front solve partials: one region per level (levels solve one after
  // another), kMrhsRows-row chunks (the single-RHS backward uses the same 64)
  {
    std::vector<int64_t> used(nlev, 0);
    for (int32_t g = 0; g < nfr; ++g) {
      HostFront& fr = h->fronts[g];
      const int nf = fr.nc + fr.nr;
      fr.s_off = used[fr.level];
      if (nf > sfm) used[fr.level] += (int64_t)((nf + kMrhsRows - 1) / kMrhsRows) * kSolveB;
    }
    for (int64_t u : used) h->s_elems = std::max(h->s_elems, u);
  }
  // update pool: static best-fit plan over level lifetimes
  {
    std::vector<std::vector<int32_t>> by_level(nlev);
    for (int32_t g = 0; g < nfr; ++g) by_level[h->fronts[g].level].push_back(g);
    BestFit ff;
    for (int l = 0; l < nlev; ++l) {
      for (int32_t g : by_level[l]) {
        int64_t nr = h->fronts[g].nr;
        h->fronts[g].u_off = ff.alloc(nr * nr);
      }
      for (int32_t g : by_level[l])
        for (int32_t t = h->h_child_ptr[g]; t < h->h_child_ptr[g + 1]; ++t) {
          const HostFront& c = h->fronts[h->h_child[t]];
          ff.release(c.u_off, (int64_t)c.nr * c.nr);
        }
    }
    h->upool_elems = std::max<int64_t>(ff.top, kAlign);
  }
  // level launch lists
  h->small_bins = std::vector<int>{32, 64, 96, 128};
  while (!h->small_bins.empty() && h->small_bins.back() > sfm) h->small_bins.pop_back();
  if (h->small_bins.empty() || h->small_bins.back() < sfm) h->small_bins.push_back(sfm);
  h->levels.assign(nlev, LevelPlan{});
  h->h_lists.clear();
  h->h_stasks.clear();
  h->solve_flags = 0;
  h->bw_part_elems = 0;
  h->max_large_count = 0;
  std::vector<std::vector<int32_t>> lev_fronts(nlev);
  for (int32_t g = 0; g < nfr; ++g) lev_fronts[h->fronts[g].level].push_back(g);
  for (int l = 0; l < nlev; ++l) {
    LevelPlan& L = h->levels[l];
    std::vector<std::vector<int32_t>> bins(h->small_bins.size());
    std::vector<int32_t> large;
    for (int32_t g : lev_fronts[l]) {
      int nf = h->fronts[g].nc + h->fronts[g].nr;
      if (nf <= sfm) {
        size_t b = 0;
        while (h->small_bins[b] < nf) ++b;
        bins[b].push_back(g);
      } else {
        large.push_back(g);
      }
    }
    for (size_t b = 0; b < bins.size(); ++b) {
      if (bins[b].empty()) continue;
      LaunchList ll;
      ll.off = push_list(h, bins[b]);
      ll.count = (int32_t)bins[b].size();
      ll.param = h->small_bins[b];
      L.small.push_back(ll);
    }
    if (large.empty()) continue;
    std::stable_sort(large.begin(), large.end(),
                     [&](int32_t a, int32_t b) { return h->fronts[a].nc > h->fronts[b].nc; });
    L.large.off = push_list(h, large);
    L.large.count = (int32_t)large.size();
    h->max_large_count = std::max(h->max_large_count, L.large.count);
    int max_entries = 0;
    int64_t max_elems = 0;
    int max_nc = 0;
    for (int32_t g : large) {
      const HostFront& fr = h->fronts[g];
      int nf = fr.nc + fr.nr;
      max_entries = std::max(max_entries, h->h_a_beg[g + 1] - h->h_a_beg[g]);
      max_elems = std::max<int64_t>(max_elems, nf);
      max_nc = std::max(max_nc, fr.nc);
      L.large_max_nf = std::max(L.large_max_nf, nf);
    }
    L.large.param = max_entries;
    L.large.param2 = max_nc;
    L.large_zero_elems = max_elems;
    // packed operands of the FP32 tensor-core update: the level's large fronts side by side,
    // each with the 128-row blocks of its largest step (step 0); reused level after level
    {
      int64_t q = 0;
      for (int32_t g : large) {
        HostFront& fr = h->fronts[g];
        const int64_t nrem = (int64_t)fr.nc + fr.nr - std::min(kFactB, fr.nc);
        fr.q_off = q;
        q += (nrem + kFactB - 1) / kFactB * kPackedBlockElems;
      }
      h->q_elems = std::max(h->q_elems, q);
    }
    // extend-add by child rank
    for (int rank = 0;; ++rank) {
      std::vector<int32_t> kids;
      int max_nr = 0;
      for (int32_t g : large) {
        int32_t t = h->h_child_ptr[g] + rank;
        if (t < h->h_child_ptr[g + 1]) {
          kids.push_back(h->h_child[t]);
          max_nr = std::max(max_nr, h->fronts[h->h_child[t]].nr);
        }
      }
      if (kids.empty()) break;
      LaunchList ll;
      ll.off = push_list(h, kids);
      ll.count = (int32_t)kids.size();
      ll.param = max_nr;
      L.ext_add.push_back(ll);
    }
    // panel steps: prefix of the nc-sorted list
    int steps = (max_nc + kFactB - 1) / kFactB;
    for (int s = 0; s < steps; ++s) {
      LaunchList ll;
      ll.off = L.large.off;
      int cntf = 0, rows = 0, tiles128 = 0, tiles64 = 0;
      for (int32_t g : large) {
        const HostFront& fr = h->fronts[g];
        if (fr.nc <= s * kFactB) break;
        ++cntf;
        int w = std::min(kFactB, fr.nc - s * kFactB);
        int nrem = fr.nc + fr.nr - s * kFactB - w;
        rows = std::max(rows, (nrem + kTrRowsH - 1) / kTrRowsH);
        tiles128 = std::max(tiles128, (nrem + kUpdTile - 1) / kUpdTile);          // tiles per side
        tiles64 = std::max(tiles64, (nrem + kUpdTileSimt - 1) / kUpdTileSimt);
      }
      ll.count = cntf;
      ll.param = rows;
      ll.param2 = tiles128;
      ll.param3 = tiles64;
      L.steps.push_back(ll);
      std::array<int32_t, 4> cls{0, 0, 0, 0};   // block widths are non-increasing along the nc-sorted list
      for (int k = 0; k < cntf; ++k) {
        const int w = std::min(kFactB, h->fronts[large[k]].nc - s * kFactB);
        ++cls[4 - (w + 31) / 32];
      }
      L.potrf_cls.push_back(cls);
    }
    // single-RHS solve tasks of the level, in dependency order (see launch_large_fused)
    {
      auto push_task = [&](int32_t g, int32_t code, int32_t flag) {
        h->h_stasks.insert(h->h_stasks.end(), {g, code, flag, 0});
      };
      std::vector<int32_t> fbase(large.size());
      for (size_t k = 0; k < large.size(); ++k) {
        fbase[k] = h->solve_flags;
        h->solve_flags += (h->fronts[large[k]].nc + kFactB - 1) / kFactB;
      }
      L.fwd_tasks.off = (int32_t)(h->h_stasks.size() / 4);
      for (int s = 0; s < steps; ++s)
        for (size_t k = 0; k < large.size(); ++k)
          if (h->fronts[large[k]].nc > s * kFactB) push_task(large[k], s, fbase[k]);
      for (size_t k = 0; k < large.size(); ++k)
        for (int j = 0; j * kFactB < h->fronts[large[k]].nr; ++j) push_task(large[k], -1 - j, fbase[k]);
      L.fwd_tasks.count = (int32_t)(h->h_stasks.size() / 4) - L.fwd_tasks.off;
      // backward: first the partial sums over the update rows (chunk j of kBwdRestRows rows
      // against column block s, no waits), then the column-block tasks from the last step down;
      // the fourth int is the front's partial-sum base in the level's scratch
      L.bwd_tasks.off = (int32_t)(h->h_stasks.size() / 4);
      std::vector<int32_t> pbase(large.size());
      int64_t pl = 0;
      for (size_t k = 0; k < large.size(); ++k) {
        const HostFront& fr = h->fronts[large[k]];
        const int ns = (fr.nc + kFactB - 1) / kFactB, nch = (fr.nr + kBwdRestRows - 1) / kBwdRestRows;
        pbase[k] = (int32_t)pl;
        pl += (int64_t)ns * nch * kFactB;
      }
      h->bw_part_elems = std::max(h->bw_part_elems, pl);
      auto push_bwd = [&](int32_t g, int32_t code, int32_t flag, int32_t pb) {
        h->h_stasks.insert(h->h_stasks.end(), {g, code, flag, pb});
      };
      for (size_t k = 0; k < large.size(); ++k) {
        const HostFront& fr = h->fronts[large[k]];
        const int ns = (fr.nc + kFactB - 1) / kFactB, nch = (fr.nr + kBwdRestRows - 1) / kBwdRestRows;
        for (int s = 0; s < ns; ++s)
          for (int j = 0; j < nch; ++j) push_bwd(large[k], -1 - ((s << 16) | j), fbase[k], pbase[k]);
      }
      for (int s = steps - 1; s >= 0; --s)
        for (size_t k = 0; k < large.size(); ++k)
          if (h->fronts[large[k]].nc > s * kFactB) push_bwd(large[k], s, fbase[k], pbase[k]);
      L.bwd_tasks.count = (int32_t)(h->h_stasks.size() / 4) - L.bwd_tasks.off;
    }
  }
  return MFD_OK;
}

int upload_plan(mfd_handle* h) {
  auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = h->st;
  const int32_t nfr = h->num_front;
  std::vector<int32_t> nc(nfr), nr(nfr), first(nfr), parent(nfr);
  std::vector<int64_t> poff(nfr), uoff(nfr), voff(nfr), soff(nfr), doff(nfr), qoff(nfr);
  for (int32_t g = 0; g < nfr; ++g) {
    const HostFront& f = h->fronts[g];
    nc[g] = f.nc; nr[g] = f.nr; first[g] = f.first; parent[g] = f.parent;
    poff[g] = f.panel_off; uoff[g] = f.u_off; voff[g] = f.v_off; soff[g] = f.s_off; doff[g] = f.d_off;
    qoff[g] = f.q_off;
  }
  std::vector<int32_t> lrow_glob;
  lrow_glob.reserve(h->h_lrow_off[nfr]);
  for (int s = 0; s < (int)h->sys.size(); ++s)
    for (int32_t v : h->sys[s].lrow) lrow_glob.push_back((int32_t)(h->col_base[s] + v - 1));
  CK(h->d_nc.upload(nc, st));
  CK(h->d_nr.upload(nr, st));
  CK(h->d_first.upload(first, st));
  CK(h->d_parent.upload(parent, st));
  CK(h->d_child_ptr.upload(h->h_child_ptr, st));
  CK(h->d_child.upload(h->h_child, st));
  CK(h->d_lrow_off.upload(h->h_lrow_off, st));
  CK(h->d_lrow.upload(lrow_glob, st));
  CK(h->d_local.alloc(std::max<size_t>(lrow_glob.size(), 1)));
  CK(h->d_a_beg.upload(h->h_a_beg, st));
  CK(h->d_panel_off.upload(poff, st));
  CK(h->d_u_off.upload(uoff, st));
  CK(h->d_v_off.upload(voff, st));
  CK(h->d_s_off.upload(soff, st));
  CK(h->d_d_off.upload(doff, st));
  CK(h->d_q_off.upload(qoff, st));
  CK(h->d_lists.upload(h->h_lists, st));
  // the fused sweeps' task entries hold 32-bit partial-sum bases and flag offsets: beyond that
  // range (far larger problems than one GPU holds) the per-step sweeps are used instead
  // (their flag array and partial-sum buffer then shrink to nothing)
  if (h->bw_part_elems > INT32_MAX || 3LL * h->solve_flags + 2LL * (int64_t)h->levels.size() + 1 > INT32_MAX) {
    h->h_stasks.clear();
    h->bw_part_elems = 0;
    h->solve_flags = 0;
  }
  if (!h->h_stasks.empty()) CK(h->d_stasks.upload(h->h_stasks, st));
  // [0] expiry, 2 tickets per level, forward flags, backward flags, backward update-row counters
  CK(h->d_ssync.alloc(1 + 2 * h->levels.size() + 3 * (size_t)h->solve_flags));
  CK(cudaMemsetAsync(h->d_ssync.p, 0, sizeof(int32_t) * h->d_ssync.n, st));
  CK(h->d_a_src.alloc(h->nnz_total));
  CK(h->d_a_pos.alloc(h->nnz_total));
  CK(h->d_sidx.alloc(h->nnz_total));
  // [0] first bad pivot column, [1] bounded-wait expiry flag, [2] test request: make the waits expire,
  // [3] FP32 diagonal sub-blocks redone in FP64 (small pivot)
  CK(h->d_info.alloc(4));
  CK(cudaMemsetAsync(h->d_info.p, 0, 4 * sizeof(int32_t), h->st));
  CK(h->d_cnt.alloc(std::max(1, h->max_large_count)));   // backward-solve tickets, one per list slot
  CK(cudaMemsetAsync(h->d_cnt.p, 0, sizeof(int32_t) * std::max(1, h->max_large_count), h->st));
  DevFronts& F = h->F;
  F.nc = h->d_nc.p; F.nr = h->d_nr.p; F.first = h->d_first.p; F.parent = h->d_parent.p;
  F.child_ptr = h->d_child_ptr.p; F.child = h->d_child.p; F.panel_off = h->d_panel_off.p; F.u_off = h->d_u_off.p;
  F.lrow_off = h->d_lrow_off.p; F.lrow = h->d_lrow.p; F.local = h->d_local.p; F.a_beg = h->d_a_beg.p;
  F.a_src = h->d_a_src.p; F.a_pos = h->d_a_pos.p; F.v_off = h->d_v_off.p; F.s_off = h->d_s_off.p;
  F.d_off = h->d_d_off.p;
  F.q_off = h->d_q_off.p;

  // permuted global A structure, value sources, front of every column
  std::vector<int32_t> acol(h->n_total + 1), arow(h->nnz_total), src(h->nnz_total), colf(h->n_total),
      perm(h->n_total);
  for (int s = 0; s < (int)h->sys.size(); ++s) {
    const Symbolic& S = h->sys[s];
    for (int32_t j = 0; j < S.n; ++j) {
      acol[h->col_base[s] + j] = (int32_t)(h->a_base[s] + S.acol_ptr[j] - 1);
      perm[h->col_base[s] + j] = (int32_t)(h->col_base[s] + S.perm[j] - 1);
    }
    for (int32_t k = 0; k < S.nnz; ++k) {
      arow[h->a_base[s] + k] = (int32_t)(h->col_base[s] + S.arow[k] - 1);
      src[h->a_base[s] + k] = (int32_t)(h->a_base[s] + S.ccs_perm[k] - 1);
    }
    for (int node = 0; node < S.num_node; ++node)
      for (int32_t j = S.node_ptr[node] - 1; j < S.node_ptr[node + 1] - 1; ++j)
        colf[h->col_base[s] + j] = h->front_base[s] + node;
  }
  acol[h->n_total] = (int32_t)h->nnz_total;
  CK(h->d_perm.upload(perm, st));
  DBuf<int32_t> d_acol, d_arow, d_src, d_colf;
  CK(d_acol.upload(acol, st));
  CK(d_arow.upload(arow, st));
  CK(d_src.upload(src, st));
  CK(d_colf.upload(colf, st));
  launch_local_index(F, h->d_local.p, nfr, st);
  launch_assembly_map(F, d_colf.p, d_acol.p, d_arow.p, d_src.p, h->d_sidx.p, h->d_a_src.p, h->d_a_pos.p,
                      (int)h->n_total, st);
  CK(cudaGetLastError());

  // block-local index per system (export for parity)
  const int nb = std::max(1, h->opt.nb);
  h->bli_node_ptr.assign(h->sys.size(), {});
  h->bli_block_ptr.assign(h->sys.size(), {});
  h->bli_pnum.assign(h->sys.size(), {});
  h->bli_cnum.assign(h->sys.size(), {});
  h->bli_off.assign(h->sys.size(), {});
  h->bli_val.assign(h->sys.size(), {});
  {
    std::vector<int32_t> all(nfr);
    for (int32_t g = 0; g < nfr; ++g) all[g] = g;
    DBuf<int32_t> d_all, d_groups;
    CK(d_all.upload(all, st));
    CK(d_groups.alloc(nfr));
    launch_bli_count(F, d_all.p, nfr, nb, d_groups.p, st);
    std::vector<int32_t> groups(nfr);
    CK(cudaMemcpyAsync(groups.data(), d_groups.p, sizeof(int32_t) * nfr, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // group / index bases relative to each system (1-based group ids)
    std::vector<int32_t> gbase(nfr), ibase(nfr);
    int64_t total_groups = 0;
    for (int s = 0; s < (int)h->sys.size(); ++s) {
      int32_t gacc = 0;
      auto& np = h->bli_node_ptr[s];
      np.assign(h->sys[s].num_node + 1, 1);
      for (int node = 0; node < h->sys[s].num_node; ++node) {
        int32_t g = h->front_base[s] + node;
        gbase[g] = (int32_t)(total_groups + gacc + 1);
        ibase[g] = h->sys[s].lrow_ptr[node] - 1;
        gacc += groups[g];
        np[node + 1] = 1 + gacc;
      }
      total_groups += gacc;
    }
    DBuf<int32_t> d_gbase, d_ibase, d_bptr, d_pnum, d_cnum, d_off, d_reb;
    CK(d_gbase.upload(gbase, st));
    CK(d_ibase.upload(ibase, st));
    CK(d_bptr.alloc(total_groups));
    CK(d_pnum.alloc(total_groups));
    CK(d_cnum.alloc(total_groups));
    CK(d_off.alloc(total_groups));
    // rebuilt values are written at the system-relative index: use a global buffer with per-system offsets
    CK(d_reb.alloc(std::max<size_t>(h->h_lrow_off[nfr], 1)));
    // rebuild index base = global lrow offset for the value array, system-relative for block_ptr
    std::vector<int32_t> vbase(nfr);
    for (int32_t g = 0; g < nfr; ++g) vbase[g] = h->h_lrow_off[g];
    DBuf<int32_t> d_vbase;
    CK(d_vbase.upload(vbase, st));
    // block_ptr needs system-relative bases; rebuilt needs global bases: run with system-relative bases for
    // block_ptr and fix the rebuilt values from local on the host side (same formula), cheaper than two passes.
    launch_bli_fill(F, d_all.p, nfr, nb, d_gbase.p, d_ibase.p, d_bptr.p, d_pnum.p, d_cnum.p, d_off.p, d_reb.p, st);
    CK(cudaGetLastError());
    std::vector<int32_t> bptr(total_groups), pn(total_groups), cn(total_groups), of(total_groups);
    std::vector<int32_t> local(h->h_lrow_off[nfr]), sidx(h->nnz_total);
    if (total_groups) {
      CK(cudaMemcpyAsync(bptr.data(), d_bptr.p, sizeof(int32_t) * total_groups, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(pn.data(), d_pnum.p, sizeof(int32_t) * total_groups, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(cn.data(), d_cnum.p, sizeof(int32_t) * total_groups, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(of.data(), d_off.p, sizeof(int32_t) * total_groups, cudaMemcpyDeviceToHost, st));
    }
    if (!local.empty())
      CK(cudaMemcpyAsync(local.data(), h->d_local.p, sizeof(int32_t) * local.size(), cudaMemcpyDeviceToHost, st));
    if (!sidx.empty())
      CK(cudaMemcpyAsync(sidx.data(), h->d_sidx.p, sizeof(int32_t) * sidx.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // every index the numeric kernels will follow must point inside its front
    for (int32_t v : local)
      if (v <= 0) return fail(MFD_E_ARG, "inconsistent symbolic structure (child row not in parent front)");
    for (int32_t v : sidx)
      if (v <= 0) return fail(MFD_E_ARG, "inconsistent symbolic structure (A entry outside its front)");
    // the rebuilt (mod nb) local values: k_bli_fill wrote them at system-relative offsets of d_reb, which
    // collide across systems; derive them per system from the device-built local index instead.
    h->local_sys.assign(h->sys.size(), {});
    h->sidx_sys.assign(h->sys.size(), {});
    int64_t goff = 0;
    for (int s = 0; s < (int)h->sys.size(); ++s) {
      int32_t ng = h->bli_node_ptr[s].back() - 1;
      h->bli_block_ptr[s].assign(bptr.begin() + goff, bptr.begin() + goff + ng);
      h->bli_block_ptr[s].push_back((int32_t)h->sys[s].lrow.size() + 1);
      h->bli_pnum[s].assign(pn.begin() + goff, pn.begin() + goff + ng);
      h->bli_cnum[s].assign(cn.begin() + goff, cn.begin() + goff + ng);
      h->bli_off[s].assign(of.begin() + goff, of.begin() + goff + ng);
      goff += ng;
      int32_t lo = h->h_lrow_off[h->front_base[s]], hi = h->h_lrow_off[h->front_base[s + 1]];
      h->local_sys[s].assign(local.begin() + lo, local.begin() + hi);
      h->bli_val[s].resize(h->local_sys[s].size());
      for (size_t i = 0; i < h->local_sys[s].size(); ++i) h->bli_val[s][i] = (h->local_sys[s][i] - 1) % nb + 1;
      h->sidx_sys[s].assign(sidx.begin() + h->a_base[s], sidx.begin() + h->a_base[s + 1]);
    }
  }

  h->setup_s[2] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  t0 = std::chrono::steady_clock::now();
  // permuted full CSR (both triangles) for residuals
  {
    std::vector<int64_t> rp(h->n_total + 1, 0);
    for (int64_t j = 0; j < h->n_total; ++j)
      for (int32_t k = acol[j]; k < acol[j + 1]; ++k) {
        rp[arow[k] + 1]++;
        if (arow[k] != j) rp[j + 1]++;
      }
    for (int64_t i = 0; i < h->n_total; ++i) rp[i + 1] += rp[i];
    std::vector<int32_t> cols(rp.back()), srcs(rp.back());
    std::vector<int64_t> fill(rp.begin(), rp.end() - 1);
    for (int64_t j = 0; j < h->n_total; ++j)
      for (int32_t k = acol[j]; k < acol[j + 1]; ++k) {
        int32_t r = arow[k];
        cols[fill[r]] = (int32_t)j; srcs[fill[r]++] = src[k];
        if (r != j) { cols[fill[j]] = r; srcs[fill[j]++] = src[k]; }
      }
    CK(h->d_csr_ptr.upload(rp, st));
    CK(h->d_csr_col.upload(cols, st));
    CK(h->d_csr_src.upload(srcs, st));
    CK(h->d_csr_val.alloc(cols.size()));
  }
  CK(cudaStreamSynchronize(st));

  // numeric storage
  size_t esz = h->fp32 ? sizeof(float) : sizeof(double);
  // 32 elements of slack: the FP32 tensor-core update copies column segments
  // in 16-byte chunks and may read up to 3 elements past the last panel
  CK(cudaMalloc(&h->d_panel, (std::max<int64_t>(h->panel_elems, 1) + 32) * esz));
  CK(cudaMalloc(&h->d_upool, std::max<int64_t>(h->upool_elems, 1) * esz));
  CK(cudaMalloc(&h->d_diag, (size_t)std::max<int64_t>(h->dinv_elems, 1) * esz));
  CK(cudaMalloc(&h->d_bwpart, (size_t)std::max<int64_t>(h->bw_part_elems, 1) * esz));
  if (h->fp32 && h->q_elems > 0) {
    CK(cudaMalloc(&h->d_q, (size_t)(2 * h->q_elems) * sizeof(float)));
    // rows past a front's last row are never written and only reach discarded outputs; zero keeps them finite
    CK(cudaMemsetAsync(h->d_q, 0, (size_t)(2 * h->q_elems) * sizeof(float), h->st));
  }
  // the inverted diagonal blocks are written on their lower w x w part only: the rest stays zero
  CK(cudaMemsetAsync(h->d_diag, 0, (size_t)std::max<int64_t>(h->dinv_elems, 1) * esz, h->st));
  h->a_len = h->nnz_total;
  CK(h->d_a.alloc(h->a_len));
  CK(h->d_norms.alloc(8));
  h->setup_s[3] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return MFD_OK;
}

int ensure_rhs(mfd_handle* h, int nrhs) {
  if (nrhs <= h->nrhs_cap) return MFD_OK;
  for (auto& kv : h->g_solve) cudaGraphExecDestroy(kv.second);
  h->g_solve.clear();
  for (auto& kv : h->g_ir) cudaGraphExecDestroy(kv.second);
  h->g_ir.clear();
  size_t esz = h->fp32 ? sizeof(float) : sizeof(double);
  for (void** p : {&h->d_X, &h->d_V, &h->d_S})
    if (*p) { cudaFree(*p); *p = nullptr; }
  CK(cudaMalloc(&h->d_X, (size_t)std::max<int64_t>(h->n_total, 1) * nrhs * esz));
  CK(cudaMalloc(&h->d_V, (size_t)std::max<int64_t>(h->v_elems, 1) * nrhs * esz));
  CK(cudaMalloc(&h->d_S, (size_t)std::max<int64_t>(h->s_elems, 1) * nrhs * esz));
  CK(h->d_b.alloc((size_t)h->n_total * nrhs));
  CK(h->d_xp.alloc((size_t)h->n_total * nrhs));
  CK(h->d_bp.alloc((size_t)h->n_total * nrhs));
  CK(h->d_r.alloc((size_t)h->n_total * nrhs));
  CK(h->d_cnorms.alloc((size_t)8 * nrhs));
  if (h->fp32 && nrhs >= kResMulti) CK(h->d_xt.alloc((size_t)h->n_total * nrhs));
  if (h->fp32) {
    CK(h->d_ir_i.alloc(2));
    CK(h->d_ir_d.alloc(2));
    CK(h->d_ir_prev.alloc(nrhs));
  }
  h->nrhs_cap = nrhs;
  return MFD_OK;
}

// ---- per-launch profiling ----------------------------------------------------------
cudaEvent_t take_event(mfd_handle* h, size_t idx) {
  while (h->event_pool.size() <= idx) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    h->event_pool.push_back(e);
  }
  return h->event_pool[idx];
}

// Side streams for one level's small-front bins: fork(k) makes the first k
// side streams wait for everything queued on st so far; join(k) makes st wait
// for them.  Concurrency is off in the profiling schedule (every kernel timed
// alone) and when reserved[4] = 1.
bool side_streams(const mfd_handle* h) { return !h->profiling && h->opt.reserved[4] != 1; }
void side_fork(mfd_handle* h, cudaStream_t st, int k) {
  cudaEventRecord(h->ev_lvl, st);
  for (int b = 0; b < k; ++b) cudaStreamWaitEvent(h->sst[b], h->ev_lvl, 0);
}
void side_join(mfd_handle* h, cudaStream_t st, int k) {
  for (int b = 0; b < k; ++b) {
    cudaEventRecord(h->ev_side[b], h->sst[b]);
    cudaStreamWaitEvent(st, h->ev_side[b], 0);
  }
}

// Runs `launch` and, when profiling, brackets it with events on the stream.
template <typename Fn>
void record(mfd_handle* h, cudaStream_t st, int kind, double flops, double bytes, Fn&& launch) {
  if (!h->profiling) {
    launch();
    return;
  }
  size_t i = h->pending.size() * 2;
  cudaEvent_t a = take_event(h, i), b = take_event(h, i + 1);
  cudaEventRecord(a, st);
  launch();
  cudaEventRecord(b, st);
  h->pending.push_back({kind, flops, bytes, a, b});
}

void collect_profile(mfd_handle* h) {
  for (auto& p : h->pending) {
    float ms = 0;
    cudaEventElapsedTime(&ms, p.a, p.b);
    mfd_kernel_profile& k = h->prof[p.kind];
    k.launches += 1;
    k.ms += ms;
    k.flops += p.flops;
    k.bytes += p.bytes;
  }
  h->pending.clear();
}

// algorithmic work of one front's fused factorization (w = element size)
void small_work(const mfd_handle* h, int32_t g, double w, double& flops, double& bytes) {
  const HostFront& f = h->fronts[g];
  double nc = f.nc, nr = f.nr, nf = nc + nr;
  for (int64_t k = f.nr + 1; k <= f.nr + f.nc; ++k) flops += (double)k * (double)k;
  bytes += w * (nf * nc - nc * (nc - 1) / 2 + nr * (nr + 1) / 2) + 12.0 * (h->h_a_beg[g + 1] - h->h_a_beg[g]);
  for (int32_t t = h->h_child_ptr[g]; t < h->h_child_ptr[g + 1]; ++t) {
    double c = h->fronts[h->h_child[t]].nr;
    bytes += w * c * (c + 1) / 2 + 4.0 * c;
  }
}

// ---- launch sequences ------------------------------------------------------------
template <typename T>
int64_t enqueue_factor(mfd_handle* h, cudaStream_t st) {
  int64_t n = 0;
  const DevFronts& F = h->F;
  T* panel = static_cast<T*>(h->d_panel);
  T* upool = static_cast<T*>(h->d_upool);
  T* diag = static_cast<T*>(h->d_diag);
  const int32_t* lists = h->d_lists.p;
  const double* a = h->d_a.p;
  const double w = sizeof(T);
  const bool prof = h->profiling;
  const int32_t* hl = h->h_lists.data();
  launch_fill_int(h->d_info.p, INT_MAX, 1, st);
  launch_fill_int(h->d_info.p + 1, 0, 1, st);
  launch_fill_int(h->d_info.p + 3, 0, 1, st);
  n += 3;
  // trailing update: 0 tensor cores (FP64: DMMA in 128 x 64 halves, two CTAs per SM; FP32: tcgen05 3xTF32),
  // 1 FFMA tiles, 2 tcgen05 1xTF32 (FP32), 3 FP64 DMMA in whole 128 x 128 tiles, one CTA per SM
  const int kind = h->opt.reserved[0];
  const bool side = side_streams(h);
  for (const LevelPlan& L : h->levels) {
    // the level's small-front bins and its large fronts are independent (their
    // children are on lower levels; their update matrices are distinct blocks)
    const int nside = side && (L.small.size() > 1 || L.large.count) ? (int)std::min<size_t>(L.small.size(), mfd_handle::kSide) : 0;
    if (nside) side_fork(h, st, nside);
    for (size_t b = 0; b < L.small.size(); ++b) {
      const LaunchList& s = L.small[b];
      cudaStream_t sb = (int)b < nside ? h->sst[b] : st;
      double fl = 0, by = 0;
      if (prof)
        for (int i = 0; i < s.count; ++i) small_work(h, hl[s.off + i], w, fl, by);
      record(h, sb, MFD_K_SMALL_FRONT, fl, by,
             [&] { launch_small_fronts<T>(F, lists + s.off, s.count, s.param, a, panel, upool, h->d_info.p, sb); });
      ++n;
    }
    if (L.large.count == 0) {
      if (nside) side_join(h, st, nside);
      continue;
    }
    double zb = 0, ab = 0;
    if (prof)
      for (int i = 0; i < L.large.count; ++i) {
        const HostFront& f = h->fronts[hl[L.large.off + i]];
        zb += w * ((double)(f.nc + f.nr) * f.nc - (double)f.nc * (f.nc - 1) / 2 + (double)f.nr * (f.nr + 1) / 2);
        ab += 12.0 * (h->h_a_beg[hl[L.large.off + i] + 1] - h->h_a_beg[hl[L.large.off + i]]);
      }
    record(h, st, MFD_K_ZERO, 0, zb,
           [&] { launch_zero_large<T>(F, lists + L.large.off, L.large.count, L.large_zero_elems, panel, upool, st); });
    record(h, st, MFD_K_ASSEMBLE, 0, ab,
           [&] { launch_assemble_large<T>(F, lists + L.large.off, L.large.count, L.large.param, a, panel, st); });
    n += 2;
    for (const LaunchList& e : L.ext_add) {
      double fl = 0, by = 0;
      if (prof)
        for (int i = 0; i < e.count; ++i) {
          double c = h->fronts[hl[e.off + i]].nr;
          fl += c * (c + 1) / 2;
          by += 3 * w * c * (c + 1) / 2 + 4.0 * c;
        }
      record(h, st, MFD_K_EXTEND_ADD, fl, by,
             [&] { launch_extend_add<T>(F, lists + e.off, e.count, e.param, panel, upool, st); });
      ++n;
    }
    // Lookahead (on unless reserved[1] = 1; profiling runs the serial schedule so
    // that every kernel is timed alone) with deferred updates (groups of D =
    // h->defer panel steps, update_k_range): after the TRSM of step s the next
    // panel's 128 columns take the current group's updates on the main stream
    // (the catch-up), so POTRF/TRSM of step s+1 can start; at a group's last
    // step the rest of the trailing matrix takes the whole group's K at once
    // (the bulk) on the side stream, in column bands: block s+1+k (k < D) first,
    // each followed by an event, then the rest.  The catch-up of step s+k waits
    // only for the band it overwrites.  Each tile sees the same K sequence in the
    // same order as in the serial schedule: bitwise identical results.
    const bool lookahead = h->opt.reserved[1] != 1 && !h->profiling;
    // programmatic dependent launch along the panel chain: opt-in (reserved[2] = 1).
    // Measured on the 64^3 Laplacian it costs 1-2 ms (early-launched CTAs wait on
    // SMs the side-stream update could use), so the default leaves it off.
    const bool pdl = h->opt.reserved[2] == 1 && !h->profiling;
    const int D = h->defer;
    // FP32 tensor-core update without deferral: the TRSM also writes the step's rows as
    // packed TF32 hi / lo operands (two buffers by step parity: with D = 1 the bulk update
    // of step s is complete before the TRSM of step s + 2 starts) for k_update_tcq
    const bool tcq = sizeof(T) == 4 && (kind == 0 || kind == 2) && D == 1 && h->d_q != nullptr;
    int pend = -1;                            // step of the latest bulk on st2 not yet fully waited for
    for (size_t s = 0; s < L.steps.size(); ++s) {
      const LaunchList& p = L.steps[s];
      double pf = 0, pb = 0, tf = 0, tb = 0;
      bool bulk_any = (s + 1) % D == 0;
      for (int i = 0; i < p.count; ++i) {
        const HostFront& f = h->fronts[hl[p.off + i]];
        if ((f.nc - 1) / kFactB <= (int)s + 1) bulk_any = true;
        if (!prof) continue;
        double c0 = (double)s * kFactB, wd = std::min<double>(kFactB, f.nc - c0);
        double nrem = f.nc + f.nr - c0 - wd;
        pf += wd * wd * wd / 3 + wd * wd * wd / 3;            // POTRF + triangular inverse
        pb += w * wd * wd * 2;
        tf += 2.0 * nrem * wd * wd;                          // X = A Li^T
        tb += w * (2.0 * nrem * wd + wd * wd);
      }
      // algorithmic work of an update launch over a band (update_k_range's rules)
      auto band_work = [&](UpdBand b, double& fl, double& by) {
        if (!prof) return;
        for (int i = 0; i < p.count; ++i) {
          const HostFront& f = h->fronts[hl[p.off + i]];
          const int last = (f.nc - 1) / kFactB, c0 = (int)s * kFactB, wd = std::min(kFactB, f.nc - c0);
          const double nrem = f.nc + f.nr - c0 - wd;
          const int g0 = (int)s >= last ? last : ((int)s / D) * D;
          const bool bulk = ((int)s + 1) % D == 0 || (int)s >= last - 1;
          const double K = std::min(f.nc, ((int)s + 1) * kFactB) - g0 * kFactB;
          for (int blk = b.blo; b.bhi < 0 || blk < b.bhi; ++blk) {
            const double a0 = (double)blk * kFactB, a1 = std::min(nrem, a0 + kFactB);
            if (a0 >= nrem) break;
            if (blk > 0 && !bulk) continue;
            const double el = (a1 - a0) * nrem - (a0 + a1 - 1) * (a1 - a0) / 2;   // lower-triangle entries
            fl += 2.0 * K * el;
            by += w * (2.0 * el + 2.0 * K * (nrem - a0));
          }
        }
      };
      record(h, st, MFD_K_PANEL, pf, pb,
             [&] {
               // many fronts: one launch per sub-block class (narrow blocks fit many CTAs per SM);
               // a few: one launch (measured: the extra launches on the panel chain cost more)
               launch_potrf<T>(F, lists + p.off, p.count, (int)s, panel, diag, h->d_info.p, st, pdl, 0,
                               h->d_info.p + 3, p.count > kPotrfSplitMin ? L.potrf_cls[s].data() : nullptr);
             });
      record(h, st, MFD_K_TRSM, tf, tb, [&] {
        launch_trsm<T>(F, lists + p.off, p.count, (int)s, p.param, panel, diag, kind == 1 ? 1 : 0, st, pdl,
                       tcq ? h->d_q + (s & 1) * h->q_elems : nullptr);
      });
      n += 2;
      auto update = [&](cudaStream_t us, UpdBand band) {
        double fl = 0, by = 0;
        band_work(band, fl, by);
        const bool upd_pdl = pdl && us == st;        // right behind the TRSM on the main stream
        record(h, us, MFD_K_UPDATE, fl, by, [&] {
          if constexpr (sizeof(T) == 4) {
            if (tcq) {
              n += launch_update_tcq(F, lists + p.off, p.count, (int)s, p.param2, h->d_q + (s & 1) * h->q_elems,
                                     reinterpret_cast<float*>(panel), reinterpret_cast<float*>(upool),
                                     kind == 0 ? 1 : 0, h->d_info.p + 1, us, band, upd_pdl);
              return;
            }
            if (kind == 0 || kind == 2) {
              n += launch_update_tc(F, lists + p.off, p.count, (int)s, p.param2, reinterpret_cast<float*>(panel),
                                    reinterpret_cast<float*>(upool), kind == 0 ? 1 : 0, h->d_info.p + 1, us, band,
                                    D, upd_pdl);
              return;
            }
          }
          n += launch_update<T>(F, lists + p.off, p.count, (int)s, p.param2, p.param3, panel, upool,
                                kind == 1 || kind == 3 ? kind : 0, us, band, D, upd_pdl && kind != 1);
        });
      };
      if (!lookahead || s + 1 == L.steps.size()) {
        if (pend >= 0) cudaStreamWaitEvent(st, h->ev_join, 0);
        pend = -1;
        update(st, UpdBand{0, -1});
        continue;
      }
      if (pend >= 0) {                       // the band of the pending bulk that holds block column s+1
        const int k = (int)s - pend;
        if (k >= D) {
          cudaStreamWaitEvent(st, h->ev_join, 0);
          pend = -1;
        } else {
          cudaStreamWaitEvent(st, h->ev_part[k], 0);
        }
      }
      update(st, UpdBand{0, 1});             // catch-up: the next panel's columns
      if (bulk_any) {
        cudaEventRecord(h->ev_fork, st);
        cudaStreamWaitEvent(h->st2, h->ev_fork, 0);
        for (int k = 1; k < D; ++k) {
          update(h->st2, UpdBand{k, k + 1});
          cudaEventRecord(h->ev_part[k], h->st2);
        }
        update(h->st2, UpdBand{D, -1});
        cudaEventRecord(h->ev_join, h->st2);
        pend = (int)s;
      }
    }
    if (nside) side_join(h, st, nside);
  }
  // values of the permuted full matrix for residuals
  record(h, st, MFD_K_OTHER, 0, 0, [&] {
    launch_gather_values(a, h->d_csr_src.p, h->d_csr_val.p, (int64_t)h->d_csr_val.n, st);
    launch_row_abs_max(h->d_csr_ptr.p, h->d_csr_val.p, h->n_total, h->d_norms.p + 7, st);
  });
  n += 2;
  return n;
}

template <typename T>
int64_t enqueue_solve_core(mfd_handle* h, int nrhs, cudaStream_t st) {
  int64_t n = 0;
  const DevFronts& F = h->F;
  const T* panel = static_cast<const T*>(h->d_panel);
  T* X = static_cast<T*>(h->d_X);
  T* V = static_cast<T*>(h->d_V);
  T* S = static_cast<T*>(h->d_S);
  const T* dinv = static_cast<const T*>(h->d_diag);
  const int32_t* lists = h->d_lists.p;
  const int64_t ldx = h->n_total;
  const double w = sizeof(T);
  const bool prof = h->profiling;
  const int32_t* hl = h->h_lists.data();
  // programmatic dependent launch between the large-front solve steps (on
  // unless reserved[3] = 1; the profiling schedule times kernels one by one)
  const bool solve_pdl = h->opt.reserved[3] != 1 && !prof;
  // one launch per level and sweep for the large fronts' steps (single right-hand side)
  const bool fused = nrhs == 1 && h->opt.reserved[6] != 1 && !h->h_stasks.empty();
  const int4* stasks = reinterpret_cast<const int4*>(h->d_stasks.p);
  int32_t* ssync = h->d_ssync.p;
  int32_t* fwd_flags = ssync + 1 + 2 * h->levels.size();
  int32_t* bwd_flags = fwd_flags + h->solve_flags;
  if (fused) {                              // a kernel, not a memset node: this also runs in the refinement loop's body
    launch_fill_int(ssync, 0, (int64_t)h->d_ssync.n, st);
    ++n;
  }
  // algorithmic work of one sweep over a list: read the panel once, 2 flops per entry per RHS
  auto work = [&](const LaunchList& l, double& fl, double& by) {
    if (!prof) return;
    for (int i = 0; i < l.count; ++i) {
      const HostFront& f = h->fronts[hl[l.off + i]];
      double e = (double)(f.nc + f.nr) * f.nc - (double)f.nc * (f.nc - 1) / 2;
      fl += 2.0 * e * nrhs;
      by += w * e + w * nrhs * (2.0 * (f.nc + f.nr) + f.nr);
    }
  };
  // per level, the small-front bins run on side streams next to the large
  // fronts (independent: each front reads its children's vectors, on lower
  // levels in the forward sweep and ancestors' X entries in the backward one)
  const bool side = side_streams(h);
  auto nside_of = [&](const LevelPlan& L) {
    return side && (L.small.size() > 1 || L.large.count) ? (int)std::min<size_t>(L.small.size(), mfd_handle::kSide) : 0;
  };
  for (const LevelPlan& L : h->levels) {
    const int nside = nside_of(L);
    if (nside) side_fork(h, st, nside);
    for (size_t b = 0; b < L.small.size(); ++b) {
      const LaunchList& s = L.small[b];
      cudaStream_t sb = (int)b < nside ? h->sst[b] : st;
      double fl = 0, by = 0;
      work(s, fl, by);
      record(h, sb, MFD_K_SOLVE_SMALL, fl, by,
             [&] { launch_fwd_small<T>(F, lists + s.off, s.count, s.param, panel, X, ldx, V, nrhs, sb); });
      ++n;
    }
    if (L.large.count) {
      double fl = 0, by = 0;
      work(L.large, fl, by);
      record(h, st, MFD_K_SOLVE_LARGE, fl, by, [&] {
        launch_fwd_large<T>(F, lists + L.large.off, L.large.count, L.large.param2, L.large_max_nf, panel, dinv, X,
                            ldx, V, h->d_cnt.p, nrhs, st, &n, solve_pdl, fused);
        if (fused) {
          const size_t lv = &L - h->levels.data();
          launch_large_fused<T>(F, stasks + L.fwd_tasks.off, L.fwd_tasks.count, false, ssync + 1 + 2 * lv, fwd_flags,
                                ssync, panel, dinv, X, V, st, h->d_info.p + 2);
          ++n;
        }
      });
    }
    if (nside) side_join(h, st, nside);
  }
  for (auto it = h->levels.rbegin(); it != h->levels.rend(); ++it) {
    const LevelPlan& L = *it;
    const int nside = nside_of(L);
    if (nside) side_fork(h, st, nside);
    for (size_t b = 0; b < L.small.size(); ++b) {
      const LaunchList& s = L.small[b];
      cudaStream_t sb = (int)b < nside ? h->sst[b] : st;
      double fl = 0, by = 0;
      work(s, fl, by);
      record(h, sb, MFD_K_SOLVE_SMALL, fl, by,
             [&] { launch_bwd_small<T>(F, lists + s.off, s.count, s.param, panel, X, ldx, nrhs, sb); });
      ++n;
    }
    if (L.large.count) {
      double fl = 0, by = 0;
      work(L.large, fl, by);
      record(h, st, MFD_K_SOLVE_LARGE, fl, by, [&] {
        launch_bwd_large<T>(F, lists + L.large.off, L.large.count, L.large.param2, L.large_max_nf, panel, dinv, X,
                            ldx, V, S, h->d_cnt.p, nrhs, st, &n, solve_pdl, fused);
        if (fused) {
          const size_t lv = &L - h->levels.data();
          launch_large_fused<T>(F, stasks + L.bwd_tasks.off, L.bwd_tasks.count, true, ssync + 2 + 2 * lv, bwd_flags,
                                ssync, panel, dinv, X, V, st, h->d_info.p + 2, static_cast<T*>(h->d_bwpart),
                                bwd_flags + h->solve_flags);
          ++n;
        }
      });
    }
    if (nside) side_join(h, st, nside);
  }
  return n;
}

template <typename Fn>
int run_graph(mfd_handle* h, cudaGraphExec_t* exec, Fn&& fn) {
  if (!h->opt.use_graph || h->profiling) {
    fn(h->st);
    CK(cudaGetLastError());
    return MFD_OK;
  }
  if (!*exec) {
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    fn(h->st);
    cudaError_t e = cudaStreamEndCapture(h->st, &g);
    if (e != cudaSuccess) return fail(MFD_E_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    // per-node priorities (captured from the streams): the panel chain of the
    // lookahead outranks the side-stream trailing updates
    e = cudaGraphInstantiateWithFlags(exec, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(MFD_E_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
  }
  CK(cudaGraphLaunch(*exec, h->st));
  return MFD_OK;
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

int do_factorize(mfd_handle* h, const double* a) {
  if (!a) return fail(MFD_E_ARG, "null values");
  CK(cudaSetDevice(h->device));
  cudaMemcpyKind kind = is_device_ptr(a) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync(h->d_a.p, a, sizeof(double) * h->a_len, kind, h->st));
  launch_fill_int(h->d_info.p + 2, h->expire_waits ? 1 : 0, 1, h->st);
  CK(cudaEventRecord(h->ev0, h->st));
  int rc = h->fp32 ? run_graph(h, &h->g_factor, [&](cudaStream_t s) { h->launches_factor = enqueue_factor<float>(h, s); })
                   : run_graph(h, &h->g_factor, [&](cudaStream_t s) { h->launches_factor = enqueue_factor<double>(h, s); });
  if (rc) return rc;
  CK(cudaEventRecord(h->ev1, h->st));
  int32_t infos[4] = {0, 0, 0, 0};
  double anorm = 0;
  CK(cudaMemcpyAsync(infos, h->d_info.p, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(&anorm, h->d_norms.p + 7, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  float ms = 0;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  collect_profile(h);
  h->factor_ms = ms;
  h->anorm = anorm;
  h->pivot_fallbacks = infos[3];
  h->time_info[6] = ms * 1e-3;
  h->factored = true;
  const int32_t info = infos[0];
  if (infos[1] != 0) {
    h->factored = false;
    return fail(MFD_E_TIMEOUT, "a bounded wait in the tensor-core update expired");
  }
  if (info != INT_MAX) {
    // map the global permuted column to the system-relative 1-based column
    int64_t col = info - 1;
    int s = (int)(std::upper_bound(h->col_base.begin(), h->col_base.end(), col) - h->col_base.begin()) - 1;
    h->factored = false;
    g_err = "matrix is not positive definite (system " + std::to_string(s) + ")";
    return (int)(col - h->col_base[s] + 1);
  }
  return MFD_OK;
}

template <typename T>
int solve_core(mfd_handle* h, int nrhs) {
  auto it = h->g_solve.find(nrhs);
  cudaGraphExec_t exec = it == h->g_solve.end() ? nullptr : it->second;
  int rc = run_graph(h, &exec, [&](cudaStream_t s) { h->launches_solve = enqueue_solve_core<T>(h, nrhs, s); });
  if (exec) h->g_solve[nrhs] = exec;
  return rc;
}

int residual_report(mfd_handle* h, const double* xp, const double* bp, mfd_report* rep, double* bwd) {
  launch_residual(h->d_csr_ptr.p, h->d_csr_col.p, h->d_csr_val.p, xp, bp, h->d_r.p, h->n_total, h->st);
  launch_norms(h->d_r.p, xp, bp, h->n_total, h->d_norms.p, h->st);
  double nv[5];
  CK(cudaMemcpyAsync(nv, h->d_norms.p, 5 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  double denom = h->anorm * nv[1] + nv[2];
  *bwd = denom > 0 ? nv[0] / denom : nv[0];
  if (rep) {
    rep->backward_error = *bwd;
    rep->residual_ref = nv[4] > 0 ? std::sqrt(nv[3]) / std::sqrt(nv[4]) : std::sqrt(nv[3]);
  }
  return MFD_OK;
}

// One refinement sweep on `st`: x_32 = r in FP32, the FP32 solve, x += x_32
// in FP64, r = b - A x and the per-column norms (launch_norms layout) in FP64.
// graph_solve: the FP32 solve as its cached graph (host-driven loop), else its
// launches directly (inside the refinement graph's body).
int ir_sweep(mfd_handle* h, int nrhs, cudaStream_t st, bool graph_solve) {
  const int64_t n = h->n_total;
  launch_to_t<float>(h->d_r.p, static_cast<float*>(h->d_X), n * nrhs, st);
  if (graph_solve) {
    int rc = solve_core<float>(h, nrhs);
    if (rc) return rc;
  } else {
    h->launches_solve = enqueue_solve_core<float>(h, nrhs, st);
  }
  launch_axpy_from_t<float>(static_cast<float*>(h->d_X), h->d_xp.p, n * nrhs, st);
  if (nrhs >= kResMulti) {               // A read once for all columns
    launch_residual_multi(h->d_csr_ptr.p, h->d_csr_col.p, h->d_csr_val.p, h->d_xp.p, h->d_xt.p, h->d_bp.p,
                          h->d_r.p, n, nrhs, h->d_cnorms.p, st);
  } else {
    for (int r = 0; r < nrhs; ++r) {
      const int64_t o = (int64_t)r * n;
      launch_residual(h->d_csr_ptr.p, h->d_csr_col.p, h->d_csr_val.p, h->d_xp.p + o, h->d_bp.p + o, h->d_r.p + o, n,
                      st);
      launch_norms(h->d_r.p + o, h->d_xp.p + o, h->d_bp.p + o, n, h->d_cnorms.p + 8 * r, st);
    }
  }
  CK(cudaGetLastError());
  return MFD_OK;
}

// The whole refinement of one solve as a graph (built once per RHS count):
// permutation, x = 0, r = b, state reset; a WHILE node around the sweep, whose
// body ends with the device convergence test setting the node's condition;
// the inverse permutation.  Launched on h->st.
int ir_graph(mfd_handle* h, int nrhs) {
  cudaGraphExec_t& exec = h->g_ir[nrhs];
  if (!exec) {
    const int64_t n = h->n_total;
    const int maxit = h->opt.ir_max_iter > 0 ? h->opt.ir_max_iter : 20;
    cudaStream_t st = h->st;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    launch_permute_in<double>(h->d_b.p, n, h->d_perm.p, h->d_bp.p, n, n, nrhs, st);
    cudaMemsetAsync(h->d_xp.p, 0, sizeof(double) * n * nrhs, st);
    cudaMemcpyAsync(h->d_r.p, h->d_bp.p, sizeof(double) * n * nrhs, cudaMemcpyDeviceToDevice, st);
    launch_ir_init(h->d_ir_i.p, h->d_ir_d.p, h->d_ir_prev.p, nrhs, st);
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps);
    cudaGraphConditionalHandle cond = 0;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode = nullptr;
    if (e == cudaSuccess) e = cudaGraphAddNode(&wnode, g, deps, ndeps, &cp);
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(st, &wnode, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(h->bst, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        int rc = ir_sweep(h, nrhs, h->bst, /*graph_solve=*/false);
        launch_ir_check(h->d_cnorms.p, h->d_norms.p + 7, nrhs, h->opt.ir_tol, maxit, h->d_ir_prev.p, h->d_ir_i.p,
                        h->d_ir_d.p, cond, h->bst);
        cudaGraph_t got = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(h->bst, &got);
        if (rc != MFD_OK) e = cudaErrorUnknown;
        else if (e2 != cudaSuccess) e = e2;
      }
    }
    launch_permute_out<double>(h->d_xp.p, n, h->d_perm.p, h->d_b.p, n, n, nrhs, st);
    cudaGraph_t outer = nullptr;
    cudaError_t e3 = cudaStreamEndCapture(st, &outer);
    if (e == cudaSuccess) e = e3;
    if (e == cudaSuccess) e = cudaGraphInstantiateWithFlags(&exec, outer, cudaGraphInstantiateFlagUseNodePriority);
    if (outer) cudaGraphDestroy(outer);
    if (e != cudaSuccess) {
      exec = nullptr;
      h->g_ir.erase(nrhs);
      return fail(MFD_E_CUDA, std::string("refinement graph: ") + cudaGetErrorString(e));
    }
  }
  CK(cudaGraphLaunch(exec, h->st));
  return MFD_OK;
}

int do_solve(mfd_handle* h, double* b, int nrhs, int64_t ldb, mfd_report* rep) {
  if (!h->factored) return fail(MFD_E_STATE, "solve before a successful factorize");
  if (!b || nrhs < 1 || ldb < h->n_total) return fail(MFD_E_ARG, "bad right-hand side");
  CK(cudaSetDevice(h->device));
  int rc = ensure_rhs(h, nrhs);
  if (rc) return rc;
  const bool dev = is_device_ptr(b);
  const int64_t n = h->n_total;
  cudaStream_t st = h->st;
  if (ldb == n) {
    CK(cudaMemcpyAsync(h->d_b.p, b, sizeof(double) * n * nrhs, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  } else {
    CK(cudaMemcpy2DAsync(h->d_b.p, sizeof(double) * n, b, sizeof(double) * ldb, sizeof(double) * n, nrhs,
                         dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  }
  launch_fill_int(h->d_info.p + 2, h->expire_waits ? 1 : 0, 1, st);   // test request (mfd_test_expire_waits)
  CK(cudaEventRecord(h->ev0, st));
  int iters = 0;
  double bwd = 0;
  bool want_report = rep != nullptr || h->fp32;
  if (!h->fp32) {
    launch_permute_in<double>(h->d_b.p, n, h->d_perm.p, static_cast<double*>(h->d_X), n, n, nrhs, st);
    rc = solve_core<double>(h, nrhs);
    if (rc) return rc;
    CK(cudaEventRecord(h->ev1, st));
    if (want_report) {
      launch_permute_in<double>(h->d_b.p, n, h->d_perm.p, h->d_bp.p, n, n, 1, st);
      rc = residual_report(h, static_cast<double*>(h->d_X), h->d_bp.p, rep, &bwd);
      if (rc) return rc;
    }
    launch_permute_out<double>(static_cast<double*>(h->d_X), n, h->d_perm.p, h->d_b.p, n, n, nrhs, st);
  } else if (h->opt.use_graph && !h->profiling) {
    // FP32 factor + FP64 iterative refinement as one graph per right-hand-side
    // count: the sweeps run in a WHILE node whose last kernel applies the
    // convergence test on the device, so the host waits once per solve
    rc = ir_graph(h, nrhs);
    if (rc) return rc;
    int32_t si[2];
    double sd[2];
    CK(cudaMemcpyAsync(si, h->d_ir_i.p, sizeof(si), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(sd, h->d_ir_d.p, sizeof(sd), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(h->ev1, st));
    CK(cudaStreamSynchronize(st));
    iters = si[0];
    bwd = sd[0];
    if (rep) {
      rep->backward_error = bwd;
      rep->residual_ref = sd[1];
    }
    if (!(bwd <= h->opt.ir_tol)) rc = MFD_E_NOCONV;
  } else {
    // FP32 factor + FP64 iterative refinement, all right-hand sides together,
    // the convergence test on the host after every sweep (schedule without
    // graphs, and the per-kernel profiling runs)
    launch_permute_in<double>(h->d_b.p, n, h->d_perm.p, h->d_bp.p, n, n, nrhs, st);
    CK(cudaMemsetAsync(h->d_xp.p, 0, sizeof(double) * n * nrhs, st));
    CK(cudaMemcpyAsync(h->d_r.p, h->d_bp.p, sizeof(double) * n * nrhs, cudaMemcpyDeviceToDevice, st));
    const int maxit = h->opt.ir_max_iter > 0 ? h->opt.ir_max_iter : 20;
    std::vector<double> prev(nrhs, 1e300), cur(nrhs, 1e300), nv((size_t)8 * nrhs);
    double worst_ref = 0;
    int it = 0;
    for (; it < maxit; ++it) {
      rc = ir_sweep(h, nrhs, st, /*graph_solve=*/true);
      if (rc) return rc;
      CK(cudaMemcpyAsync(nv.data(), h->d_cnorms.p, sizeof(double) * 8 * nrhs, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      bool all_ok = true, all_stalled = it > 2;
      bwd = 0;
      for (int r = 0; r < nrhs; ++r) {
        const double* c = nv.data() + 8 * r;
        const double denom = h->anorm * c[1] + c[2];
        cur[r] = denom > 0 ? c[0] / denom : c[0];
        if (cur[r] > h->opt.ir_tol) {
          all_ok = false;
          if (cur[r] <= 0.9 * prev[r]) all_stalled = false;
        }
        if (cur[r] >= bwd) {
          bwd = cur[r];
          worst_ref = c[4] > 0 ? std::sqrt(c[3]) / std::sqrt(c[4]) : std::sqrt(c[3]);
        }
        prev[r] = cur[r];
      }
      if (all_ok || all_stalled) { ++it; break; }
    }
    iters = it;
    const bool converged = bwd <= h->opt.ir_tol;
    if (rep) {
      rep->backward_error = bwd;
      rep->residual_ref = worst_ref;
    }
    launch_permute_out<double>(h->d_xp.p, n, h->d_perm.p, h->d_b.p, n, n, nrhs, st);
    CK(cudaEventRecord(h->ev1, st));
    if (!converged) rc = MFD_E_NOCONV;
  }
  if (ldb == n) {
    CK(cudaMemcpyAsync(b, h->d_b.p, sizeof(double) * n * nrhs, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  } else {
    CK(cudaMemcpy2DAsync(b, sizeof(double) * ldb, h->d_b.p, sizeof(double) * n, sizeof(double) * n, nrhs,
                         dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  }
  int32_t expired = 0;                      // a bounded wait of the single-RHS large-front sweeps gave up
  if (nrhs == 1 && !h->h_stasks.empty()) CK(cudaMemcpyAsync(&expired, h->d_ssync.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (expired) return fail(MFD_E_TIMEOUT, "a device wait of the solve timed out");
  float ms = 0;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  collect_profile(h);
  h->solve_ms = ms;
  h->time_info[3] = ms * 1e-3;
  if (rep) {
    rep->iterations = iters;
    rep->converged = bwd <= h->opt.ir_tol;
    rep->time_ms = ms;
  }
  if (rc == MFD_E_NOCONV) g_err = "iterative refinement did not reach the tolerance";
  return rc;
}

int create_common(mfd_handle** out, std::vector<Symbolic>&& syms, const mfd_options* opt) {
  if (!out) return fail(MFD_E_ARG, "null handle pointer");
  std::unique_ptr<mfd_handle> h(new mfd_handle());
  mfd_default_options(&h->opt);
  if (opt) h->opt = *opt;
  if (h->opt.nb <= 0) h->opt.nb = 10;
  if (h->opt.ir_tol <= 0) h->opt.ir_tol = 1e-12;
  h->fp32 = h->opt.precision == MFD_PREC_FP32_IR;
  h->device = h->opt.device;
  h->sys = std::move(syms);
  CK(cudaSetDevice(h->device));
  CK(prepare_kernels());
  int prio_lo = 0, prio_hi = 0;
  CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  CK(cudaStreamCreateWithPriority(&h->st, cudaStreamNonBlocking, prio_hi));
  CK(cudaStreamCreateWithPriority(&h->st2, cudaStreamNonBlocking, prio_lo));
  CK(cudaStreamCreateWithPriority(&h->bst, cudaStreamNonBlocking, prio_hi));
  CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
  for (int k = 0; k < mfd_handle::kMaxDefer; ++k) CK(cudaEventCreateWithFlags(&h->ev_part[k], cudaEventDisableTiming));
  // deferred updates: reserved[5] = group size (1 = none); 0 = default
  h->defer = h->opt.reserved[5] > 0 ? std::min(h->opt.reserved[5], mfd_handle::kMaxDefer)
                                     : (h->opt.precision == MFD_PREC_FP32_IR ? kDeferDefaultFp32 : kDeferDefaultFp64);
  CK(cudaEventCreateWithFlags(&h->ev_lvl, cudaEventDisableTiming));
  for (int b = 0; b < mfd_handle::kSide; ++b) {
    CK(cudaStreamCreateWithPriority(&h->sst[b], cudaStreamNonBlocking, prio_lo));
    CK(cudaEventCreateWithFlags(&h->ev_side[b], cudaEventDisableTiming));
  }
  CK(cudaEventCreate(&h->ev0));
  CK(cudaEventCreate(&h->ev1));
  auto t0 = std::chrono::steady_clock::now();
  int rc = build_plan(h.get());
  if (rc) return rc;
  h->setup_s[1] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  rc = upload_plan(h.get());
  if (rc) return rc;
  *out = h.release();
  return MFD_OK;
}

int check_symbolic(const mfd_symbolic& s) {
  if (s.n <= 0 || s.num_node <= 0 || s.nnz <= 0) return -1;
  if (!s.node_ptr || !s.parent || !s.lrow_ptr || !s.acol_ptr || !s.arow || !s.ccs_perm || !s.perm) return -1;
  if (s.node_ptr[0] != 1 || s.node_ptr[s.num_node] != s.n + 1) return -1;
  if (s.lrow_ptr[0] != 1 || s.acol_ptr[0] != 1 || s.acol_ptr[s.n] != s.nnz + 1) return -1;
  for (int i = 0; i < s.num_node; ++i) {
    if (s.node_ptr[i + 1] <= s.node_ptr[i] || s.lrow_ptr[i + 1] < s.lrow_ptr[i]) return -1;
    if (s.parent[i] < 0 || s.parent[i] > s.num_node || (s.parent[i] != 0 && s.parent[i] <= i + 1)) return -1;
    int last = s.node_ptr[i + 1] - 1;
    for (int k = s.lrow_ptr[i] - 1; k < s.lrow_ptr[i + 1] - 1; ++k) {
      if (s.lrow[k] <= last || s.lrow[k] > s.n) return -1;
      if (k > s.lrow_ptr[i] - 1 && s.lrow[k] <= s.lrow[k - 1]) return -1;
    }
  }
  for (int j = 0; j < s.n; ++j)
    for (int k = s.acol_ptr[j] - 1; k < s.acol_ptr[j + 1] - 1; ++k) {
      if (s.arow[k] < j + 1 || s.arow[k] > s.n) return -1;
      if (s.ccs_perm[k] < 1 || s.ccs_perm[k] > s.nnz) return -1;
    }
  for (int i = 0; i < s.n; ++i)
    if (s.perm[i] < 1 || s.perm[i] > s.n) return -1;
  return 0;
}

Symbolic copy_symbolic(const mfd_symbolic& s) {
  Symbolic o;
  o.n = s.n; o.nnz = s.nnz; o.num_node = s.num_node;
  o.node_ptr.assign(s.node_ptr, s.node_ptr + s.num_node + 1);
  o.parent.assign(s.parent, s.parent + s.num_node);
  o.lrow_ptr.assign(s.lrow_ptr, s.lrow_ptr + s.num_node + 1);
  o.lrow.assign(s.lrow, s.lrow + (s.lrow_ptr[s.num_node] - 1));
  o.acol_ptr.assign(s.acol_ptr, s.acol_ptr + s.n + 1);
  o.arow.assign(s.arow, s.arow + s.nnz);
  o.ccs_perm.assign(s.ccs_perm, s.ccs_perm + s.nnz);
  o.perm.assign(s.perm, s.perm + s.n);
  return o;
}

}  // namespace

namespace mfd {
// CSR input (input.cu): the caller's values come in another order; entry k of
// the analysed lower CCS is entry d_map[k] of the caller's array (a_len long).
// Every value source of the handle (assembly, residual matrix) is re-pointed.
int handle_set_value_map(mfd_handle* h, const int32_t* d_map, int64_t a_len) {
  if (!h || h->sys.size() != 1) return fail(MFD_E_ARG, "value map: single-system handles only");
  CK(cudaSetDevice(h->device));
  launch_remap_int(d_map, h->d_a_src.p, h->nnz_total, h->st);
  launch_remap_int(d_map, h->d_csr_src.p, (int64_t)h->d_csr_src.n, h->st);
  h->a_len = a_len;
  CK(h->d_a.alloc(a_len));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  for (auto& kv : h->g_solve) cudaGraphExecDestroy(kv.second);
  h->g_solve.clear();
  if (h->g_factor) cudaGraphExecDestroy(h->g_factor);
  h->g_factor = nullptr;
  return MFD_OK;
}
}  // namespace mfd

// ==================================================================================
// C ABI
// ==================================================================================
extern "C" {

#pragma GCC visibility push(default)

void mfd_default_options(mfd_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->nb = 10;
  opt->max_zero = 10;
  opt->precision = MFD_PREC_FP64;
  opt->ir_max_iter = 20;
  opt->ir_tol = 1e-12;
  opt->use_graph = 1;
  opt->device = 0;
}

const char* mfd_last_error(void) { return g_err.c_str(); }

int mfd_create(mfd_handle** h, const mfd_symbolic* sym, const mfd_options* opt) {
  if (!sym || check_symbolic(*sym)) return fail(MFD_E_ARG, "malformed symbolic input");
  std::vector<Symbolic> v;
  v.push_back(copy_symbolic(*sym));
  return create_common(h, std::move(v), opt);
}

int mfd_create_batch(mfd_handle** h, int32_t num_systems, const mfd_symbolic* syms, const mfd_options* opt) {
  if (num_systems <= 0 || !syms) return fail(MFD_E_ARG, "empty batch");
  std::vector<Symbolic> v;
  v.reserve(num_systems);
  for (int i = 0; i < num_systems; ++i) {
    if (check_symbolic(syms[i])) return fail(MFD_E_ARG, "malformed symbolic input in system " + std::to_string(i));
    v.push_back(copy_symbolic(syms[i]));
  }
  return create_common(h, std::move(v), opt);
}

int mfd_analyze(mfd_handle** h, int32_t n, const int32_t* ccs_col, const int32_t* ccs_row, const int32_t* order_perm,
                const mfd_options* opt) {
  mfd_options o;
  mfd_default_options(&o);
  if (opt) o = *opt;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<Symbolic> v(1);
  if (analyze(n, ccs_col, ccs_row, order_perm, o.max_zero, v[0])) return fail(MFD_E_ARG, "malformed matrix or ordering");
  double ta = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  int rc = create_common(h, std::move(v), &o);
  if (rc == MFD_OK) (*h)->time_info[1] = (*h)->setup_s[0] = ta;
  return rc;
}

struct mfd_analysis {
  Symbolic s;
};

int mfd_symbolic_analyze(mfd_analysis** out, int32_t n, const int32_t* ccs_col, const int32_t* ccs_row,
                         const int32_t* order_perm, int32_t max_zero) {
  if (!out) return fail(MFD_E_ARG, "null output");
  std::unique_ptr<mfd_analysis> a(new mfd_analysis());
  if (analyze(n, ccs_col, ccs_row, order_perm, max_zero, a->s)) return fail(MFD_E_ARG, "malformed matrix or ordering");
  *out = a.release();
  return MFD_OK;
}

int mfd_symbolic_view(const mfd_analysis* a, mfd_symbolic* v) {
  if (!a || !v) return fail(MFD_E_ARG, "null argument");
  const Symbolic& s = a->s;
  v->n = s.n; v->nnz = s.nnz; v->num_node = s.num_node;
  v->node_ptr = s.node_ptr.data(); v->parent = s.parent.data(); v->lrow_ptr = s.lrow_ptr.data();
  v->lrow = s.lrow.data(); v->acol_ptr = s.acol_ptr.data(); v->arow = s.arow.data();
  v->ccs_perm = s.ccs_perm.data(); v->perm = s.perm.data();
  return MFD_OK;
}

int mfd_symbolic_free(mfd_analysis* a) {
  delete a;
  return MFD_OK;
}

int mfd_analyze_batch(mfd_handle** h, int32_t num_systems, const int32_t* n, const int32_t* const* ccs_col,
                      const int32_t* const* ccs_row, const int32_t* const* order_perm, const mfd_options* opt) {
  if (num_systems <= 0) return fail(MFD_E_ARG, "empty batch");
  mfd_options o;
  mfd_default_options(&o);
  if (opt) o = *opt;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<Symbolic> v(num_systems);
  std::vector<int> rcs(num_systems, 0);
  unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&, t]() {
      for (int s = (int)t; s < num_systems; s += (int)nt)
        rcs[s] = analyze(n[s], ccs_col[s], ccs_row[s], order_perm ? order_perm[s] : nullptr, o.max_zero, v[s]);
    });
  for (auto& x : th) x.join();
  for (int s = 0; s < num_systems; ++s)
    if (rcs[s]) return fail(MFD_E_ARG, "malformed matrix or ordering in system " + std::to_string(s));
  double ta = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  int rc = create_common(h, std::move(v), &o);
  if (rc == MFD_OK) (*h)->time_info[1] = (*h)->setup_s[0] = ta;
  return rc;
}

int mfd_factorize(mfd_handle* h, const double* a) {
  if (!h) return fail(MFD_E_ARG, "null handle");
  return do_factorize(h, a);
}

int mfd_solve(mfd_handle* h, double* b, int32_t nrhs, int64_t ldb, mfd_report* rep) {
  if (!h) return fail(MFD_E_ARG, "null handle");
  return do_solve(h, b, nrhs, ldb, rep);
}

int mfd_autotune(mfd_handle* h, const double* a, int32_t repeats, mfd_options* best, double* best_ms) {
  if (!h || !a || !best || repeats < 1) return fail(MFD_E_ARG, "autotune: null handle, values or output");
  double best_t = 1e300;
  mfd_options best_o = h->opt;
  // one candidate: a temporary handle on h's symbolic data, one warm-up
  // factorization (graph capture), then the median of `repeats`
  auto trial = [&](const mfd_options& o, int* err) -> double {
    std::vector<Symbolic> syms = h->sys;
    mfd_handle* t = nullptr;
    if (create_common(&t, std::move(syms), &o) != MFD_OK) return 1e300;   // e.g. out of memory: skip it
    std::unique_ptr<mfd_handle> guard(t);
    int rc = do_factorize(t, a);
    if (rc != MFD_OK) { *err = rc; return 1e300; }
    std::vector<double> ms;
    for (int r = 0; r < repeats; ++r) {
      rc = do_factorize(t, a);
      if (rc != MFD_OK) { *err = rc; return 1e300; }
      ms.push_back(t->factor_ms);
    }
    std::sort(ms.begin(), ms.end());
    return ms[ms.size() / 2];
  };
  auto consider = [&](const mfd_options& o) -> int {
    int err = MFD_OK;
    const double t = trial(o, &err);
    if (err != MFD_OK) return err;
    if (t < best_t) {
      best_t = t;
      best_o = o;
    }
    return MFD_OK;
  };
  // stage 1: the schedule -- small-front / blocked split x lookahead
  const int sfms[] = {32, 64, 96, 128};   // small-front split (at most kSmallFrontMax)
  for (int sfm : sfms)
    for (int lookahead_off = 0; lookahead_off <= 1; ++lookahead_off) {
      mfd_options o = h->opt;
      o.small_front_max = sfm;
      o.reserved[1] = lookahead_off;
      int rc = consider(o);
      if (rc) return rc;
    }
  // stage 2, at the best schedule: the trailing-update kernel (FP64: DMMA in
  // 128 x 64 halves / whole 128 x 128 tiles / FFMA; FP32: 3xTF32 tcgen05 /
  // FFMA) and the deferral depth of the bulk update (1, 2 panel steps)
  const mfd_options base = best_o;
  const bool fp32 = base.precision == MFD_PREC_FP32_IR;
  const int kinds64[] = {0, 3, 1}, kinds32[] = {0, 1};
  const int* kinds = fp32 ? kinds32 : kinds64;
  const int nk = fp32 ? 2 : 3;
  for (int ki = 0; ki < nk; ++ki)
    for (int d = 1; d <= 2; ++d) {
      mfd_options o = base;
      o.reserved[0] = kinds[ki];
      o.reserved[5] = d;
      const int base_d = base.reserved[5] > 0 ? base.reserved[5] : (fp32 ? kDeferDefaultFp32 : kDeferDefaultFp64);
      if (kinds[ki] == base.reserved[0] && d == base_d) continue;   // timed in stage 1
      int rc = consider(o);
      if (rc) return rc;
    }
  *best = best_o;
  if (best_ms) *best_ms = best_t;
  return MFD_OK;
}

int mfd_factorize_solve(mfd_handle* h, const double* a, double* b, int32_t nrhs, int64_t ldb, mfd_report* rep) {
  int rc = mfd_factorize(h, a);
  if (rc) return rc;
  return mfd_solve(h, b, nrhs, ldb, rep);
}

int mfd_get_stats(mfd_handle* h, mfd_stats* st) {
  if (!h || !st) return fail(MFD_E_ARG, "null argument");
  std::memset(st, 0, sizeof(*st));
  st->n = h->n_total;
  st->nnz_a = h->nnz_total;
  st->num_front = h->num_front;
  st->num_level = (int64_t)h->levels.size();
  st->cost = h->cost;
  st->nonzero = h->nonzero;
  size_t esz = h->fp32 ? sizeof(float) : sizeof(double);
  st->panel_bytes = h->panel_elems * (int64_t)esz;
  st->update_pool_bytes = h->upool_elems * (int64_t)esz;
  st->launches_factor = h->launches_factor;
  st->launches_solve = h->launches_solve;
  st->max_front = h->max_nf;
  st->factor_ms = h->factor_ms;
  st->solve_ms = h->solve_ms;
  st->pivot_fallbacks = h->pivot_fallbacks;
  std::memcpy(st->time_info, h->time_info, sizeof(st->time_info));
  std::memcpy(st->setup_s, h->setup_s, sizeof(st->setup_s));
  return MFD_OK;
}

int64_t mfd_get_index(mfd_handle* h, int32_t system, int32_t which, int32_t* out) {
  if (!h || system < 0 || system >= (int32_t)h->sys.size()) return fail(MFD_E_ARG, "bad system");
  const std::vector<int32_t>* v = nullptr;
  switch (which) {
    case 1: v = &h->local_sys[system]; break;
    case 2: v = &h->sidx_sys[system]; break;
    case 3: v = &h->bli_node_ptr[system]; break;
    case 4: v = &h->bli_block_ptr[system]; break;
    case 5: v = &h->bli_pnum[system]; break;
    case 6: v = &h->bli_cnum[system]; break;
    case 7: v = &h->bli_val[system]; break;
    case 8: v = &h->bli_off[system]; break;
    default: return fail(MFD_E_ARG, "bad index id");
  }
  if (out && !v->empty()) std::memcpy(out, v->data(), v->size() * sizeof(int32_t));
  return (int64_t)v->size();
}

int64_t mfd_get_symbolic(mfd_handle* h, int32_t system, int32_t which, int32_t* out) {
  if (!h || system < 0 || system >= (int32_t)h->sys.size()) return fail(MFD_E_ARG, "bad system");
  const Symbolic& S = h->sys[system];
  const std::vector<int32_t>* v = nullptr;
  switch (which) {
    case 1: v = &S.node_ptr; break;
    case 2: v = &S.parent; break;
    case 3: v = &S.lrow_ptr; break;
    case 4: v = &S.lrow; break;
    case 5: v = &S.acol_ptr; break;
    case 6: v = &S.arow; break;
    case 7: v = &S.ccs_perm; break;
    case 8: v = &S.perm; break;
    default: return fail(MFD_E_ARG, "bad symbolic id");
  }
  if (out && !v->empty()) std::memcpy(out, v->data(), v->size() * sizeof(int32_t));
  return (int64_t)v->size();
}

int64_t mfd_get_front_panel(mfd_handle* h, int32_t system, int32_t node, double* out) {
  if (!h || system < 0 || system >= (int32_t)h->sys.size()) return fail(MFD_E_ARG, "bad system");
  if (node < 1 || node > h->sys[system].num_node) return fail(MFD_E_ARG, "bad node");
  const HostFront& f = h->fronts[h->front_base[system] + node - 1];
  int64_t cnt = (int64_t)(f.nc + f.nr) * f.nc;
  if (!out) return cnt;
  if (!h->factored) return fail(MFD_E_STATE, "not factorized");
  CK(cudaSetDevice(h->device));
  if (h->fp32) {
    std::vector<float> tmp(cnt);
    CK(cudaMemcpy(tmp.data(), static_cast<float*>(h->d_panel) + f.panel_off, cnt * sizeof(float), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < cnt; ++i) out[i] = tmp[i];
  } else {
    CK(cudaMemcpy(out, static_cast<double*>(h->d_panel) + f.panel_off, cnt * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return cnt;
}

int mfd_set_profiling(mfd_handle* h, int32_t enable) {
  if (!h) return fail(MFD_E_ARG, "null handle");
  h->profiling = enable != 0;
  std::memset(h->prof, 0, sizeof(h->prof));
  h->pending.clear();
  return MFD_OK;
}

int mfd_test_expire_waits(mfd_handle* h, int32_t enable) {
  if (!h) return fail(MFD_E_ARG, "null handle");
  h->expire_waits = enable != 0;
  return MFD_OK;
}

int mfd_get_profile(mfd_handle* h, int32_t kind, mfd_kernel_profile* out) {
  if (!h || !out || kind < 0 || kind >= MFD_K_COUNT) return fail(MFD_E_ARG, "bad argument");
  *out = h->prof[kind];
  return MFD_OK;
}

int mfd_destroy(mfd_handle* h) {
  delete h;
  return MFD_OK;
}

// ---- reference-named entry points: one module-global instance (hppllt_data_m.f90) ----
static struct {
  std::vector<int32_t> options;
  std::vector<int32_t> order;
  int32_t precision = MFD_PREC_FP64;
  mfd_handle* h = nullptr;
  double times[7] = {0, 0, 0, 0, 0, 0, 0};
} g_ref;

int hppllt_init(const int32_t* options, int32_t noptions) {
  if (noptions != 4 || !options) {
    std::fprintf(stderr, "incorrect size of options\n");
    return -1;
  }
  g_ref.options.assign(options, options + 4);
  return 0;
}

int hppllt_set_precision(int32_t precision) {
  g_ref.precision = precision;
  return 0;
}

int hppllt_set_ordering(const int32_t* order_perm, int32_t n) {
  if (!order_perm || n <= 0) { g_ref.order.clear(); return 0; }
  g_ref.order.assign(order_perm, order_perm + n);
  return 0;
}

int hppllt_analyze(const int32_t* ccs_col, const int32_t* ccs_row, int32_t n) {
  if (g_ref.options.size() != 4) return fail(MFD_E_STATE, "hppllt_init not called");
  if (g_ref.h) { mfd_destroy(g_ref.h); g_ref.h = nullptr; }
  mfd_options o;
  mfd_default_options(&o);
  o.nb = g_ref.options[0];
  o.max_zero = g_ref.options[1];
  o.precision = g_ref.precision;
  const int32_t* ord = nullptr;
  std::vector<int32_t> nd;
  auto t0 = std::chrono::steady_clock::now();
  if (g_ref.options[3] == 1) {
    // use_metis = 1 (hppllt.f90:47-51): a caller-supplied ordering, else the
    // library's nested dissection where the reference calls METIS_NodeND
    if ((int32_t)g_ref.order.size() == n) {
      ord = g_ref.order.data();
    } else {
      nd.resize(n > 0 ? n : 1);
      if (n < 1 || nested_dissection(n, ccs_col, ccs_row, nd.data())) return fail(MFD_E_ARG, "bad matrix for ordering");
      ord = nd.data();
    }
  }
  g_ref.times[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  t0 = std::chrono::steady_clock::now();
  int rc = mfd_analyze(&g_ref.h, n, ccs_col, ccs_row, ord, &o);
  g_ref.times[1] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return rc;
}

int mfd_subtree_partition(int32_t num_node, const int32_t* node_size, const int32_t* cc, const int32_t* num_child,
                          const int32_t* child, double tol, int32_t p, int32_t* roots, int32_t* count) {
  if (!node_size || !cc || !num_child || (!child && num_node > 1) || !roots || !count)
    return fail(MFD_E_ARG, "mfd_subtree_partition: null argument");
  std::vector<int32_t> r = subtree_partition(num_node, node_size, cc, num_child, child, tol, p);
  if (r.empty()) return fail(MFD_E_ARG, "mfd_subtree_partition: bad tree or p < 1");
  std::memcpy(roots, r.data(), sizeof(int32_t) * r.size());
  *count = (int32_t)r.size();
  return MFD_OK;
}

int mfd_order(int32_t n, const int32_t* ccs_col, const int32_t* ccs_row, int32_t* order_perm) {
  if (nested_dissection(n, ccs_col, ccs_row, order_perm)) return fail(MFD_E_ARG, "mfd_order: bad matrix");
  return MFD_OK;
}

int hppllt_factorize(const double* a) {
  if (!g_ref.h) return fail(MFD_E_STATE, "hppllt_analyze not called");
  auto t0 = std::chrono::steady_clock::now();
  int rc = mfd_factorize(g_ref.h, a);
  g_ref.times[2] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  g_ref.times[6] = g_ref.h->factor_ms * 1e-3;
  return rc;
}

int hppllt_solve(double* b) {
  if (!g_ref.h) return fail(MFD_E_STATE, "hppllt_analyze not called");
  auto t0 = std::chrono::steady_clock::now();
  int rc = mfd_solve(g_ref.h, b, 1, g_ref.h->n_total, nullptr);
  g_ref.times[3] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return rc;
}

int hppllt_finalize(void) {
  g_ref.options.clear();
  if (g_ref.h) { mfd_destroy(g_ref.h); g_ref.h = nullptr; }
  return 0;
}

double hppllt_get_time_info(int32_t num) {
  if (num < 1 || num > 7) return 0.0;
  return g_ref.times[num - 1];
}

int64_t hppllt_get_cost(void) { return g_ref.h ? g_ref.h->cost : 0; }
int64_t hppllt_get_nonzero(void) { return g_ref.h ? g_ref.h->nonzero : 0; }

int64_t hppllt_get_array_size(int32_t num) {
  // sizes of the reference's three FP64 buffers for the same partition and nb
  // (supernode_matrix_extractor_m.f90:41-54, work_matrix_extractor_m.f90:51-74,
  // border_matrix_extractor_m.f90:28-47)
  if (!g_ref.h || num < 1 || num > 3) return 0;
  const Symbolic& S = g_ref.h->sys[0];
  const int64_t nb = g_ref.h->opt.nb;
  auto ps = [](int64_t e) { return e < 1 ? (int64_t)0 : e * (e + 1) / 2; };
  auto ps2 = [&](int64_t s, int64_t e) { return e < s ? (int64_t)0 : ps(e) - ps(s - 1); };
  auto bsz = [&](int64_t idx, int64_t n) { return idx * nb > n ? n % nb : nb; };
  int64_t total = 0;
  for (int i = 0; i < S.num_node; ++i) {
    int64_t nc = S.node_ptr[i + 1] - S.node_ptr[i], nr = S.lrow_ptr[i + 1] - S.lrow_ptr[i], n = nc + nr;
    int64_t ss = nc % nb, ws = std::min(nb - ss, nr);
    int64_t wstart = nr == 0 ? (nc - 1) / nb + 2 : nc / nb + 1;
    int64_t nblk = (n - 1) / nb + 1;
    if (num == 1) {
      total += ps2(nr + 1, nc + nr) + ps(nb - 1) * (nc / nb) + ps(ss - 1);
    } else if (num == 2) {
      int64_t wn = nblk - wstart + 1 - 2;
      total += nr * ws + ps(wn) * nb * nb + (nr - ws) * bsz(nblk, n);
    } else {
      if (ss != 0 && nr != 0) total += (n - (nc / nb) * nb) * bsz(wstart, n);
    }
  }
  return total;
}

#pragma GCC visibility pop

}  // extern "C"
