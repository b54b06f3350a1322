// Device-side description of an analysed system (or batch of systems) and the
// host launch plan built from it.
//
// Layout in HBM (one handle):
//   panel pool  : for every front f, its factor columns as an nf x nc
//                 column-major block (ld = nf) -- resident for the solves
//   update pool : for every front f, its nr x nr update matrix (ld = nr); the
//                 offsets come from a static lifetime plan over the level
//                 schedule, so storage is reused once the parent has consumed it
//   vector pool : nf entries per front per right-hand side (solve work vectors)
// Front positions 0..nc-1 are the supernode's columns, nc..nf-1 its L rows.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace mfd {

// Pointers into the device copies of the per-front tables (all 0-based).
struct DevFronts {
  const int32_t* nc;          // supernode columns
  const int32_t* nr;          // update rows
  const int32_t* first;       // first permuted (global) column
  const int32_t* parent;      // parent front, -1 for a root
  const int32_t* child_ptr;   // children of f: child[child_ptr[f] .. child_ptr[f+1])
  const int32_t* child;       // ascending (the reference's tree_child order)
  const int64_t* panel_off;   // element offset of the panel in the panel pool
  const int64_t* u_off;       // element offset of the update matrix in the update pool
  const int32_t* lrow_off;    // offset of f's L rows in lrow / local
  const int32_t* lrow;        // L rows, global permuted 0-based
  const int32_t* local;       // reference local_index values (1-based positions in the parent front)
  const int32_t* a_beg;       // entries of A assembled into f: [a_beg[f], a_beg[f+1])
  const int32_t* a_src;       // per A entry: index into the caller's value array
  const int32_t* a_pos;       // per A entry: row + col*nf inside the front
  const int64_t* v_off;       // offset of f's solve vector (units of one RHS)
  const int64_t* s_off;       // scratch offset (large-front solve partial sums)
  const int64_t* d_off;       // offset of f's inverted 128 x 128 diagonal blocks (one per panel step);
                              // null: the inverse of list slot i lives at linv + i * 128 * 128
  const int64_t* q_off;       // FP32: offset of f's packed update operands (null when unused)
};

struct HostFront {
  int32_t nc, nr, first, parent, level, sys, node;
  int64_t panel_off, u_off, v_off, s_off, d_off, q_off;
};

struct LaunchList {          // a list of front ids in the device list pool
  int32_t off = 0, count = 0;
  int32_t param = 0;         // kernel-specific (size bin, grid extent, step, ...)
  int32_t param2 = 0;
  int32_t param3 = 0;
};

struct LevelPlan {
  std::vector<LaunchList> small;     // fused one-CTA fronts, one list per size bin
  LaunchList large;                  // blocked fronts (sorted by nc descending)
  std::vector<LaunchList> ext_add;   // per child rank: children of large fronts
  std::vector<LaunchList> steps;     // per panel step: prefix of `large`; param = TRSM row blocks,
                                     // param2 = 128-tiles, param3 = 64-tiles of the trailing triangle
  std::vector<LaunchList> solve_steps;
  // per panel step: how many fronts of the step's list (in order) need 4, 3, 2, 1
  // sub-blocks of 32 columns in the diagonal-block POTRF
  std::vector<std::array<int32_t, 4>> potrf_cls;
  // single-RHS large-front solve in one launch per sweep: task lists (4 ints per task)
  // in the solve task pool, forward and backward
  LaunchList fwd_tasks, bwd_tasks;
  int32_t large_max_nf = 0;
  int64_t large_zero_elems = 0;
};

}  // namespace mfd
