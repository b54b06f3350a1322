// Host symbolic analysis of the supernodal multifrontal Cholesky solver.
//
// Restates the reference's hppllt_analyze (src/main/hppllt.f90:24-81) and
// analyze_phase (src/main/analyse_phase_m.f90:22-108): optional external
// ordering (the METIS branch), elimination tree, postorder, column counts,
// fundamental supernodes, relaxed-supernode amalgamation, supernodal L row
// structure, and the composed permutations.  The output arrays are exactly the
// reference's (1-based int32) so the index data built on the device from them
// is bit-exact with the reference's.
#pragma once
#include <cstdint>
#include <vector>

namespace mfd {

struct Symbolic {
  int32_t n = 0, nnz = 0, num_node = 0;
  std::vector<int32_t> node_ptr;   // num_node+1 (node_sets%ptr)
  std::vector<int32_t> parent;     // num_node (0 = root)
  std::vector<int32_t> lrow_ptr;   // num_node+1
  std::vector<int32_t> lrow;       // L row lists (ascending, permuted numbering)
  std::vector<int32_t> acol_ptr;   // n+1 (a_structure)
  std::vector<int32_t> arow;       // nnz
  std::vector<int32_t> ccs_perm;   // nnz
  std::vector<int32_t> perm;       // n
};

// Returns 0 on success, -1 on malformed input (non-lower entry, missing
// diagonal-first column, disconnected elimination tree, bad ordering).
int analyze(int32_t n, const int32_t* ccs_col, const int32_t* ccs_row, const int32_t* order_perm,
            int32_t max_zero, Symbolic& out);

// Nested-dissection ordering of the matrix graph (ordering.cpp): order_perm
// (n entries) receives new -> old, 1-based.  Returns 0, or -1 on bad input.
int nested_dissection(int32_t n, const int32_t* ccs_col, const int32_t* ccs_row, int32_t* order_perm);

// Subtree partition of the supernodal tree for p workers (partition.cpp, the
// reference's tree_pruning): subtree roots (1-based) in list order; empty on bad input.
std::vector<int32_t> subtree_partition(int32_t num_node, const int32_t* node_size, const int32_t* cc,
                                       const int32_t* num_child, const int32_t* child, double tol, int32_t p);

}  // namespace mfd
