"""Golden vectors transcribed from the reference's own Fortran unit tests.

Each constant cites the reference file (path within the project) and line range
it was transcribed from.  ``check_transcription.py`` in this directory re-reads
those files (when the reference tree is present) and confirms that every integer
list below appears verbatim at the cited location.

Conventions follow the reference: all indices are 1-based.
"""

# ---------------------------------------------------------------------------
# 9x9 symbolic fixture: src/test_mod/sparse_matrix_maker_m.f90, tree_maker_m.f90,
# perm_maker_m.f90
# ---------------------------------------------------------------------------
CCS9_NUM_ROW = [3, 4, 3, 2, 3, 2, 2, 1, 1]                      # sparse_matrix_maker_m.f90:25
CCS9_ROW = [1, 7, 8, 2, 4, 6, 9, 3, 5, 8, 4, 9, 5, 6, 8, 6, 9, 7, 9, 8, 9]  # :26
CRS9_NUM_COL = [1, 1, 1, 2, 2, 3, 2, 4, 5]                      # :45
CRS9_COL = [1, 2, 3, 2, 4, 3, 5, 2, 5, 6, 1, 7, 1, 3, 5, 8, 2, 4, 6, 7, 9]  # :46
POST9_NUM_ROW = [3, 2, 4, 2, 3, 3, 2, 1, 1]                     # :65
POST9_ROW = [1, 2, 8, 2, 9, 3, 4, 7, 9, 4, 9, 5, 6, 8, 6, 7, 8, 7, 9, 8, 9]  # :66
SN9_NUM_ROW = [2, 2, 2, 2, 2, 2, 0]                             # :84 (also the supernodal column counts)
SN9_ROW = [2, 8, 8, 9, 7, 9, 6, 8, 7, 8, 8, 9]                  # :88
SN9_NODE_SIZE = [1, 1, 2, 1, 1, 1, 2]                           # :92

ORIG_TREE_PARENT = [7, 4, 5, 6, 6, 8, 8, 9, 0]                  # tree_maker_m.f90:7
ORIG_TREE_NUM_CHILD = [0, 0, 0, 1, 1, 2, 1, 2, 1]               # :11
ORIG_TREE_CHILD_VAL = [2, 3, 4, 5, 1, 6, 7, 8]                  # :15
POST_TREE_PARENT = [2, 8, 4, 7, 6, 7, 8, 9, 0]                  # :23
POST_TREE_NUM_CHILD = [0, 1, 0, 1, 0, 1, 2, 2, 1]               # :27
POST_TREE_CHILD_VAL = [1, 3, 5, 4, 6, 2, 7, 8]                  # :31
SN_TREE_NUM_CHILD = [0, 1, 0, 0, 1, 2, 2]                       # :39
SN_TREE_CHILD_VAL = [1, 4, 3, 5, 2, 6]                          # :43

POST_PERM = [1, 7, 2, 4, 3, 5, 6, 8, 9]                         # perm_maker_m.f90:7
POST_IPERM = [1, 3, 5, 4, 6, 7, 2, 8, 9]                        # :11

# supernodal 7-node fixture of tree_pruning_test.f90: nr and node sizes
SN_CC = [2, 2, 2, 2, 2, 2, 0]                                    # src/test_mod/sparse_matrix_maker_m.f90:88
SN_NODE_SIZE = [1, 1, 2, 1, 1, 1, 2]                             # src/test_mod/sparse_matrix_maker_m.f90:96

# ---------------------------------------------------------------------------
# algorithm tests
# ---------------------------------------------------------------------------
# tree_pruning_test.f90:23-33: (tol, p) -> subtree roots in list order
TREE_PRUNING_P1 = [7]                                            # src/test/algorithms/tree_pruning_test.f90:24
TREE_PRUNING_P2 = [6, 2]                                         # src/test/algorithms/tree_pruning_test.f90:27
TREE_PRUNING_TOL071 = [5, 3, 2]                                  # src/test/algorithms/tree_pruning_test.f90:30
TREE_PRUNING_TOL073 = [5, 3, 2]                                  # src/test/algorithms/tree_pruning_test.f90:33
TREE_PRUNING_CASES = [(0.0, 1, TREE_PRUNING_P1), (0.0, 2, TREE_PRUNING_P2), (0.71, 2, TREE_PRUNING_TOL071),
                      (0.73, 2, TREE_PRUNING_TOL073)]
COLUMN_COUNT = [3, 3, 4, 3, 3, 3, 3, 2, 1]                      # src/test/algorithms/column_count_test.f90:17
FINDING_LEAVES_SUBTREE = [1, 2, 1, 2, 1, 2, 5, 8, 9]            # finding_leaves_test.f90:13
FINDING_LEAVES = [1, 1, 1, 0, 1, 1, 0, 0, 0]                    # :15
TREE_SUBTREE_SIZE = [1, 1, 1, 2, 2, 5, 2, 8, 9]                 # src/test/data_structure_creators/tree_test.f90:21
TREE_POSTORDER = [2, 4, 3, 5, 6, 1, 7, 8, 9]                    # :24
FUND_FIRST_NODE = [1, 2, 3, 5, 6, 7, 8, 10]                     # fundamental_supernode_test.f90:24
FUND_SN_CCS_LEN = [2, 1, 2, 2, 2, 1, 0]                         # :30
FUND_SN_CCS_ROW = [2, 8, 9, 7, 9, 6, 8, 7, 8, 9]                # :31
SYMFACT_A_NUM_ROW = [2, 1, 2, 2, 2, 1, 0]                       # src/test/algorithms/symbolic_factorize_test.f90:17
SYMFACT_A_ROW = [2, 8, 9, 7, 9, 6, 8, 7, 8, 9]                  # :18
SYMFACT_L = [2, 8, 8, 9, 7, 9, 6, 8, 7, 8, 8, 9]                # :27
LOCAL_INDEX = [1, 2, 1, 2, 1, 3, 1, 3, 1, 2, 1, 2]              # create_local_index_test.f90:21
SIDX_NODE_SIZE = [2, 2, 2, 3]                                   # create_supernodal_index_test.f90:14
SIDX_L_LEN = [2, 2, 2, 0]                                       # :15
SIDX_L_VAL = [8, 9, 7, 9, 7, 8]                                 # :15
SIDX_A_LEN = [3, 2, 4, 2, 3, 3, 2, 1, 1]                        # :17
SIDX_A_VAL = [1, 2, 8, 2, 9, 3, 4, 7, 9, 4, 9, 5, 6, 8, 6, 7, 8, 7, 9, 8, 9]  # :17
SIDX = [1, 2, 3, 2, 4, 1, 2, 3, 4, 2, 4, 1, 2, 4, 2, 3, 4, 1, 3, 2, 3]  # :19

# relax_supernode_test.f90:20-48 : merge lists per max_zero, {list head: members}
RELAX_MERGE = {
    0: {1: [1], 2: [2], 3: [3], 4: [4], 5: [5], 7: [7, 6]},
    1: {2: [2, 1], 3: [3], 5: [5, 4], 7: [7, 6]},
    2: {5: [5, 4], 6: [6, 3], 7: [7, 2, 1]},
}

# ---------------------------------------------------------------------------
# block_local_index_info_test.f90 (4 cases) and block_local_index_creator_test.f90
# ---------------------------------------------------------------------------
BLI_CASES = [
    {   # test1 :21-62
        "l_len": [4, 0], "l_val": [2, 3, 7, 8], "nc": [5, 8], "nr": [4, 0], "nb": 3,
        "groups": {(1, 1): [2], (1, 2): [3], (1, 3): [1, 2]},
        "start_row": {(1, 1): 1, (1, 2): 2, (1, 3): 3},
        "offset": {(1, 1): 0, (1, 2): 0, (1, 3): 1},
        "parent": {(1, 1): 1, (1, 2): 1, (1, 3): 3},
        "child": {(1, 1): 2, (1, 2): 3, (1, 3): 3},
        "num_block": {1: 3, 2: 0},
    },
    {   # test2 :64-140
        "l_len": [3, 2, 2, 1, 0], "l_val": [2, 4, 6, 1, 5, 2, 3, 1], "nc": [3, 2, 4, 1, 3],
        "nr": [3, 2, 2, 1, 0], "nb": 2,
        "groups": {(1, 1): [2], (1, 2): [2], (1, 3): [2], (2, 1): [1], (2, 2): [1], (3, 1): [2],
                   (3, 2): [1], (4, 1): [1]},
        "start_row": {(1, 1): 1, (1, 2): 2, (1, 3): 3, (2, 1): 1, (2, 2): 2, (3, 1): 1, (3, 2): 2, (4, 1): 1},
        "offset": {(1, 1): 0, (1, 2): 0, (1, 3): 1, (2, 1): 0, (2, 2): 1, (3, 1): 0, (3, 2): 1, (4, 1): 0},
        "parent": {(1, 1): 1, (1, 2): 2, (1, 3): 3, (2, 1): 1, (2, 2): 3, (3, 1): 1, (3, 2): 2, (4, 1): 1},
        "child": {(1, 1): 2, (1, 2): 3, (1, 3): 3, (2, 1): 2, (2, 2): 2, (3, 1): 3, (3, 2): 3, (4, 1): 1},
        "num_block": {1: 3, 2: 2, 3: 2, 4: 1, 5: 0},
    },
    {   # test3 :142-218
        "l_len": [3, 2, 3, 1, 0], "l_val": [2, 4, 7, 1, 6, 1, 2, 3, 1], "nc": [3, 2, 4, 1, 3],
        "nr": [3, 2, 3, 1, 0], "nb": 2,
        "groups": {(1, 1): [2], (1, 2): [2], (1, 3): [1], (2, 1): [1], (2, 2): [2], (3, 1): [1, 2],
                   (3, 2): [1], (4, 1): [1]},
        "start_row": {(1, 1): 1, (1, 2): 2, (1, 3): 3, (2, 1): 1, (2, 2): 2, (3, 1): 1, (3, 2): 3, (4, 1): 1},
        "offset": {(1, 1): 0, (1, 2): 0, (1, 3): 1, (2, 1): 0, (2, 2): 1, (3, 1): 0, (3, 2): 0, (4, 1): 0},
        "parent": {(1, 1): 1, (1, 2): 2, (1, 3): 4, (2, 1): 1, (2, 2): 3, (3, 1): 1, (3, 2): 2, (4, 1): 1},
        "child": {(1, 1): 2, (1, 2): 3, (1, 3): 3, (2, 1): 2, (2, 2): 2, (3, 1): 3, (3, 2): 4, (4, 1): 1},
        "num_block": {1: 3, 2: 2, 3: 2, 4: 1, 5: 0},
    },
    {   # test4 :220-239
        "l_len": [5, 3, 0], "l_val": [2, 3, 4, 5, 7, 1, 3, 4], "nc": [4, 5, 4], "nr": [5, 2, 0], "nb": 3,
        "groups": {(1, 1): [2, 3], (1, 2): [1, 2], (1, 3): [1], (2, 1): [1], (2, 2): [3], (2, 3): [1]},
        "offset": {(1, 1): 0, (1, 2): 0, (1, 3): 2, (2, 1): 0, (2, 2): 0, (2, 3): 1},
        "num_block": {1: 3, 2: 3, 3: 0},
    },
]
# block_local_index_creator_test.f90: rebuilt (mod nb) values and per-group index counts
BLI_CREATOR = [
    {"case": 0, "num_indices": [1, 1, 2], "rebuilt": [2, 3, 1, 2]},                       # :21-36
    {"case": 1, "num_indices": [1, 1, 1, 1, 1, 1, 1, 1], "rebuilt": [2, 2, 2, 1, 1, 2, 1, 1]},  # :38-62
    {"case": 2, "num_indices": [1, 1, 1, 1, 1, 2, 1, 1], "rebuilt": [2, 2, 1, 1, 2, 1, 2, 1, 1]},  # :64-88
]

# ---------------------------------------------------------------------------
# node geometry: node_data_test.f90 and cost_calculator_test.f90
# ---------------------------------------------------------------------------
NODE_DATA = {
    "nc": [5, 6, 7, 5, 3, 6], "nr": [5, 4, 4, 4, 6, 0], "nb": 3,                          # node_data_test.f90:13-15
    "ssize": [2, 0, 1, 2, 0, 0],                                                          # :22
    "wsize": [1, 3, 2, 1, 3, 0],                                                          # :26
    "num_block": [4, 4, 4, 3, 3, 2],                                                      # :27-34
    "work_start": [2, 3, 3, 2, 2],                                                        # :35-41 (nodes 1-5)
}
COST = {"nc": [5, 8], "nr": [4, 0], "nb": 3, "cost": 459, "nonzero": 71}                  # cost_calculator_test.f90:10-20
BIG_COST = {"nc": [1], "nr": [999999999], "cost": 1000000000000000000}                  # :13-15

# ---------------------------------------------------------------------------
# whole numeric phase on the 3-supernode toy (13x13, integer-valued L):
# seq_factorize/seq_factorize_test.f90:23-100, seq_solve/seq_forward_test.f90,
# seq_solve/seq_backward_test.f90
# ---------------------------------------------------------------------------
TOY_NODE_SIZE = [4, 5, 4]                                                                 # seq_factorize_test.f90:24
TOY_WORK_SIZE = [5, 3, 0]                                                                 # :30
TOY_LOCAL_LEN = [5, 3, 0]                                                                 # :25
TOY_LOCAL_VAL = [2, 3, 4, 5, 7, 1, 3, 4]                                                  # :25
TOY_PARENT = [2, 3, 0]                                                                    # :35
TOY_VALUES = [1, 2, 3, 4, 1, 2, 3, 4, 5, 8, 12, 16, 4, 8, 12, 16, 20, 27, 36, 9, 18, 27, 36, 45, 64, 16, 32, 48, 64,
              80, 1, 2, 3, 4, 5, 1, 2, 3, 12, 20, 28, 36, 4, 28, 12, 43, 60, 77, 9, 58, 27, 100, 128, 16, 92, 48,
              189, 25, 130, 75, 6, 2, 13, 19, 8, 12, 16, 147, 66, 109]                      # :27
TOY_SIDX_LEN = [9, 8, 7, 6, 8, 7, 6, 5, 4, 4, 3, 2, 1]                                    # :28
TOY_SIDX_VAL = [1, 2, 3, 4, 5, 6, 7, 8, 9, 2, 3, 4, 5, 6, 7, 8, 9, 3, 4, 5, 6, 7, 8, 9, 4, 5, 6, 7, 8, 9, 1, 2, 3,
                4, 5, 6, 7, 8, 2, 3, 4, 5, 6, 7, 8, 3, 4, 5, 6, 7, 8, 4, 5, 6, 7, 8, 5, 6, 7, 8, 1, 2, 3, 4, 2, 3,
                4, 3, 4, 4]                                                               # :28

# expected factor tiles get_supernode(node, i, j); "tri" entries list the upper
# triangle of an n x n tile column by column (test_util add_test_tri semantics)
TOY_FACTOR_NB2 = [                                                                        # :55-79
    ("tri", 1, 1, 1, [1, 2, 2], 2), ("full", 1, 2, 1, [3, 3, 4, 4]), ("full", 1, 3, 1, [1, 1, 2, 2]),
    ("full", 1, 4, 1, [3, 3, 4, 4]), ("full", 1, 5, 1, [5, 5]), ("tri", 1, 2, 2, [3, 4, 4], 2),
    ("full", 1, 3, 2, [1, 1, 2, 2]), ("full", 1, 4, 2, [3, 3, 4, 4]), ("full", 1, 5, 2, [5, 5]),
    ("tri", 2, 1, 1, [1, 2, 2], 2), ("full", 2, 2, 1, [3, 3, 4, 4]), ("full", 2, 3, 1, [5, 5, 1, 1]),
    ("full", 2, 4, 1, [2, 2, 3, 3]), ("tri", 2, 2, 2, [3, 4, 4], 2), ("full", 2, 3, 2, [5, 5, 1, 1]),
    ("full", 2, 4, 2, [2, 2, 3, 3]), ("full", 2, 4, 3, [2, 3]),
    ("tri", 3, 1, 1, [1, 2, 2], 2), ("full", 3, 2, 1, [3, 3, 4, 4]), ("tri", 3, 2, 2, [3, 4, 4], 2),
]
TOY_FACTOR_NB3 = [                                                                        # :81-100
    ("tri", 1, 1, 1, [1, 2, 2, 3, 3, 3], 3), ("full", 1, 2, 1, [4, 4, 4, 1, 1, 1, 2, 2, 2]),
    ("full", 1, 3, 1, [3, 3, 3, 4, 4, 4, 5, 5, 5]), ("full", 1, 2, 2, [4, 1, 2]), ("full", 1, 3, 2, [3, 4, 5]),
    ("tri", 2, 1, 1, [1, 2, 2, 3, 3, 3], 3), ("full", 2, 2, 1, [4, 4, 4, 5, 5, 5, 1, 1, 1]),
    ("full", 2, 3, 1, [2, 2, 2, 3, 3, 3]), ("tri_head", 2, 2, 2, [4, 5, 5], 2), ("rect_tail", 2, 2, 2, [1, 1], 4),
    ("full", 2, 3, 2, [2, 2, 3, 3]),
    ("tri", 3, 1, 1, [1, 2, 2, 3, 3, 3], 3), ("full", 3, 2, 1, [4, 4, 4]), ("tri", 3, 2, 2, [4], 1),
]

# factor tiles preset by the solve tests (seq_forward_test.f90:35-55, :73-85)
TOY_L_TILES_NB2 = [
    (1, 1, 1, [1, 0, 2, 2]), (1, 2, 1, [3, 3, 4, 4]), (1, 3, 1, [1, 1, 2, 2]), (1, 4, 1, [3, 3, 4, 4]),
    (1, 5, 1, [5, 5]), (1, 2, 2, [3, 0, 4, 4]), (1, 3, 2, [1, 1, 2, 2]), (1, 4, 2, [3, 3, 4, 4]), (1, 5, 2, [5, 5]),
    (2, 1, 1, [1, 0, 2, 2]), (2, 2, 1, [3, 3, 4, 4]), (2, 3, 1, [5, 5, 1, 1]), (2, 4, 1, [2, 2, 3, 3]),
    (2, 2, 2, [3, 0, 4, 4]), (2, 3, 2, [5, 5, 1, 1]), (2, 4, 2, [2, 2, 3, 3]), (2, 3, 3, [5, 1]), (2, 4, 3, [2, 3]),
    (3, 1, 1, [1, 0, 2, 2]), (3, 2, 1, [3, 3, 4, 4]), (3, 2, 2, [3, 0, 4, 4]),
]
TOY_L_TILES_NB3 = [
    (1, 1, 1, [1, 0, 0, 2, 2, 0, 3, 3, 3]), (1, 2, 1, [4, 4, 4, 1, 1, 1, 2, 2, 2]),
    (1, 3, 1, [3, 3, 3, 4, 4, 4, 5, 5, 5]), (1, 2, 2, [4, 1, 2]), (1, 3, 2, [3, 4, 5]),
    (2, 1, 1, [1, 0, 0, 2, 2, 0, 3, 3, 3]), (2, 2, 1, [4, 4, 4, 5, 5, 5, 1, 1, 1]), (2, 3, 1, [2, 2, 2, 3, 3, 3]),
    (2, 2, 2, [4, 0, 5, 5, 1, 1]), (2, 3, 2, [2, 2, 3, 3]),
    (3, 1, 1, [1, 0, 0, 2, 2, 0, 3, 3, 3]), (3, 2, 1, [4, 4, 4, 4]), (3, 2, 2, [4]),
]
TOY_FORWARD_RHS = [1, 4, 9, 16, 1, 8, 17, 28, 41, 6, 4, 39, 31]                          # seq_forward_test.f90:32
TOY_BACKWARD_RHS = [25, 24, 22, 19, 21, 20, 18, 15, 11, 10, 9, 7, 4]                     # seq_backward_test.f90:30

# end-to-end fixture matrices used by src/test/hppllt_test.f90:12-15 (generated
# into mtx_fixtures.json by make_mtx_fixtures.py); the test asserts error <= 1e-8
HPPLLT_TEST_OPTIONS = [10, 10, 1, 0]                                                      # src/test/hppllt_test.f90:14
HPPLLT_TEST_TOL = 1e-8
