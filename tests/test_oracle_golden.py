"""Pin the CPU oracle against the reference's own unit-test vectors.

Every expected value comes from tests/golden/reference_vectors.py, which is a
transcription (with file:line citations) of the reference's Fortran tests.
"""
import numpy as np
import pytest

from golden import reference_vectors as R
from oracle import oracle as O


def test_compute_tree():                                   # compute_tree_test.f90
    assert list(O.compute_tree(R.CRS9_NUM_COL, R.CRS9_COL)) == R.ORIG_TREE_PARENT


def test_postorder_and_subtree():                         # tree_test.f90:21-24
    perm, sub = O.postorder(R.ORIG_TREE_PARENT)
    assert list(perm) == R.TREE_POSTORDER
    assert list(sub) == R.TREE_SUBTREE_SIZE


def test_parent_in_postordering_tree():                   # tree_test.f90:28-30
    assert list(O.parent_in_postordering_tree(R.POST_TREE_NUM_CHILD)) == R.POST_TREE_PARENT


def test_column_count():                                  # column_count_test.f90
    cc = O.column_count(R.POST9_NUM_ROW, R.POST9_ROW, R.POST_TREE_PARENT)
    assert list(cc) == R.COLUMN_COUNT


def test_finding_leaves():                                # finding_leaves_test.f90
    assert list(O.finding_leaves(R.FINDING_LEAVES_SUBTREE, R.POST9_NUM_ROW, R.POST9_ROW)) == R.FINDING_LEAVES


def test_fundamental_supernodes():                        # fundamental_supernode_test.f90
    sets = O.search_node_sets(R.FINDING_LEAVES, R.POST_TREE_NUM_CHILD, R.POST_TREE_CHILD_VAL)
    assert list(sets) == R.FUND_FIRST_NODE
    lens, rows = O.supernodal_ccs(R.POST9_NUM_ROW, R.POST9_ROW, sets)
    assert list(lens) == R.FUND_SN_CCS_LEN
    assert list(rows) == R.FUND_SN_CCS_ROW


@pytest.mark.parametrize("max_zero", [0, 1, 2])
def test_relax_merge_lists(max_zero):                     # relax_supernode_test.f90
    lists = O.merge_lists(R.SN9_NUM_ROW, R.SN_TREE_NUM_CHILD, R.SN_TREE_CHILD_VAL, R.SN9_NODE_SIZE, max_zero)
    for head, members in R.RELAX_MERGE[max_zero].items():
        assert lists[head - 1] == members, (max_zero, head)


def test_symbolic_factorize():                            # symbolic_factorize_test.f90
    out = O.symbolic_factorize(R.SYMFACT_A_NUM_ROW, R.SYMFACT_A_ROW, R.SN9_NUM_ROW, R.SN9_NODE_SIZE,
                               R.SN_TREE_NUM_CHILD, R.SN_TREE_CHILD_VAL)
    assert list(out) == R.SYMFACT_L


def test_local_index():                                   # create_local_index_test.f90
    out = O.local_index(R.SN9_NODE_SIZE, R.SN9_NUM_ROW, R.SN9_ROW, R.SN_TREE_NUM_CHILD, R.SN_TREE_CHILD_VAL)
    assert list(out) == R.LOCAL_INDEX


def test_supernodal_index():                              # create_supernodal_index_test.f90
    out = O.supernodal_index(R.SIDX_NODE_SIZE, R.SIDX_L_LEN, R.SIDX_L_VAL, R.SIDX_A_LEN, R.SIDX_A_VAL)
    assert list(out) == R.SIDX


@pytest.mark.parametrize("case", range(len(R.BLI_CASES)))
def test_block_local_index(case):                         # block_local_index_info_test.f90
    c = R.BLI_CASES[case]
    b = O.block_local_index(c["nc"], c["nr"], c["nb"], c["l_len"], c["l_val"])
    node_ptr = b["node_ptr"]
    for node, nb in c["num_block"].items():
        assert node_ptr[node] - node_ptr[node - 1] == nb
    for (node, idx), vals in c["groups"].items():
        g = node_ptr[node - 1] - 1 + idx            # 1-based group id
        lo, hi = b["block_ptr"][g - 1] - 1, b["block_ptr"][g] - 1
        assert list(b["val"][lo:hi]) == vals, (node, idx)
        assert b["offset"][g - 1] == c["offset"][(node, idx)]
        if "start_row" in c:
            assert b["start_row"][g - 1] == c["start_row"][(node, idx)]
        if "parent" in c:
            assert b["parent_num"][g - 1] == c["parent"][(node, idx)]
            assert b["child_num"][g - 1] == c["child"][(node, idx)]


@pytest.mark.parametrize("entry", R.BLI_CREATOR)
def test_block_local_index_creator(entry):                # block_local_index_creator_test.f90
    c = R.BLI_CASES[entry["case"]]
    b = O.block_local_index(c["nc"], c["nr"], c["nb"], c["l_len"], c["l_val"])
    assert list(np.diff(b["block_ptr"])) == entry["num_indices"]
    assert list(b["val"]) == entry["rebuilt"]


def test_node_geometry():                                 # node_data_test.f90
    d = R.NODE_DATA
    g = O.node_geometry(d["nc"], d["nr"], d["nb"])
    assert list(g["ssize"]) == d["ssize"]
    assert list(g["wsize"]) == d["wsize"]
    assert list(g["num_block"]) == d["num_block"]
    assert list(g["work_start"][:5]) == d["work_start"]


def test_cost():                                          # cost_calculator_test.f90
    o = O.Oracle.from_internal([5, 8], [4, 0], [6, 7, 8, 9], [2, 0], 13,
                               O.sets_from_lengths([1] * 13), np.arange(1, 14), 3)
    assert o.cost() == R.COST["cost"]
    assert o.nonzero() == R.COST["nonzero"]


def _toy(nb):
    """The 3-supernode fixture of seq_factorize_test.f90:23-35 in oracle form."""
    sizes = R.TOY_NODE_SIZE
    first = np.concatenate([[1], 1 + np.cumsum(sizes)])
    # L row lists from the local index: child position p in the parent front maps
    # to the parent's column (p <= nc_p) or the parent's L row p-nc_p.
    lrows = [[], [], []]
    for node in (3, 2, 1):
        pass
    loc = [R.TOY_LOCAL_VAL[0:5], R.TOY_LOCAL_VAL[5:8], []]
    parent = R.TOY_PARENT
    for node in (2, 1):                                   # parents before children
        p = parent[node - 1]
        for pos in loc[node - 1]:
            if pos <= sizes[p - 1]:
                lrows[node - 1].append(int(first[p - 1] + pos - 1))
            else:
                lrows[node - 1].append(lrows[p - 1][pos - sizes[p - 1] - 1])
    # A structure in global (permuted) numbering from the supernodal index
    arow, node_of_col = [], np.repeat(np.arange(1, 4), sizes)
    k = 0
    for col in range(13):
        node = node_of_col[col]
        nc = sizes[node - 1]
        for _ in range(R.TOY_SIDX_LEN[col]):
            pos = R.TOY_SIDX_VAL[k]
            arow.append(int(first[node - 1] + pos - 1) if pos <= nc else lrows[node - 1][pos - nc - 1])
            k += 1
    acol = O.sets_from_lengths(R.TOY_SIDX_LEN)
    o = O.Oracle.from_internal(sizes, [len(x) for x in lrows], sum(lrows, []), parent, 13, acol, arow, nb)
    return o, lrows, acol, arow


def test_toy_local_and_supernodal_index():               # the toy's own index data must round-trip
    o, *_ = _toy(2)
    assert list(o.get(O.LOCAL)) == R.TOY_LOCAL_VAL
    assert list(o.get(O.SIDX)) == R.TOY_SIDX_VAL


@pytest.mark.parametrize("nb,expect", [(2, R.TOY_FACTOR_NB2), (3, R.TOY_FACTOR_NB3)])
@pytest.mark.parametrize("schedule", ["seq", "dag"])
def test_seq_factorize_toy(nb, expect, schedule):       # seq_factorize_test.f90:23-100
    """The integer-exact factor of the reference's toy fixture, from the
    sequential loop (seq_factorize) and from the task DAG of the StarPU path
    (starpu_factorize_m.f90, task_test/starpu_factorize_test.f90:103-148
    checks the same values through StarPU) on 4 threads."""
    o, *_ = _toy(nb)
    vals = np.array(R.TOY_VALUES, dtype=np.float64)
    assert (o.factorize(vals) if schedule == "seq" else o.factorize(vals, nthreads=4, schedule="dag")) == 0
    for e in expect:
        kind, node, i, j, vals = e[:5]
        t = o.tile(node, i, j, buffer=1)
        if kind == "full":
            assert list(t) == vals, e
        elif kind in ("tri", "tri_head"):
            n = e[5]
            a = t[: n * n].reshape(n, n, order="F")
            got = [a[jj, ii] for ii in range(n) for jj in range(ii + 1)]
            assert got == vals, e
        elif kind == "rect_tail":
            assert list(t[e[5]:]) == vals, e


@pytest.mark.parametrize("nb,tiles", [(2, R.TOY_L_TILES_NB2), (3, R.TOY_L_TILES_NB3)])
def test_seq_forward_backward_toy(nb, tiles):            # seq_forward_test.f90, seq_backward_test.f90
    o, *_ = _toy(nb)
    for node, i, j, vals in tiles:
        o.set_tile(node, i, j, vals)
    fw = o.sweep(R.TOY_FORWARD_RHS, backward=False)
    assert np.array_equal(fw, np.ones(13))
    bw = o.sweep(R.TOY_BACKWARD_RHS, backward=True)
    assert np.array_equal(bw, np.ones(13))
