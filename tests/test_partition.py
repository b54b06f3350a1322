"""Subtree-to-GPU mapping of one system: the reference's tree_pruning
(src/main/algorithms/tree_pruning_m.f90:13-155), restated in the product
(mfd_subtree_partition) and in the oracle, pinned on the reference's own test
(tree_pruning_test.f90:23-33) and compared on the configurations' trees."""
import numpy as np
import pytest

from golden import reference_vectors as R
from mfdag import hppllt as H
from mfdag import problems as P
from mfdag import sharding
from oracle import oracle as O


@pytest.mark.parametrize("tol,p,want", R.TREE_PRUNING_CASES)
def test_tree_pruning_reference_cases(tol, p, want):
    args = (R.SN_NODE_SIZE, R.SN_CC, R.SN_TREE_NUM_CHILD, R.SN_TREE_CHILD_VAL, tol, p)
    assert O.tree_pruning(*args) == want
    assert H.subtree_partition(*args) == want


@pytest.mark.parametrize("mk", [lambda: P.laplace3d(24), lambda: P.diffusion3d(16), lambda: P.laplace2d(80),
                                lambda: P.elasticity3d(8, 4, 1)], ids=["lap3d", "diff3d", "lap2d", "elast"])
def test_product_matches_oracle_on_config_trees(mk):
    p = mk()
    sym = H.symbolic_analyze(p.n, p.col, p.row, p.order, max_zero=100)
    tree = H.tree_of(sym)
    for workers in (1, 2, 3, 4, 8):
        for tol in (0.0, 0.5, 0.8):
            assert H.subtree_partition(*tree, tol, workers) == O.tree_pruning(*tree, tol, workers), (workers, tol)


def test_subtrees_cover_disjoint_parts_and_balance():
    """The roots are disjoint subtrees; with tol = 0.8 and 4 workers the LPT
    packing of their weights (sharding.assign_subtrees) is within 1/0.8 of the
    lightest worker."""
    p = P.laplace3d(24)
    sym = H.symbolic_analyze(p.n, p.col, p.row, p.order, max_zero=100)
    ns, cc, nch, ch = H.tree_of(sym)
    roots = H.subtree_partition(ns, cc, nch, ch, 0.8, 4)
    parent = np.asarray(sym["parent"])
    anc = set()
    for r in roots:                                         # no root lies inside another root's subtree
        v = parent[r - 1]
        while v:
            assert v not in roots
            anc.add(int(v))
            v = parent[v - 1]
    w = sharding.subtree_weights(ns, cc, nch, ch)
    parts = sharding.assign_subtrees([w[r - 1] for r in roots], 4)
    loads = [sum(w[roots[i] - 1] for i in part) for part in parts]
    assert min(loads) / max(loads) > 0.8
    assert sorted(i for part in parts for i in part) == list(range(len(roots)))
