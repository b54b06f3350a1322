"""The library's fill-reducing ordering (mfd_order: nested dissection of the
matrix graph), which stands where the reference calls METIS_NodeND
(ordering_m.f90:11-36, use_metis = 1).  METIS's own output is pinned by no
reference test; what is checked is what the analysis relies on: a valid,
deterministic permutation (new -> old, 1-based), fill far below the natural
order's, and a correct factorization under it (oracle on the CPU, the GPU
path through the reference-named API)."""
import json
import os

import numpy as np
import pytest

from mfdag import hppllt as H
from mfdag import problems as P
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def fill(p, order, max_zero=10):
    sym = H.symbolic_analyze(p.n, p.col, p.row, order, max_zero=max_zero)
    nc = np.diff(sym["node_ptr"]).astype(np.int64)
    nr = np.diff(sym["lptr"]).astype(np.int64)
    return int(((nr + nc) * (nr + nc + 1) // 2 - nr * (nr + 1) // 2).sum())


CASES = [("lap2d_60", lambda: P.laplace2d(60)), ("lap3d_20", lambda: P.laplace3d(20)),
         ("diff3d_16", lambda: P.diffusion3d(16)), ("elast_8", lambda: P.elasticity3d(8, 4, 1))]


@pytest.mark.parametrize("name,mk", CASES, ids=[c[0] for c in CASES])
def test_order_is_a_deterministic_permutation(name, mk):
    p = mk()
    o = H.order(p.n, p.col, p.row)
    assert o.dtype == np.int32 and sorted(o.tolist()) == list(range(1, p.n + 1))
    assert np.array_equal(o, H.order(p.n, p.col, p.row))


@pytest.mark.parametrize("name,mk,vs_nat,vs_geo", [("lap2d_60", lambda: P.laplace2d(60), 0.4, 1.0),
                                                    ("lap3d_20", lambda: P.laplace3d(20), 0.25, 0.7),
                                                    ("elast_12", lambda: P.elasticity3d(12, 4, 1), 0.85, 1.6)],
                         ids=["lap2d_60", "lap3d_20", "elast_12"])
def test_order_fill(name, mk, vs_nat, vs_geo):
    """nnz(L) under the ordering against the natural order and against the
    geometric nested dissection on the grid's own coordinates (which the graph
    ordering does not see).  On the 5- and 7-point grids the level-structure
    separators (diagonal planes) beat the axis planes; on the elasticity mesh,
    whose nodes couple to all 26 neighbours, BFS levels are cube shells and
    the ordering trails the geometric one."""
    p = mk()
    nd = fill(p, H.order(p.n, p.col, p.row))
    assert nd <= vs_nat * fill(p, None)
    assert nd <= vs_geo * fill(p, p.order)


def test_unknowns_of_a_node_stay_together():
    """Compression: the three unknowns of each mesh node of the elasticity
    problem have identical graph neighbourhoods and come out consecutive."""
    p = P.elasticity3d(6, 4, 1)
    o = H.order(p.n, p.col, p.row) - 1
    node = o // 3
    assert np.all(node.reshape(-1, 3) == node.reshape(-1, 3)[:, :1])


def test_oracle_factorization_under_the_ordering():
    p = P.laplace3d(16)
    o = H.order(p.n, p.col, p.row)
    orc = O.Oracle.analyze(p.n, p.col, p.row, nb=10, max_zero=10, order_perm=o)
    assert orc.factorize(p.val) == 0
    x = orc.solve(p.rhs)
    assert P.backward_error(p.n, p.col, p.row, p.val, x, p.rhs) <= 1e-14


def test_order_rejects_bad_input():
    p = P.laplace2d(5)
    bad = p.row.copy()
    bad[3] = p.n + 4
    with pytest.raises(H.MfdError):
        H.order(p.n, p.col, bad)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["bcsstk01.mtx", "poisson_9_9.mtx"])
def test_hppllt_use_metis_without_an_ordering(name):
    """hppllt_init with use_metis = 1 and no hppllt_set_ordering: the analysis
    takes mfd_order's ordering (the reference would call METIS_NodeND) and the
    fixture's end-to-end check passes, like hppllt_test.f90:12-37 with metis on."""
    from golden import reference_vectors as R
    from test_oracle_e2e import coo_to_ccs, sym_matvec
    m = json.load(open(os.path.join(HERE, "golden", "mtx_fixtures.json")))[name]
    n = m["n"]
    ptr, row, val = coo_to_ccs(n, m["row"], m["col"], m["val"])
    opts = list(R.HPPLLT_TEST_OPTIONS[:2]) + [1, 1]
    H.hppllt_init(opts)
    H.hppllt_set_ordering(np.zeros(0, np.int32))                # none supplied
    H.hppllt_analyze(ptr, row, n)
    assert H.hppllt_factorize(val) == 0
    b = np.full(n, 10.0)
    H.hppllt_solve(b)
    r = 10.0 - sym_matvec(n, ptr, row, val, b)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= R.HPPLLT_TEST_TOL
    H.hppllt_finalize()
