"""End-to-end oracle runs on the reference's own fixture matrices
(src/test/hppllt_test.f90:12-15, error <= 1e-8) with use_metis = 0."""
import json
import os

import numpy as np
import pytest

from golden import reference_vectors as R
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def coo_to_ccs(n, row, col, val):
    """example.f90:95-145: counting sorts, rows ascending inside each column."""
    row, col, val = (np.asarray(x) for x in (row, col, val))
    order = np.lexsort((row, col))
    row, col, val = row[order], col[order], val[order]
    ptr = np.concatenate([[1], 1 + np.cumsum(np.bincount(col - 1, minlength=n))]).astype(np.int32)
    return ptr, row.astype(np.int32), val.astype(np.float64)


def sym_matvec(n, ptr, row, val, x):
    y = np.zeros(n)
    for j in range(n):
        lo, hi = ptr[j] - 1, ptr[j + 1] - 1
        r = row[lo:hi] - 1
        v = val[lo:hi]
        y[r] += v * x[j]
        off = r != j
        y[j] += np.dot(v[off], x[r[off]])
    return y


@pytest.mark.parametrize("name", ["bcsstk01.mtx", "poisson_9_9.mtx"])
def test_hppllt_fixture(name):
    m = json.load(open(os.path.join(HERE, "golden", "mtx_fixtures.json")))[name]
    n = m["n"]
    ptr, row, val = coo_to_ccs(n, m["row"], m["col"], m["val"])
    nb, max_zero = R.HPPLLT_TEST_OPTIONS[0], R.HPPLLT_TEST_OPTIONS[1]
    o = O.Oracle.analyze(n, ptr, row, nb=nb, max_zero=max_zero)
    assert o.factorize(val) == 0
    b = np.full(n, 10.0)
    x = o.solve(b)
    r = b - sym_matvec(n, ptr, row, val, x)
    assert np.linalg.norm(r) / np.linalg.norm(x) <= R.HPPLLT_TEST_TOL
    anorm = np.abs(val).max() * 10
    assert np.abs(r).max() / (anorm * np.abs(x).max() + np.abs(b).max()) < 1e-14


@pytest.mark.parametrize("nb", [7, 32, 128])
def test_task_dag_factorization_matches_sequential(nb):
    """The CPU baseline's task-DAG schedule (the StarPU path's tile tasks as
    OpenMP tasks) against the sequential loop, on fronts with and without
    border tile columns: the same factor to rounding (the extend-adds into one
    parent tile commute, so their order may differ) and the same pivot info
    for a matrix that is not positive definite."""
    from mfdag import problems as P
    O.use_system_blas(True)
    p = P.laplace3d(14)
    xs = []
    for sched in ("seq", "dag"):
        o = O.Oracle.analyze(p.n, p.col, p.row, nb=nb, max_zero=200, order_perm=p.order)
        assert (o.factorize(p.val) if sched == "seq" else o.factorize(p.val, nthreads=6, schedule="dag")) == 0
        xs.append(o.solve(p.rhs))
    assert np.abs(xs[0] - xs[1]).max() <= 1e-13 * np.abs(xs[0]).max()
    bad = p.val.copy()
    bad[p.col[300] - 1] = -1.0
    infos = []
    for sched in ("seq", "dag"):
        o = O.Oracle.analyze(p.n, p.col, p.row, nb=nb, max_zero=200, order_perm=p.order)
        infos.append(o.factorize(bad) if sched == "seq" else o.factorize(bad, nthreads=6, schedule="dag"))
    assert infos[0] > 0 and infos[0] == infos[1]
