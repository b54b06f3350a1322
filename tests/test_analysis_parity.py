"""The product's C++ host analysis (mfd_symbolic_analyze) against the oracle's
literal restatement of the reference's hppllt_analyze: every symbolic array
must be bit-exact."""
import json
import os

import numpy as np
import pytest

from mfdag import hppllt, problems as P
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
KEYS = ["node_ptr", "parent", "lptr", "lrow", "aptr", "arow", "ccs_perm", "perm"]


def compare(n, col, row, order, max_zero):
    got = hppllt.symbolic_analyze(n, col, row, order, max_zero)
    o = O.Oracle.analyze(n, col, row, nb=10, max_zero=max_zero, order_perm=order)
    ref = o.symbolic()
    assert got["num_node"] == ref["num_node"]
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k
    return got


def random_spd_pattern(n, density, seed):
    rng = np.random.default_rng(seed)
    rows, cols = [np.arange(n)], [np.arange(n)]
    m = int(density * n * n / 2)
    r = rng.integers(0, n, m)
    c = rng.integers(0, n, m)
    lo, hi = np.minimum(r, c), np.maximum(r, c)
    keep = lo != hi
    rows.append(hi[keep]); cols.append(lo[keep])
    # chain keeps the graph connected (one elimination tree)
    rows.append(np.arange(1, n)); cols.append(np.arange(n - 1))
    R, Cc = np.concatenate(rows), np.concatenate(cols)
    key = np.unique(Cc.astype(np.int64) * n + R)
    Cc, R = key // n, key % n
    v = np.where(R == Cc, float(n), -1.0)
    return P._lower_ccs(n, R, Cc, v)


@pytest.mark.parametrize("max_zero", [0, 10, 1000])
def test_laplace2d(max_zero):
    p = P.laplace2d(24)
    compare(p.n, p.col, p.row, p.order, max_zero)
    compare(p.n, p.col, p.row, None, max_zero)


@pytest.mark.parametrize("max_zero", [10, 1000])
def test_laplace3d(max_zero):
    p = P.laplace3d(10)
    compare(p.n, p.col, p.row, p.order, max_zero)


def test_diffusion3d():
    p = P.diffusion3d(9)
    compare(p.n, p.col, p.row, p.order, 10)


@pytest.mark.parametrize("seed", range(6))
def test_random_patterns(seed):
    n = 60 + 17 * seed
    col, row, _ = random_spd_pattern(n, 0.04, seed)
    rng = np.random.default_rng(100 + seed)
    order = (rng.permutation(n) + 1).astype(np.int32)
    for mz in (0, 5, 50):
        compare(n, col, row, None, mz)
        compare(n, col, row, order, mz)


@pytest.mark.parametrize("name", ["bcsstk01.mtx", "poisson_9_9.mtx"])
def test_fixture_matrices(name):
    from test_oracle_e2e import coo_to_ccs
    m = json.load(open(os.path.join(HERE, "golden", "mtx_fixtures.json")))[name]
    ptr, row, _ = coo_to_ccs(m["n"], m["row"], m["col"], m["val"])
    compare(m["n"], ptr, row, None, 10)


def test_cfg1_size():
    p = P.laplace2d(100)
    s = compare(p.n, p.col, p.row, p.order, 10)
    assert s["num_node"] > 1000
