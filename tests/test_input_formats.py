"""The input path ahead of the analysis: the Matrix Market reader, the COO ->
CCS conversion on the GPU, and direct CSR input.

The reference driver reads a Matrix Market file (read_data, example.f90:63-93)
and converts its coordinate lists with two counting sorts (coo_to_ccs,
example.f90:95-145).  The oracle restates that conversion step by step; its
output order -- rows ascending in each column, entries with equal (row, col)
in reverse input order -- is pinned here by a case worked by hand through the
Fortran loops, and the GPU conversion must reproduce the oracle bit for bit.
"""
import json
import os

import numpy as np
import pytest

from mfdag import hppllt as H
from mfdag import problems as P
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = json.load(open(os.path.join(HERE, "golden", "mtx_fixtures.json")))

# Hand-worked through example.f90:95-145 (n = 3): input order
# (1,1)=1, (3,1)=2, (2,1)=3, (3,1)=4, (2,2)=5, (3,3)=6.  The row sort fills each
# row's segment from its end: tmp = (1,1)1 (2,2)5 (2,1)3 (3,3)6 (3,1)4 (3,1)2; the
# column pass walks tmp backwards and fills each column from its end.
KAT_IN = ([1, 3, 2, 3, 2, 3], [1, 1, 1, 1, 2, 3], [1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
KAT_OUT = ([1, 5, 6, 7], [1, 2, 3, 3, 2, 3], [1.0, 3.0, 4.0, 2.0, 5.0, 6.0])


def write_mtx(path, m, style):
    """A Matrix Market file with the layouts of the reference's two test
    matrices: a banner and comment header (bcsstk01.mtx) or none with
    right-aligned fixed-width columns (poisson_9_9.mtx)."""
    with open(path, "w") as f:
        if style == "banner":
            f.write("%%MatrixMarket matrix coordinate real symmetric\n")
            f.write("%-------------------------------------------------------------------------------\n")
            f.write("% a comment line\n")
            f.write(f"{m['n']} {m['n']} {len(m['row'])}\n")
            for r, c, v in zip(m["row"], m["col"], m["val"]):
                f.write(f"{r} {c} {v!r}\n")
        else:
            f.write(f"{m['n']:10d}{m['n']:10d}{len(m['row']):10d}\n")
            for r, c, v in zip(m["row"], m["col"], m["val"]):
                f.write(f"{r:10d}{c:10d}{v:20.1f}\n")


# ---------------------------------------------------------------------------
# CPU: the reader and the oracle's conversion
# ---------------------------------------------------------------------------
def test_oracle_coo_to_ccs_hand_worked_case():
    ptr, row, val = O.coo_to_ccs(3, *KAT_IN)
    assert ptr.tolist() == KAT_OUT[0] and row.tolist() == KAT_OUT[1] and val.tolist() == KAT_OUT[2]


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_oracle_coo_to_ccs_on_reference_matrices(name):
    """Without duplicate entries the conversion is the (column, row) sort."""
    m = FIXTURES[name]
    ptr, row, val = O.coo_to_ccs(m["n"], m["row"], m["col"], m["val"])
    order = np.lexsort((np.array(m["row"]), np.array(m["col"])))
    assert row.tolist() == np.array(m["row"])[order].tolist()
    assert val.tolist() == np.array(m["val"])[order].tolist()
    assert ptr[-1] == len(m["row"]) + 1 and np.all(np.diff(ptr) >= 0)


@pytest.mark.parametrize("name,style", [("bcsstk01.mtx", "banner"), ("poisson_9_9.mtx", "fixed")])
def test_mm_read_reference_layouts(tmp_path, name, style):
    m = FIXTURES[name]
    path = tmp_path / name
    write_mtx(path, m, style)
    got = H.mm_read(str(path))
    assert got["n"] == m["n"]
    assert got["row"].tolist() == m["row"] and got["col"].tolist() == m["col"]
    assert np.array_equal(got["val"], np.array(m["val"]))


def test_mm_read_pattern_and_errors(tmp_path):
    p = tmp_path / "pat.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n1 1\n3 2\n")
    got = H.mm_read(str(p))
    assert got["row"].tolist() == [1, 3] and got["val"].tolist() == [1.0, 1.0]
    short = tmp_path / "short.mtx"
    short.write_text("3 3 4\n1 1 1.0\n2 2 1.0\n")
    with pytest.raises(H.MfdError):
        H.mm_read(str(short))
    rect = tmp_path / "rect.mtx"
    rect.write_text("3 4 1\n1 1 1.0\n")
    with pytest.raises(H.MfdError):
        H.mm_read(str(rect))
    with pytest.raises(H.MfdError):
        H.mm_read(str(tmp_path / "missing.mtx"))


# ---------------------------------------------------------------------------
# GPU: conversion, CSR input, the driver's whole flow
# ---------------------------------------------------------------------------
def shuffled_lower_coo(p, seed, dup=0):
    """The lower-triangle entries of a problem as COO in a random order, with
    `dup` entries repeated (a duplicate keeps its own value)."""
    cols = np.repeat(np.arange(1, p.n + 1), np.diff(p.col)).astype(np.int32)
    rows, vals = p.row.copy(), p.val.copy()
    rng = np.random.default_rng(seed)
    if dup:
        d = rng.choice(rows.size, dup, replace=False)
        rows, cols, vals = (np.concatenate([x, x[d]]) for x in (rows, cols, vals))
        vals[-dup:] += 1.0
    o = rng.permutation(rows.size)
    return rows[o], cols[o], vals[o]


@pytest.mark.gpu
def test_device_coo_to_ccs_matches_oracle():
    cases = [(3,) + KAT_IN]
    for name in sorted(FIXTURES):
        m = FIXTURES[name]
        cases.append((m["n"], m["row"], m["col"], m["val"]))
    p = P.laplace3d(12)
    cases.append((p.n,) + shuffled_lower_coo(p, 1, dup=50))
    for n, r, c, v in cases:
        want = O.coo_to_ccs(n, r, c, v)
        got = H.coo_to_ccs(n, r, c, v)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
        ptr, row, none = H.coo_to_ccs(n, r, c)                  # structure only
        assert none is None and np.array_equal(ptr, want[0]) and np.array_equal(row, want[1])


@pytest.mark.gpu
def test_device_coo_to_ccs_device_pointers_and_size():
    """Device-resident input and output; a 3D Laplacian of 216,000 rows in a
    shuffled order comes back as its lower CCS; a bad index is refused."""
    import torch
    p = P.laplace3d(60)
    r, c, v = shuffled_lower_coo(p, 2)
    tr, tc, tv = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (r, c, v))
    ptr, row, val = H.coo_to_ccs(p.n, tr, tc, tv)
    assert np.array_equal(ptr.cpu().numpy(), p.col)
    assert np.array_equal(row.cpu().numpy(), p.row)
    assert np.array_equal(val.cpu().numpy(), p.val)
    bad = r.copy()
    bad[7] = p.n + 1
    with pytest.raises(H.MfdError):
        H.coo_to_ccs(p.n, bad, c, v)


def full_csr(p, base, lower_only):
    """CSR (0- or 1-based) of a problem stored as its lower CCS: the lower
    triangle's CSR is the upper CCS; the whole matrix has both.  Also the map
    from CSR positions to the problem's CCS entries (-1 for upper entries)."""
    cols = np.repeat(np.arange(p.n), np.diff(p.col))
    rows = p.row - 1
    ent = [(rows, cols, np.arange(rows.size))]
    if not lower_only:
        off = rows != cols
        ent.append((cols[off], rows[off], -1 - np.arange(rows.size)[off]))
    R = np.concatenate([e[0] for e in ent]); Cc = np.concatenate([e[1] for e in ent])
    K = np.concatenate([e[2] for e in ent])
    o = np.lexsort((Cc, R))
    R, Cc, K = R[o], Cc[o], K[o]
    ptr = np.concatenate([[0], np.cumsum(np.bincount(R, minlength=p.n))]) + base
    vals = p.val[np.where(K >= 0, K, -1 - K)]
    return ptr.astype(np.int32), (Cc + base).astype(np.int32), vals


@pytest.mark.gpu
@pytest.mark.parametrize("base,lower_only", [(0, False), (1, True)], ids=["full_0based", "lower_1based"])
def test_analyze_csr_matches_ccs_path(base, lower_only):
    """mfd_analyze_csr: the handle takes values in the caller's CSR order and
    factors to the same bits as the lower-CCS path."""
    p = P.laplace3d(16)
    ptr, col, vals = full_csr(p, base, lower_only)
    s = H.Solver.analyze_csr(p.n, ptr, col, base, p.order, max_zero=10)
    assert s.factorize(vals) == 0
    x = p.rhs.copy()
    rep, rc = s.solve(x)
    assert rc == 0 and rep.backward_error <= 1e-12
    t = H.Solver.analyze(p.n, p.col, p.row, p.order, max_zero=10)
    assert t.factorize(p.val) == 0
    y = p.rhs.copy()
    t.solve(y)
    assert np.array_equal(x, y)
    assert np.array_equal(s.index(H.SUPERNODAL_INDEX), t.index(H.SUPERNODAL_INDEX))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_matrix_market_file_through_the_reference_api(tmp_path, name):
    """The reference driver's flow (example.f90:13-60, the checks of
    hppllt_test.f90:12-37) from a file: read, convert on the GPU, analyse,
    factor and solve with the reference-named entry points."""
    from golden import reference_vectors as R
    from test_oracle_e2e import sym_matvec
    m = FIXTURES[name]
    path = tmp_path / name
    write_mtx(path, m, "banner")
    coo = H.mm_read(str(path))
    ptr, row, val = H.coo_to_ccs(coo["n"], coo["row"], coo["col"], coo["val"])
    n = coo["n"]
    H.hppllt_init(R.HPPLLT_TEST_OPTIONS)
    H.hppllt_analyze(ptr, row, n)
    assert H.hppllt_factorize(val) == 0
    b = np.full(n, 10.0)
    H.hppllt_solve(b)
    r = 10.0 - sym_matvec(n, ptr, row, val, b)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= R.HPPLLT_TEST_TOL
    H.hppllt_finalize()
