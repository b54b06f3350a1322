"""The allocation-free front factorization (mfd_factor_fronts_noalloc).

Some callers cannot call cudaMalloc -- code that owns all device memory through
its own arena, or a loop that must not take the allocator's lock -- so this
entry point keeps its only scratch in a static device array.  The test factors
a dense SPD front through it twice in a row (the second call reuses the
scratch array's leftover contents) and compares each result with the factor
the regular handle path (mfd_analyze + mfd_factorize) produces for the same
matrix, within the FP64 factor tolerance of the other parity tests.  It runs the
same alone in a fresh process and after the rest of the suite.
"""
import numpy as np
import pytest

from mfdag import hppllt as H

pytestmark = pytest.mark.gpu
FACTOR_TOL = 1e-12


def dense_spd(n, seed):
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((n, n))
    return m @ m.T / n + 2.0 * np.eye(n)


def lower_ccs(a):
    n = a.shape[0]
    ptr, rows, vals = [1], [], []
    for j in range(n):
        rows.extend(range(j + 1, n + 1))
        vals.extend(a[j:, j])
        ptr.append(len(rows) + 1)
    return np.array(ptr, np.int32), np.array(rows, np.int32), np.array(vals, np.float64)


def handle_factor(a):
    """Factor through the existing entry points; the dense matrix is one front."""
    n = a.shape[0]
    col, row, val = lower_ccs(a)
    s = H.Solver.analyze(n, col, row, None, max_zero=0)
    assert s.stats().num_front == 1
    assert s.factorize(val) == 0
    perm = s.symbolic(H.SYM_PERM) - 1
    panel = s.front_panel(1).reshape(n, n).T          # rows/cols in the permuted order
    return np.tril(panel), perm


def test_noalloc_matches_handle_path_twice():
    import torch
    n = 300                                             # above the fused-kernel limit: the blocked path
    a = dense_spd(n, 11)
    ref, perm = handle_factor(a)
    ap = a[np.ix_(perm, perm)]
    for call in range(2):
        buf = torch.from_numpy(np.asfortranarray(np.tril(ap)).ravel(order="F").copy()).cuda()
        info = H.factor_fronts_noalloc(buf, [0], [0], [n], [n])
        assert info == 0
        got = np.tril(buf.cpu().numpy().reshape(n, n, order="F"))
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= FACTOR_TOL, (call, err)


def test_noalloc_partial_fronts_and_limits():
    import torch
    nf, nc = 260, 170
    nr = nf - nc
    fronts, expect = [], []
    for seed in (3, 4):
        a = dense_spd(nf, seed)
        L11 = np.linalg.cholesky(a[:nc, :nc])
        L21 = np.linalg.solve(L11, a[nc:, :nc].T).T
        expect.append((np.vstack([L11, L21]), np.tril(a[nc:, nc:] - L21 @ L21.T)))
        fronts.append(a)
    buf = np.zeros(2 * (nf * nc + nr * nr))
    poff, uoff = [], []
    off = 0
    for a in fronts:
        poff.append(off)
        buf[off:off + nf * nc] = np.tril(a[:, :nc]).ravel(order="F")
        off += nf * nc
        uoff.append(off)
        buf[off:off + nr * nr] = np.tril(a[nc:, nc:]).ravel(order="F")
        off += nr * nr
    t = torch.from_numpy(buf).cuda()
    assert H.factor_fronts_noalloc(t, poff, uoff, [nf, nf], [nc, nc]) == 0
    out = t.cpu().numpy()
    for i, (lp, schur) in enumerate(expect):
        p = np.tril(out[poff[i]:poff[i] + nf * nc].reshape(nf, nc, order="F"))
        u = np.tril(out[uoff[i]:uoff[i] + nr * nr].reshape(nr, nr, order="F"))
        assert np.abs(p - lp).max() <= FACTOR_TOL * np.abs(lp).max()
        assert np.abs(u - schur).max() <= 1e-11 * np.abs(schur).max()
    with pytest.raises(H.MfdError):
        H.factor_fronts_noalloc(t, [0] * 9, [0] * 9, [4] * 9, [4] * 9)


def test_noalloc_reports_the_failing_front():
    """Two fronts in one call, the second not positive definite at its column
    38: the per-front info names that front and column, and the first front's
    factor is still exact."""
    import torch
    nf = nc = 200
    good = dense_spd(nf, 21)
    bad = dense_spd(nf, 22)
    bad[37, 37] = -100.0                                 # pivots 1..37 are unchanged, pivot 38 fails
    buf = np.concatenate([np.tril(good).ravel(order="F"), np.tril(bad).ravel(order="F")])
    t = torch.from_numpy(buf.copy()).cuda()
    info = H.factor_fronts_noalloc(t, [0, nf * nc], [0, 0], [nf, nf], [nc, nc], per_front=True)
    assert info == [0, 38], info
    got = np.tril(t.cpu().numpy()[:nf * nc].reshape(nf, nc, order="F"))
    ref = np.linalg.cholesky(good)
    assert np.abs(got - ref).max() <= FACTOR_TOL * np.abs(ref).max()
    # the next call starts from cleared info slots
    t2 = torch.from_numpy(np.tril(good).ravel(order="F").copy()).cuda()
    assert H.factor_fronts_noalloc(t2, [0], [0], [nf], [nf], per_front=True) == [0]


def test_noalloc_refuses_a_capturing_stream():
    """A call on a stream that is being captured into a CUDA graph returns
    MFD_E_ARG and issues nothing: its host table copy and info read-back cannot
    be recorded.  The capture around it still completes (the graph replays the
    one op captured beside the call), the front is untouched, and the next call
    outside the capture factors it."""
    import torch
    n = 64
    a = dense_spd(n, 5)
    host = np.tril(a).ravel(order="F").copy()
    t = torch.from_numpy(host.copy()).cuda()
    z = torch.zeros(4, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        z.add_(1.0)
        with pytest.raises(H.MfdError) as e:
            H.factor_fronts_noalloc(t, [0], [0], [n], [n], stream=s.cuda_stream)
    assert e.value.code == -1                            # MFD_E_ARG
    g.replay()
    torch.cuda.synchronize()
    assert z.cpu().tolist() == [1.0] * 4
    assert np.array_equal(t.cpu().numpy(), host)
    assert H.factor_fronts_noalloc(t, [0], [0], [n], [n]) == 0
    got = np.tril(t.cpu().numpy().reshape(n, n, order="F"))
    ref = np.linalg.cholesky(a)
    assert np.abs(got - ref).max() <= FACTOR_TOL * np.abs(ref).max()
