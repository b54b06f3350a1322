"""Failure paths of the GPU numeric phase, injected without any GPU fault.

* A bounded device wait that runs out: mfd_test_expire_waits makes every CTA
  of the FP32 tensor-core trailing update wait on an mbarrier that nothing
  arrives at (a ~1 ms limit) before it issues any MMA.  The factorization must
  return MFD_E_TIMEOUT (-4), refuse a solve, and factor normally once the
  request is withdrawn, on the same handle.
* The same request makes the single-RHS large-front solve sweeps' flag waits
  run out: the solve returns MFD_E_TIMEOUT and the handle solves normally
  once the request is withdrawn.
* A non-positive pivot in the blocked large-front path and in the fused
  small-front path: the returned info is the pivot's 1-based column, the same
  column the oracle's LAPACK-convention check reports.
"""
import time

import numpy as np
import pytest

from mfdag import hppllt as H
from mfdag import problems as P

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_timeout_and_handle_recovers():
    p = P.laplace3d(16)
    s = H.Solver.analyze(p.n, p.col, p.row, p.order, max_zero=10, small_front_max=48,
                         precision=H.MFD_PREC_FP32_IR)
    assert s.factorize(p.val) == 0                      # the tensor-core update runs on this handle
    s.test_expire_waits(True)
    t0 = time.perf_counter()
    with pytest.raises(H.MfdError) as e:
        s.factorize(p.val)
    assert e.value.code == -4
    assert time.perf_counter() - t0 < 30.0              # every wait is bounded
    with pytest.raises(H.MfdError) as e2:
        s.solve(p.rhs.copy())
    assert e2.value.code == -6                          # no valid factor after the expiry
    s.test_expire_waits(False)
    assert s.factorize(p.val) == 0
    x = p.rhs.copy()
    rep, rc = s.solve(x)
    assert rc == 0 and rep.converged == 1
    assert P.backward_error(p.n, p.col, p.row, p.val, x, p.rhs) <= 1e-12


def test_expire_request_leaves_fp64_factor_alone():
    """In the factorization the request only concerns the FP32 tensor-core
    update: an FP64 handle factors normally with it set."""
    p = P.laplace3d(12)
    s = H.Solver.analyze(p.n, p.col, p.row, p.order, max_zero=10, small_front_max=48)
    s.test_expire_waits(True)
    assert s.factorize(p.val) == 0


@pytest.mark.parametrize("precision", [0, 1])
def test_expired_solve_wait_reports_timeout_and_handle_recovers(precision):
    """The single-RHS large-front solve sweeps (one launch per level, tasks
    waiting on other tasks' flags) under the request: their waits look for a
    value nothing writes and give up after ~1 ms; the solve returns
    MFD_E_TIMEOUT (-4) within seconds, and once the request is withdrawn the
    same handle, without refactoring, solves to backward error <= 1e-12."""
    p = P.laplace3d(16)
    s = H.Solver.analyze(p.n, p.col, p.row, p.order, max_zero=1000, small_front_max=48, precision=precision)
    assert s.factorize(p.val) == 0
    s.test_expire_waits(True)
    t0 = time.perf_counter()
    with pytest.raises(H.MfdError) as e:
        s.solve(p.rhs.copy())
    assert e.value.code == -4
    assert time.perf_counter() - t0 < 30.0              # every wait is bounded
    s.test_expire_waits(False)
    x = p.rhs.copy()
    rep, rc = s.solve(x)
    assert rc == 0
    assert P.backward_error(p.n, p.col, p.row, p.val, x, p.rhs) <= 1e-12


@pytest.mark.parametrize("small_max", [0, 48])
@pytest.mark.parametrize("precision", [0, 1])
def test_non_spd_pivot_column_matches_oracle(small_max, precision):
    """A negative diagonal entry at one column: the GPU reports the first
    non-positive pivot column in the permuted numbering, as the oracle does."""
    from oracle import oracle as O
    p = P.laplace3d(12)
    val = p.val.copy()
    diag_pos = p.col[:-1] - 1                          # diagonal entries come first in each column
    val[diag_pos[700]] = -50.0
    s = H.Solver.analyze(p.n, p.col, p.row, p.order, max_zero=10, small_front_max=small_max,
                         precision=precision)
    info = s.factorize(val)
    o = O.Oracle.analyze(p.n, p.col, p.row, nb=10, max_zero=10, order_perm=p.order)
    oinfo = o.factorize(val)
    assert info > 0 and oinfo > 0
    assert info == oinfo, (info, oinfo)
