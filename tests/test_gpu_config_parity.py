"""GPU parity at the benchmark configurations' own sizes.

Each case runs the CUDA path through the C ABI on the full-size synthetic
workload and compares it with the oracle (the CPU restatement of the
reference's numeric phase) on the same inputs:

* 3D 7-point Laplacian 64^3 (n = 262,144): every device-built index map
  (local_index, supernodal_index, the six block_local_index arrays at the
  reference's test tile size nb = 10) and the symbolic arrays bit-exact; cost
  and nnz(L) equal; FP64 and FP32 + FP64-refinement solutions against the
  oracle's FP64 solve.
* 3D Q1 elasticity, 40^3 elements, 3 dofs per node (n = 201,720), 64
  right-hand sides: every column against the oracle's FP64 solve, FP64 and
  FP32 + refinement.
* 2,000 uneven 2D systems (sides 16..128): bit-exact per-system index maps for
  all 2,000 systems; solutions of a fixed sample of 50 systems (the largest
  among them) against the oracle, FP64 and FP32 + refinement.
* 3D variable-coefficient diffusion 80^3 (n = 512,000, condition number up
  to ~1e8): FP32 + refinement and FP64 against the oracle's FP64 solve.

Tolerances (written here, used below):
  X_TOL_FP64  ||x - x_oracle||_inf / ||x_oracle||_inf for two FP64 solves that
              differ only in summation order (the oracle against itself with
              another tile size differs by ~1e-14 on these systems)
  X_TOL_IR    the same for the FP32 factor refined in FP64 to backward error
              <= 1e-12: the forward difference is bounded by about cond(A) x
              (backward errors of both solutions)
  X_TOL_IR_DIFF  the same for the 80^3 diffusion problem, whose condition
              number reaches ~1e8
  BWD_TOL     normwise backward error ||b - Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf)
"""
import os

import numpy as np
import pytest

from mfdag import hppllt as H
from mfdag import problems as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

X_TOL_FP64 = 1e-10
X_TOL_IR = 1e-8
X_TOL_IR_DIFF = 1e-6
BWD_TOL = 1e-12
CORES = os.cpu_count() or 1
INDEX_IDS = [H.LOCAL_INDEX, H.SUPERNODAL_INDEX, H.BLI_NODE_PTR, H.BLI_BLOCK_PTR, H.BLI_PARENT, H.BLI_CHILD,
             H.BLI_VAL, H.BLI_OFFSET]
ORACLE_IDS = [O.LOCAL, O.SIDX, O.BLI_NODE_PTR, O.BLI_BLOCK_PTR, O.BLI_PARENT, O.BLI_CHILD, O.BLI_VAL, O.BLI_OFFSET]


def rel(x, xo):
    return float(np.abs(x - xo).max() / np.abs(xo).max())


def oracle_solution(p, max_zero, nb=128):
    """The oracle's FP64 factorization (all host threads) and solve of every column."""
    O.use_system_blas(True)
    o = O.Oracle.analyze(p.n, p.col, p.row, nb=nb, max_zero=max_zero, order_perm=p.order)
    assert o.factorize(p.val, nthreads=CORES) == 0
    B = p.rhs if p.rhs.ndim == 2 else p.rhs[:, None]
    return o, o.solve_many(B)


def gpu_solution(p, max_zero, precision):
    s = H.Solver.analyze(p.n, p.col, p.row, p.order, max_zero=max_zero, nb=10, precision=precision)
    assert s.factorize(p.val) == 0
    X = np.asfortranarray(p.rhs if p.rhs.ndim == 2 else p.rhs[:, None]).copy(order="F")
    rep, rc = s.solve(X if X.shape[1] > 1 else X[:, 0])
    assert rc == 0, rc
    return s, X, rep


def check_columns(p, X, XO, xtol):
    B = p.rhs if p.rhs.ndim == 2 else p.rhs[:, None]
    worst_x, worst_b = 0.0, 0.0
    for r in range(B.shape[1]):
        worst_x = max(worst_x, rel(X[:, r], XO[:, r]))
        worst_b = max(worst_b, P.backward_error(p.n, p.col, p.row, p.val, X[:, r], B[:, r]))
    assert worst_x <= xtol, worst_x
    assert worst_b <= BWD_TOL, worst_b
    return worst_x, worst_b


def check_index_maps(s, o, system=0):
    for hid, oid in zip(INDEX_IDS, ORACLE_IDS):
        assert np.array_equal(s.index(hid, system), o.get(oid)), (system, hid)


# ---------------------------------------------------------------------------
# 3D 7-point Laplacian 64^3
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def lap3d64():
    p = P.laplace3d(64, 1)
    o, XO = oracle_solution(p, 1000)
    return p, o, XO


def test_lap3d64_index_and_symbolic_bit_exact():
    p = P.laplace3d(64, 1)
    s = H.Solver.analyze(p.n, p.col, p.row, p.order, max_zero=1000, nb=10)
    o = O.Oracle.analyze(p.n, p.col, p.row, nb=10, max_zero=1000, order_perm=p.order)
    check_index_maps(s, o)
    sym = o.symbolic()
    for hid, key in [(H.SYM_NODE_PTR, "node_ptr"), (H.SYM_PARENT, "parent"), (H.SYM_LPTR, "lptr"),
                     (H.SYM_LROW, "lrow"), (H.SYM_PERM, "perm")]:
        assert np.array_equal(s.symbolic(hid), sym[key]), key
    st = s.stats()
    assert st.cost == o.cost() and st.nonzero == o.nonzero()
    assert st.max_front > 4000                               # the top separator fronts of this size


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32ir"])
def test_lap3d64_solution_against_oracle(lap3d64, precision):
    p, o, XO = lap3d64
    s, X, rep = gpu_solution(p, 1000, precision)
    check_columns(p, X, XO, X_TOL_FP64 if precision == 0 else X_TOL_IR)
    assert rep.backward_error <= BWD_TOL
    if precision == 1:
        assert rep.converged == 1 and rep.iterations <= 3


# ---------------------------------------------------------------------------
# 3D Q1 hex elasticity, 40^3 elements, 64 right-hand sides
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def elast40():
    p = P.elasticity3d(40, 4, 64)
    o, XO = oracle_solution(p, 1000)
    return p, o, XO


def test_elasticity_structure():
    p = P.elasticity3d(40, 4, 64)
    assert p.n == 201720 and p.rhs.shape == (p.n, 64)
    s = H.Solver.analyze(p.n, p.col, p.row, p.order, max_zero=1000, nb=10)
    o = O.Oracle.analyze(p.n, p.col, p.row, nb=10, max_zero=1000, order_perm=p.order)
    check_index_maps(s, o)
    assert s.stats().cost == o.cost() and s.stats().nonzero == o.nonzero()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32ir"])
def test_elasticity_64rhs_every_column(elast40, precision):
    p, o, XO = elast40
    s, X, rep = gpu_solution(p, 1000, precision)
    check_columns(p, X, XO, X_TOL_FP64 if precision == 0 else X_TOL_IR)
    if precision == 1:
        assert rep.converged == 1


# ---------------------------------------------------------------------------
# 2,000 uneven 2D systems
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def batch2000():
    systems = P.laplace2d_batch(2000, 3)
    return systems


def batch_solver(systems, precision):
    s = H.Solver.analyze_batch([(q.n, q.col, q.row, q.order) for q in systems], max_zero=100, nb=10,
                               precision=precision)
    assert s.factorize(np.concatenate([q.val for q in systems])) == 0
    return s


def test_batch2000_index_maps_every_system(batch2000):
    systems = batch2000
    s = H.Solver.analyze_batch([(q.n, q.col, q.row, q.order) for q in systems], max_zero=100, nb=10)
    cost = 0
    for i, q in enumerate(systems):
        o = O.Oracle.analyze(q.n, q.col, q.row, nb=10, max_zero=100, order_perm=q.order)
        check_index_maps(s, o, i)
        cost += o.cost()
    assert s.stats().cost == cost


def sample_ids(systems, k=50):
    sizes = np.array([q.n for q in systems])
    rng = np.random.default_rng(2024)
    ids = set(rng.choice(len(systems), k - 2, replace=False).tolist())
    ids.add(int(np.argmax(sizes)))
    ids.add(int(np.argmin(sizes)))
    return sorted(ids)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32ir"])
def test_batch2000_solutions_sample(batch2000, precision):
    systems = batch2000
    s = batch_solver(systems, precision)
    b = np.concatenate([q.rhs for q in systems])
    x = b.copy()
    rep, rc = s.solve(x)
    assert rc == 0 and rep.backward_error <= BWD_TOL
    offs = np.concatenate([[0], np.cumsum([q.n for q in systems])])
    O.use_system_blas(True)
    tol = X_TOL_FP64 if precision == 0 else X_TOL_IR
    for i in sample_ids(systems):
        q = systems[i]
        o = O.Oracle.analyze(q.n, q.col, q.row, nb=10, max_zero=100, order_perm=q.order)
        assert o.factorize(q.val) == 0
        xo = o.solve(q.rhs)
        xi = x[offs[i]:offs[i + 1]]
        assert rel(xi, xo) <= tol, (i, rel(xi, xo))
        assert P.backward_error(q.n, q.col, q.row, q.val, xi, q.rhs) <= BWD_TOL, i


# ---------------------------------------------------------------------------
# 3D variable-coefficient diffusion 80^3
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def diff80():
    p = P.diffusion3d(80, 2)
    o, XO = oracle_solution(p, 1000)
    return p, o, XO


@pytest.mark.parametrize("precision", [1, 0], ids=["fp32ir", "fp64"])
def test_diffusion80_against_oracle(diff80, precision):
    p, o, XO = diff80
    s, X, rep = gpu_solution(p, 1000, precision)
    check_columns(p, X, XO, X_TOL_FP64 if precision == 0 else X_TOL_IR_DIFF)
    if precision == 1:
        assert rep.converged == 1
    assert s.stats().cost == o.cost()
