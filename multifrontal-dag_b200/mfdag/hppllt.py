"""Python side of the C ABI in include/mfdag.h (ctypes over libmfdag.so).

Two layers, as in the header:

* ``hppllt_init / hppllt_analyze / hppllt_factorize / hppllt_solve /
  hppllt_finalize / hppllt_get_*`` -- the reference's public API
  (src/main/hppllt.f90:8-9) with its names, argument meaning and single
  module-global instance.
* ``Solver`` -- the handle API (mfd_*), used for batches, multiple right-hand
  sides, device pointers and statistics.

The shared library is built in-tree (multifrontal-dag_b200/build.py).  There is
no CPU fallback: if the library cannot be loaded or no CUDA device is present,
every numeric call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmfdag.so")

MFD_PREC_FP64 = 0
MFD_PREC_FP32_IR = 1

I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class Options(C.Structure):
    _fields_ = [("nb", C.c_int32), ("max_zero", C.c_int32), ("precision", C.c_int32), ("ir_max_iter", C.c_int32),
                ("ir_tol", C.c_double), ("use_graph", C.c_int32), ("device", C.c_int32),
                ("small_front_max", C.c_int32), ("panel_width", C.c_int32), ("reserved", C.c_int32 * 7)]


class Symbolic(C.Structure):
    _fields_ = [("n", C.c_int32), ("nnz", C.c_int32), ("num_node", C.c_int32),
                ("node_ptr", C.c_void_p), ("parent", C.c_void_p), ("lrow_ptr", C.c_void_p), ("lrow", C.c_void_p),
                ("acol_ptr", C.c_void_p), ("arow", C.c_void_p), ("ccs_perm", C.c_void_p), ("perm", C.c_void_p)]


class Coo(C.Structure):
    _fields_ = [("n", C.c_int32), ("nnz", C.c_int64), ("row", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p)]


class Report(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("backward_error", C.c_double),
                ("residual_ref", C.c_double), ("time_ms", C.c_double)]


class KernelProfile(C.Structure):
    _fields_ = [("launches", C.c_int64), ("ms", C.c_double), ("flops", C.c_double), ("bytes", C.c_double)]


KERNEL_CLASSES = ["small_front", "zero", "assemble", "extend_add", "panel", "update", "solve_small", "solve_large",
                  "other", "trsm"]


class Stats(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz_a", C.c_int64), ("num_front", C.c_int64), ("num_level", C.c_int64),
                ("cost", C.c_int64), ("nonzero", C.c_int64), ("panel_bytes", C.c_int64),
                ("update_pool_bytes", C.c_int64), ("launches_factor", C.c_int64), ("launches_solve", C.c_int64),
                ("max_front", C.c_int64), ("factor_ms", C.c_double), ("solve_ms", C.c_double),
                ("time_info", C.c_double * 7), ("pivot_fallbacks", C.c_int64), ("setup_s", C.c_double * 4)]


EXPORTS = [
    "mfd_default_options", "mfd_create", "mfd_create_batch", "mfd_analyze", "mfd_analyze_batch", "mfd_factorize",
    "mfd_autotune",
    "mfd_solve", "mfd_factorize_solve", "mfd_get_stats", "mfd_get_index", "mfd_get_symbolic", "mfd_get_front_panel",
    "mfd_destroy", "mfd_last_error", "mfd_set_profiling", "mfd_get_profile", "mfd_test_expire_waits",
    "mfd_factor_fronts_noalloc",
    "mfd_noalloc_last_error", "mfd_symbolic_analyze", "mfd_symbolic_view", "mfd_symbolic_free", "mfd_mm_read",
    "mfd_coo_free", "mfd_coo_to_ccs", "mfd_analyze_csr", "mfd_order", "mfd_subtree_partition", "hppllt_init", "hppllt_set_precision", "hppllt_analyze",
    "hppllt_set_ordering",
    "hppllt_factorize", "hppllt_solve", "hppllt_finalize", "hppllt_get_time_info", "hppllt_get_cost",
    "hppllt_get_nonzero", "hppllt_get_array_size",
]

_lib = None


class MfdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mfdag error {code}: {msg}")
        self.code = code


def load(build_if_missing: bool = True):
    """Load libmfdag.so (building it with nvcc if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) and build_if_missing:
        import importlib.util
        spec = importlib.util.spec_from_file_location("mfdag_build", os.path.join(os.path.dirname(_HERE), "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    L = C.CDLL(LIB_PATH)
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    L.mfd_default_options.argtypes = [C.POINTER(Options)]
    L.mfd_create.argtypes = [C.POINTER(vp), C.POINTER(Symbolic), C.POINTER(Options)]
    L.mfd_create_batch.argtypes = [C.POINTER(vp), i32, C.POINTER(Symbolic), C.POINTER(Options)]
    L.mfd_analyze.argtypes = [C.POINTER(vp), i32, vp, vp, vp, C.POINTER(Options)]
    L.mfd_analyze_batch.argtypes = [C.POINTER(vp), i32, vp, vp, vp, vp, C.POINTER(Options)]
    L.mfd_factorize.argtypes = [vp, vp]
    L.mfd_solve.argtypes = [vp, vp, i32, i64, C.POINTER(Report)]
    L.mfd_factorize_solve.argtypes = [vp, vp, vp, i32, i64, C.POINTER(Report)]
    L.mfd_get_stats.argtypes = [vp, C.POINTER(Stats)]
    L.mfd_autotune.argtypes = [vp, vp, i32, C.POINTER(Options), C.POINTER(C.c_double)]
    L.mfd_get_index.restype = i64
    L.mfd_get_index.argtypes = [vp, i32, i32, vp]
    L.mfd_get_symbolic.restype = i64
    L.mfd_get_symbolic.argtypes = [vp, i32, i32, vp]
    L.mfd_get_front_panel.restype = i64
    L.mfd_get_front_panel.argtypes = [vp, i32, i32, vp]
    L.mfd_destroy.argtypes = [vp]
    L.mfd_factor_fronts_noalloc.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp]
    L.mfd_noalloc_last_error.restype = C.c_char_p
    L.mfd_set_profiling.argtypes = [vp, i32]
    L.mfd_get_profile.argtypes = [vp, i32, C.POINTER(KernelProfile)]
    L.mfd_test_expire_waits.argtypes = [vp, i32]
    L.mfd_symbolic_analyze.argtypes = [C.POINTER(vp), i32, vp, vp, vp, i32]
    L.mfd_symbolic_view.argtypes = [vp, C.POINTER(Symbolic)]
    L.mfd_symbolic_free.argtypes = [vp]
    L.mfd_last_error.restype = C.c_char_p
    L.mfd_mm_read.argtypes = [C.c_char_p, C.POINTER(Coo)]
    L.mfd_coo_free.argtypes = [C.POINTER(Coo)]
    L.mfd_coo_free.restype = None
    L.mfd_coo_to_ccs.argtypes = [i32, i64, vp, vp, vp, vp, vp, vp, i32]
    L.mfd_analyze_csr.argtypes = [C.POINTER(vp), i32, vp, vp, i32, vp, C.POINTER(Options)]
    L.mfd_order.argtypes = [i32, vp, vp, vp]
    L.mfd_subtree_partition.argtypes = [i32, vp, vp, vp, vp, C.c_double, i32, vp, vp]
    L.hppllt_init.argtypes = [vp, i32]
    L.hppllt_set_precision.argtypes = [i32]
    L.hppllt_analyze.argtypes = [vp, vp, i32]
    L.hppllt_set_ordering.argtypes = [vp, i32]
    L.hppllt_factorize.argtypes = [vp]
    L.hppllt_solve.argtypes = [vp]
    L.hppllt_get_time_info.restype = C.c_double
    L.hppllt_get_time_info.argtypes = [i32]
    L.hppllt_get_cost.restype = i64
    L.hppllt_get_nonzero.restype = i64
    L.hppllt_get_array_size.restype = i64
    L.hppllt_get_array_size.argtypes = [i32]
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise MfdError(rc, load().mfd_last_error().decode())


def _ptr(a) -> int:
    """Address of a numpy array or of a torch tensor's device storage."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def symbolic_analyze(n, ccs_col, ccs_row, order_perm=None, max_zero=10) -> dict:
    """Host-only symbolic analysis (no device needed): the reference's symbolic
    arrays after hppllt_analyze, as 1-based int32 numpy arrays."""
    L = load()
    col, row = _i32(ccs_col), _i32(ccs_row)
    op = _i32(order_perm) if order_perm is not None else None
    a = C.c_void_p()
    _check(L.mfd_symbolic_analyze(C.byref(a), int(n), col.ctypes.data, row.ctypes.data,
                                  op.ctypes.data if op is not None else None, int(max_zero)))
    try:
        v = Symbolic()
        _check(L.mfd_symbolic_view(a, C.byref(v)))

        def arr(ptr, cnt):
            if cnt <= 0:
                return np.zeros(0, np.int32)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(cnt,)).copy()

        nn = v.num_node
        lptr = arr(v.lrow_ptr, nn + 1)
        return {"n": v.n, "nnz": v.nnz, "num_node": nn, "node_ptr": arr(v.node_ptr, nn + 1),
                "parent": arr(v.parent, nn), "lptr": lptr, "lrow": arr(v.lrow, int(lptr[-1]) - 1),
                "aptr": arr(v.acol_ptr, v.n + 1), "arow": arr(v.arow, v.nnz), "ccs_perm": arr(v.ccs_perm, v.nnz),
                "perm": arr(v.perm, v.n)}
    finally:
        L.mfd_symbolic_free(a)


def order(n, ccs_col, ccs_row) -> np.ndarray:
    """Nested-dissection ordering of the lower CCS (mfd_order): new -> old, 1-based."""
    col, row = _i32(ccs_col), _i32(ccs_row)
    out = np.zeros(int(n), np.int32)
    _check(load().mfd_order(int(n), col.ctypes.data, row.ctypes.data, out.ctypes.data))
    return out


def subtree_partition(node_size, cc, num_child, child, tol: float, p: int) -> list:
    """Subtree roots (1-based, the reference's list order) for p workers (mfd_subtree_partition)."""
    ns, c, nch = _i32(node_size), _i32(cc), _i32(num_child)
    ch = _i32(child) if len(child) else np.zeros(1, np.int32)
    roots = np.zeros(max(1, ns.size), np.int32)
    cnt = np.zeros(1, np.int32)
    _check(load().mfd_subtree_partition(int(ns.size), ns.ctypes.data, c.ctypes.data, nch.ctypes.data, ch.ctypes.data,
                                        float(tol), int(p), roots.ctypes.data, cnt.ctypes.data))
    return roots[:int(cnt[0])].tolist()


def tree_of(sym: dict):
    """(node_size, cc, num_child, child) of an analysed system's supernodal tree
    (children ascending, as the reference's tree_child)."""
    nn = int(sym["num_node"])
    node_size = np.diff(sym["node_ptr"]).astype(np.int32)
    cc = np.diff(sym["lptr"]).astype(np.int32)
    parent = np.asarray(sym["parent"])
    num_child = np.bincount(parent[parent > 0] - 1, minlength=nn).astype(np.int32)
    child = (np.argsort(parent, kind="stable")[np.sum(parent == 0):] + 1).astype(np.int32)
    return node_size, cc, num_child, child


def mm_read(path) -> dict:
    """Matrix Market coordinate file (mfd_mm_read): {"n", "row", "col", "val"}, 1-based."""
    L = load()
    coo = Coo()
    _check(L.mfd_mm_read(os.fsencode(path), C.byref(coo)))
    try:
        k = int(coo.nnz)

        def arr(ptr, ct):
            if k == 0:
                return np.zeros(0, np.dtype(ct))
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(k,)).copy()

        return {"n": int(coo.n), "row": arr(coo.row, C.c_int32), "col": arr(coo.col, C.c_int32),
                "val": arr(coo.val, C.c_double)}
    finally:
        L.mfd_coo_free(C.byref(coo))


def coo_to_ccs(n, row, col, val=None, device: int = 0):
    """COO -> lower CCS on the GPU (mfd_coo_to_ccs): (ccs_col, ccs_row, ccs_val or None).
    Host numpy inputs give host outputs; CUDA tensors give CUDA tensors."""
    L = load()
    if hasattr(row, "data_ptr"):
        import torch
        nnz = int(row.numel())
        ptr = torch.empty(int(n) + 1, dtype=torch.int32, device=row.device)
        r = torch.empty(max(nnz, 1), dtype=torch.int32, device=row.device)
        v = torch.empty(max(nnz, 1), dtype=torch.float64, device=row.device) if val is not None else None
        _check(L.mfd_coo_to_ccs(int(n), nnz, row.data_ptr(), col.data_ptr(), val.data_ptr() if val is not None else None,
                                ptr.data_ptr(), r.data_ptr(), v.data_ptr() if v is not None else None, int(device)))
        return ptr, r[:nnz], (v[:nnz] if v is not None else None)
    row, col = _i32(row), _i32(col)
    nnz = int(row.size)
    ptr = np.zeros(int(n) + 1, np.int32)
    r = np.zeros(max(nnz, 1), np.int32)
    vv = np.ascontiguousarray(val, dtype=np.float64) if val is not None else None
    out = np.zeros(max(nnz, 1), np.float64) if val is not None else None
    _check(L.mfd_coo_to_ccs(int(n), nnz, row.ctypes.data, col.ctypes.data, vv.ctypes.data if vv is not None else None,
                            ptr.ctypes.data, r.ctypes.data, out.ctypes.data if out is not None else None, int(device)))
    return ptr, r[:nnz], (out[:nnz] if out is not None else None)


def default_options(**kw) -> Options:
    o = Options()
    load().mfd_default_options(C.byref(o))
    for k, v in kw.items():
        if k == "reserved":
            for i, x in enumerate(v):
                o.reserved[i] = int(x)
        else:
            setattr(o, k, v)
    return o


def _i32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


class Solver:
    """One handle: an analysed system (or batch) with its device-resident plan."""

    def __init__(self, handle, n_total: int, keep=()):
        self._h = handle
        self.n = n_total
        self._keep = keep

    # ---- construction -----------------------------------------------------
    @classmethod
    def analyze(cls, n, ccs_col, ccs_row, order_perm=None, **opts) -> "Solver":
        L = load()
        o = default_options(**opts)
        col, row = _i32(ccs_col), _i32(ccs_row)
        op = _i32(order_perm) if order_perm is not None else None
        h = C.c_void_p()
        _check(L.mfd_analyze(C.byref(h), int(n), col.ctypes.data, row.ctypes.data,
                             op.ctypes.data if op is not None else None, C.byref(o)))
        return cls(h, int(n))

    @classmethod
    def analyze_csr(cls, n, csr_ptr, csr_col, base: int = 0, order_perm=None, **opts) -> "Solver":
        """Symmetric matrix given as the CSR of its lower triangle or of the whole
        matrix (mfd_analyze_csr); factorize() then takes values in CSR order."""
        L = load()
        o = default_options(**opts)
        ptr, col = _i32(csr_ptr), _i32(csr_col)
        op = _i32(order_perm) if order_perm is not None else None
        h = C.c_void_p()
        _check(L.mfd_analyze_csr(C.byref(h), int(n), ptr.ctypes.data, col.ctypes.data, int(base),
                                 op.ctypes.data if op is not None else None, C.byref(o)))
        return cls(h, int(n))

    @classmethod
    def analyze_batch(cls, problems, **opts) -> "Solver":
        """problems: sequence of (n, ccs_col, ccs_row, order_perm or None)."""
        L = load()
        o = default_options(**opts)
        k = len(problems)
        cols = [_i32(p[1]) for p in problems]
        rows = [_i32(p[2]) for p in problems]
        ords = [(_i32(p[3]) if p[3] is not None else None) for p in problems]
        ns = np.array([p[0] for p in problems], dtype=np.int32)
        pc = (C.c_void_p * k)(*[c.ctypes.data for c in cols])
        pr = (C.c_void_p * k)(*[r.ctypes.data for r in rows])
        po = (C.c_void_p * k)(*[(x.ctypes.data if x is not None else None) for x in ords])
        h = C.c_void_p()
        _check(L.mfd_analyze_batch(C.byref(h), k, ns.ctypes.data, C.cast(pc, C.c_void_p), C.cast(pr, C.c_void_p),
                                   C.cast(po, C.c_void_p) if any(x is not None for x in ords) else None, C.byref(o)))
        return cls(h, int(ns.sum()))

    @classmethod
    def from_symbolic(cls, sym: dict, **opts) -> "Solver":
        """Create from the reference's symbolic arrays (keys as in mfd_symbolic)."""
        L = load()
        o = default_options(**opts)
        arrs = {k: _i32(sym[k]) for k in ("node_ptr", "parent", "lptr", "lrow", "aptr", "arow", "ccs_perm", "perm")}
        s = Symbolic(int(sym["n"]), int(sym["nnz"]), int(sym["num_node"]),
                     arrs["node_ptr"].ctypes.data, arrs["parent"].ctypes.data, arrs["lptr"].ctypes.data,
                     arrs["lrow"].ctypes.data if arrs["lrow"].size else arrs["lptr"].ctypes.data,
                     arrs["aptr"].ctypes.data, arrs["arow"].ctypes.data, arrs["ccs_perm"].ctypes.data,
                     arrs["perm"].ctypes.data)
        h = C.c_void_p()
        _check(L.mfd_create(C.byref(h), C.byref(s), C.byref(o)))
        return cls(h, int(sym["n"]))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            load().mfd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- numeric --------------------------------------------------------------
    def factorize(self, a) -> int:
        """a: float64 values (numpy host array or torch CUDA tensor). Returns info (0 ok)."""
        if isinstance(a, np.ndarray):
            a = np.ascontiguousarray(a, dtype=np.float64)
        rc = load().mfd_factorize(self._h, _ptr(a))
        if rc > 0:
            return rc
        _check(rc)
        return 0

    def solve(self, b, report: bool = True, nrhs: int | None = None):
        """Solve in place.  b holds nrhs column-major right-hand sides of length
        n: a numpy array (n,) or Fortran-ordered (n, nrhs), or a float64 tensor
        (host or CUDA) whose storage is that column-major block -- a contiguous
        (nrhs, n) tensor, or (n,) with nrhs = 1.  ``nrhs`` overrides the count
        read from the shape."""
        rep = Report()
        if isinstance(b, np.ndarray):
            if b.dtype != np.float64 or not (b.flags.f_contiguous or b.ndim == 1):
                raise ValueError("b must be float64, 1-D or Fortran ordered")
            k = 1 if b.ndim == 1 else b.shape[1]
            size = b.size
        else:
            if not b.is_contiguous():
                raise ValueError("tensor right-hand sides must be contiguous (nrhs, n) storage")
            k = 1 if b.dim() == 1 else (b.shape[0] if b.shape[-1] == self.n else b.shape[1])
            size = b.numel()
        nrhs = k if nrhs is None else int(nrhs)
        if nrhs < 1 or size != nrhs * self.n:
            raise ValueError(f"right-hand side holds {size} values, expected {nrhs} x {self.n}")
        rc = load().mfd_solve(self._h, _ptr(b), int(nrhs), int(self.n), C.byref(rep) if report else None)
        if rc not in (0, -5):
            _check(rc)
        return rep, rc

    def autotune(self, a, repeats: int = 3):
        """Time the factorization of `a` under the candidate schedule settings
        (mfd_autotune) and return (options dict for Solver.analyze, factor ms)."""
        if isinstance(a, np.ndarray):
            a = np.ascontiguousarray(a, dtype=np.float64)
        best = Options()
        ms = C.c_double()
        rc = load().mfd_autotune(self._h, _ptr(a), int(repeats), C.byref(best), C.byref(ms))
        if rc > 0:
            raise MfdError(rc, "matrix is not positive definite")
        _check(rc)
        return {"small_front_max": best.small_front_max, "reserved": tuple(best.reserved)}, ms.value

    def stats(self) -> Stats:
        st = Stats()
        _check(load().mfd_get_stats(self._h, C.byref(st)))
        return st

    def set_profiling(self, enable: bool) -> None:
        _check(load().mfd_set_profiling(self._h, 1 if enable else 0))

    def test_expire_waits(self, enable: bool) -> None:
        """Make the tensor-core update's first wait run out (mfd_test_expire_waits)."""
        _check(load().mfd_test_expire_waits(self._h, 1 if enable else 0))

    def profile(self) -> dict:
        out = {}
        for k, name in enumerate(KERNEL_CLASSES):
            p = KernelProfile()
            _check(load().mfd_get_profile(self._h, k, C.byref(p)))
            out[name] = {"launches": p.launches, "ms": p.ms, "flops": p.flops, "bytes": p.bytes}
        return out

    def index(self, which: int, system: int = 0) -> np.ndarray:
        L = load()
        n = L.mfd_get_index(self._h, system, which, None)
        if n < 0:
            _check(n)
        out = np.zeros(max(n, 1), np.int32)
        L.mfd_get_index(self._h, system, which, out.ctypes.data)
        return out[:n]

    def symbolic(self, which: int, system: int = 0) -> np.ndarray:
        L = load()
        n = L.mfd_get_symbolic(self._h, system, which, None)
        if n < 0:
            _check(n)
        out = np.zeros(max(n, 1), np.int32)
        L.mfd_get_symbolic(self._h, system, which, out.ctypes.data)
        return out[:n]

    def front_panel(self, node: int, system: int = 0) -> np.ndarray:
        L = load()
        n = L.mfd_get_front_panel(self._h, system, node, None)
        if n < 0:
            _check(n)
        out = np.zeros(max(n, 1), np.float64)
        rc = L.mfd_get_front_panel(self._h, system, node, out.ctypes.data)
        if rc < 0:
            _check(rc)
        return out[:n]


NOALLOC_MAX_FRONTS = 8


def factor_fronts_noalloc(fronts, panel_off, update_off, nf, nc, stream=None, per_front=False):
    """Partial Cholesky of dense fronts held in one caller-owned device buffer
    (a float64 CUDA tensor), without any device allocation (see
    mfd_factor_fronts_noalloc in include/mfdag.h).  Returns info: per front
    (a list, 0 or the front's 1-based bad-pivot column) with per_front=True,
    else the first nonzero entry of that list (0 if none)."""
    L = load()
    po = np.ascontiguousarray(panel_off, dtype=np.int64)
    uo = np.ascontiguousarray(update_off, dtype=np.int64)
    f = _i32(nf)
    c = _i32(nc)
    info = np.zeros(max(1, len(f)), np.int32)
    rc = L.mfd_factor_fronts_noalloc(_ptr(fronts), int(len(f)), po.ctypes.data, uo.ctypes.data, f.ctypes.data,
                                     c.ctypes.data, info.ctypes.data, stream)
    if rc != 0:
        raise MfdError(rc, L.mfd_noalloc_last_error().decode())
    if per_front:
        return [int(v) for v in info[:len(f)]]
    bad = [int(v) for v in info[:len(f)] if v]
    return bad[0] if bad else 0


# index ids of mfd_get_index
LOCAL_INDEX, SUPERNODAL_INDEX, BLI_NODE_PTR, BLI_BLOCK_PTR, BLI_PARENT, BLI_CHILD, BLI_VAL, BLI_OFFSET = range(1, 9)
# symbolic ids of mfd_get_symbolic
SYM_NODE_PTR, SYM_PARENT, SYM_LPTR, SYM_LROW, SYM_APTR, SYM_AROW, SYM_CCS_PERM, SYM_PERM = range(1, 9)


# ---------------------------------------------------------------------------
# the reference's API (hppllt.f90), module-global single instance
# ---------------------------------------------------------------------------
_keep = {}


def hppllt_init(options) -> None:
    opts = _i32(options)
    _keep["options"] = opts
    load().hppllt_init(opts.ctypes.data, int(opts.size))


def hppllt_set_precision(precision: int) -> None:
    load().hppllt_set_precision(int(precision))


def hppllt_set_ordering(order_perm) -> None:
    op = _i32(order_perm)
    _keep["order"] = op
    load().hppllt_set_ordering(op.ctypes.data, int(op.size))


def hppllt_analyze(ccs_col, ccs_row, n) -> None:
    col, row = _i32(ccs_col), _i32(ccs_row)
    _check(load().hppllt_analyze(col.ctypes.data, row.ctypes.data, int(n)))


def hppllt_factorize(a) -> int:
    a = np.ascontiguousarray(a, dtype=np.float64)
    rc = load().hppllt_factorize(a.ctypes.data)
    if rc < 0:
        _check(rc)
    return rc


def hppllt_solve(b: np.ndarray) -> None:
    if b.dtype != np.float64 or not b.flags.c_contiguous:
        raise ValueError("b must be a contiguous float64 array (solved in place)")
    _check(load().hppllt_solve(b.ctypes.data))


def hppllt_finalize() -> None:
    load().hppllt_finalize()


def hppllt_get_time_info(num: int) -> float:
    return float(load().hppllt_get_time_info(int(num)))


def hppllt_get_cost() -> int:
    return int(load().hppllt_get_cost())


def hppllt_get_nonzero() -> int:
    return int(load().hppllt_get_nonzero())


def hppllt_get_array_size(num: int) -> int:
    return int(load().hppllt_get_array_size(int(num)))
