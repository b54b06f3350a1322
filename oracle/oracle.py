"""ctypes front end of the CPU oracle (oracle/mfdag_oracle.c).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference solver's symbolic
analysis, index/layout layer and sequential FP64 numeric phase on the CPU.
tests/, the smoke check and bench.py's CPU-baseline leg use it as the checker;
the product never imports it.

All integer arrays are the reference's 1-based values (int32); dense values are
float64.  Function names follow the reference modules they restate.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
I64P = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")

# accessor ids (enum in mfdag_oracle.c)
NODE_SETS, PARENT, LPTR, LROW, APTR, AROW, CCS_PERM, PERM, SIDX, LOCAL = range(1, 11)
BLI_NODE_PTR, BLI_BLOCK_PTR, BLI_PARENT, BLI_CHILD, BLI_VAL, BLI_OFFSET = range(11, 17)
TREE_CHILD_PTR, TREE_CHILD = 17, 18


def build() -> str:
    """Compile the oracle with the committed Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
        os.path.join(_HERE, "mfdag_oracle.c")
    ):
        build()
    L = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    L.orc_analyze.restype = vp
    L.orc_analyze.argtypes = [C.c_int, I32P, I32P, C.c_int, C.c_int, vp]
    L.orc_from_internal.restype = vp
    L.orc_from_internal.argtypes = [C.c_int, I32P, I32P, I32P, I32P, C.c_int, I32P, I32P, C.c_int]
    L.orc_free.argtypes = [vp]
    L.orc_factorize.restype = C.c_int
    L.orc_factorize.argtypes = [vp, F64P]
    L.orc_factorize_parallel.restype = C.c_int
    L.orc_factorize_parallel.argtypes = [vp, F64P, C.c_int]
    L.orc_factorize_dag.restype = C.c_int
    L.orc_factorize_dag.argtypes = [vp, F64P, C.c_int]
    L.orc_solve.argtypes = [vp, F64P]
    L.orc_sweep.argtypes = [vp, F64P, C.c_int]
    L.orc_solve_many.argtypes = [vp, F64P, C.c_int, C.c_int64, C.c_int]
    L.orc_coo_to_ccs.argtypes = [C.c_int, C.c_int, I32P, I32P, F64P, I32P, I32P, F64P]
    L.orc_tree_pruning.restype = C.c_int
    L.orc_tree_pruning.argtypes = [C.c_int, I32P, I32P, I32P, I32P, C.c_double, C.c_int, I32P]
    L.orc_get_size.restype = C.c_int
    L.orc_get_size.argtypes = [vp, C.c_int]
    L.orc_get.restype = C.c_int
    L.orc_get.argtypes = [vp, C.c_int, I32P]
    L.orc_num_node.restype = C.c_int
    L.orc_num_node.argtypes = [vp]
    L.orc_cost.restype = C.c_int64
    L.orc_cost.argtypes = [vp]
    L.orc_nonzero.restype = C.c_int64
    L.orc_nonzero.argtypes = [vp]
    L.orc_array_size.restype = C.c_int64
    L.orc_array_size.argtypes = [vp, C.c_int]
    L.orc_tile.restype = C.c_int64
    L.orc_tile.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]
    L.orc_set_tile.argtypes = [vp, C.c_int, C.c_int, C.c_int, F64P]
    L.orc_use_blas.restype = C.c_int
    L.orc_use_blas.argtypes = [C.c_char_p, C.c_char_p]
    L.orc_max_threads.restype = C.c_int
    L.orc_t_compute_tree.argtypes = [C.c_int, I32P, I32P, I32P]
    L.orc_t_column_count.argtypes = [C.c_int, I32P, I32P, I32P, I32P]
    L.orc_t_postorder.argtypes = [C.c_int, I32P, I32P, I32P]
    L.orc_t_parent_in_postordering_tree.argtypes = [C.c_int, I32P, I32P]
    L.orc_t_finding_leaves.argtypes = [C.c_int, I32P, I32P, I32P, I32P]
    L.orc_t_search_node_sets.restype = C.c_int
    L.orc_t_search_node_sets.argtypes = [C.c_int, I32P, I32P, I32P, I32P]
    L.orc_t_merge_lists.argtypes = [C.c_int, I32P, I32P, I32P, I32P, C.c_int, I32P]
    L.orc_t_symbolic_factorize.argtypes = [C.c_int, I32P, I32P, I32P, I32P, I32P, I32P, I32P]
    L.orc_t_supernodal_ccs.restype = C.c_int
    L.orc_t_supernodal_ccs.argtypes = [C.c_int, I32P, I32P, C.c_int, I32P, I32P, I32P]
    L.orc_t_supernodal_index.argtypes = [C.c_int, I32P, I32P, I32P, C.c_int, I32P, I32P, I32P]
    L.orc_t_local_index.argtypes = [C.c_int, I32P, I32P, I32P, I32P, I32P, I32P]
    L.orc_t_block_local_index.restype = C.c_int
    L.orc_t_block_local_index.argtypes = [C.c_int, I32P, I32P, C.c_int, I32P, I32P,
                                          I32P, I32P, I32P, I32P, I32P, I32P, I32P]
    L.orc_t_node_geometry.argtypes = [C.c_int, I32P, I32P, C.c_int, I32P, I32P, I32P, I32P, I64P]
    L.orc_t_tile_start.restype = C.c_int64
    L.orc_t_tile_start.argtypes = [C.c_int, I32P, I32P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    _lib = L
    return L


def i32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


def f64(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def sets_from_lengths(lengths) -> np.ndarray:
    """contiguous_sets_c%ptr for the given lengths (1-based)."""
    lengths = np.asarray(lengths, dtype=np.int64)
    return i32(np.concatenate([[1], 1 + np.cumsum(lengths)]))


def use_system_blas(enable: bool = True) -> bool:
    """Route the oracle's dense kernels through the OpenBLAS bundled with scipy
    (the reference links a sequential BLAS/LAPACK); returns True on success."""
    L = lib()
    if not enable:
        L.orc_use_blas(None, None)
        return True
    import scipy  # noqa: F401  (locates scipy.libs)
    cands = glob.glob(os.path.join(os.path.dirname(scipy.__file__) + ".libs", "libscipy_openblas*.so"))
    for path in cands:
        if L.orc_use_blas(path.encode(), b"scipy_") == 0:
            _openblas_single_thread(path)
            return True
    return False


def _openblas_single_thread(path: str) -> None:
    try:
        h = C.CDLL(path)
        for sym in ("scipy_openblas_set_num_threads64_", "scipy_openblas_set_num_threads", "openblas_set_num_threads"):
            fn = getattr(h, sym, None)
            if fn is not None:
                fn(C.c_int(1))
                return
    except OSError:
        pass


class Oracle:
    """State after hppllt_analyze (hppllt_data_m.f90:14-29) plus the numeric phase."""

    def __init__(self, handle, n: int, nnz: int):
        self._h = handle
        self.n = n
        self.nnz = nnz

    # -- construction ---------------------------------------------------------
    @classmethod
    def analyze(cls, n, ccs_col, ccs_row, nb=10, max_zero=10, order_perm=None) -> "Oracle":
        """hppllt_analyze; order_perm (new->old, 1-based) stands in for METIS."""
        L = lib()
        ccs_col, ccs_row = i32(ccs_col), i32(ccs_row)
        op = None
        if order_perm is not None:
            order_perm = i32(order_perm)
            op = order_perm.ctypes.data_as(C.c_void_p)
        h = L.orc_analyze(int(n), ccs_col, ccs_row, int(nb), int(max_zero), op)
        o = cls(h, int(n), int(ccs_col[-1] - 1))
        o._keep = order_perm
        return o

    @classmethod
    def from_internal(cls, node_size, l_lengths, l_rows, parent, n, a_col, a_row_global, nb) -> "Oracle":
        L = lib()
        node_size = i32(node_size)
        h = L.orc_from_internal(len(node_size), node_size, sets_from_lengths(l_lengths), i32(l_rows),
                                i32(parent), int(n), i32(a_col), i32(a_row_global), int(nb))
        return cls(h, int(n), int(a_col[-1] - 1))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_free(self._h)
            self._h = None

    # -- accessors ------------------------------------------------------------
    def get(self, which: int) -> np.ndarray:
        L = lib()
        s = L.orc_get_size(self._h, which)
        out = np.zeros(max(s, 1), dtype=np.int32)
        L.orc_get(self._h, which, out)
        return out[:s]

    @property
    def num_node(self) -> int:
        return lib().orc_num_node(self._h)

    def symbolic(self) -> dict:
        """The symbolic arrays the reference holds after analysis (1-based int32)."""
        return {
            "n": self.n, "nnz": self.nnz, "num_node": self.num_node,
            "node_ptr": self.get(NODE_SETS), "parent": self.get(PARENT),
            "lptr": self.get(LPTR), "lrow": self.get(LROW),
            "aptr": self.get(APTR), "arow": self.get(AROW),
            "ccs_perm": self.get(CCS_PERM), "perm": self.get(PERM),
        }

    def cost(self) -> int:
        return int(lib().orc_cost(self._h))

    def nonzero(self) -> int:
        return int(lib().orc_nonzero(self._h))

    def array_size(self, which: int) -> int:
        return int(lib().orc_array_size(self._h, which))

    def tile(self, node, i, j, buffer=1) -> np.ndarray:
        """Copy out tile (i,j) of node from buffer 1=supernode 2=work 3=border (0=get_matrix)."""
        L = lib()
        ln = L.orc_tile(self._h, buffer, node, i, j, None)
        out = np.zeros(max(ln, 0), dtype=np.float64)
        if ln > 0:
            L.orc_tile(self._h, buffer, node, i, j, out.ctypes.data_as(C.c_void_p))
        return out

    def set_tile(self, node, i, j, vals) -> None:
        lib().orc_set_tile(self._h, node, i, j, f64(vals))

    # -- numeric --------------------------------------------------------------
    def factorize(self, a, nthreads: int = 0, schedule: str = "tree") -> int:
        """Numeric factorization.  nthreads <= 1: the sequential loop
        (seq_factorize); otherwise schedule "tree" runs the supernodes of one
        tree level in parallel, "dag" the reference's StarPU task DAG as
        OpenMP tasks over tiles (starpu_factorize)."""
        a = f64(a)
        if nthreads and nthreads > 1:
            if schedule == "dag":
                return lib().orc_factorize_dag(self._h, a, int(nthreads))
            return lib().orc_factorize_parallel(self._h, a, int(nthreads))
        return lib().orc_factorize(self._h, a)

    def solve(self, b) -> np.ndarray:
        x = f64(np.array(b, dtype=np.float64, copy=True))
        lib().orc_solve(self._h, x)
        return x

    def solve_many(self, B, nthreads: int = 0) -> np.ndarray:
        """Solve every column of B (n x k) as solve() does, columns over host threads."""
        X = np.array(B, dtype=np.float64, order="F", copy=True)
        if X.ndim == 1:
            X = X[:, None]
        flat = X.ravel(order="F")
        nt = nthreads if nthreads > 0 else (os.cpu_count() or 1)
        lib().orc_solve_many(self._h, flat, int(X.shape[1]), int(X.shape[0]), int(nt))
        return flat.reshape(X.shape, order="F")

    def sweep(self, permuted_rhs, backward: bool) -> np.ndarray:
        x = f64(np.array(permuted_rhs, dtype=np.float64, copy=True))
        lib().orc_sweep(self._h, x, 1 if backward else 0)
        return x


# ---------------------------------------------------------------------------
# unit-level restatements used by the golden-vector tests
# ---------------------------------------------------------------------------
def coo_to_ccs(n, row, col, val):
    """The reference driver's COO -> CCS (example.f90:95-145): 1-based
    (ccs_col, ccs_row, ccs_val)."""
    row, col, val = i32(row), i32(col), f64(val)
    ptr = np.zeros(n + 1, np.int32)
    rows = np.zeros(max(1, row.size), np.int32)
    vals = np.zeros(max(1, row.size), np.float64)
    lib().orc_coo_to_ccs(int(n), int(row.size), row, col, val, ptr, rows, vals)
    return ptr, rows[:row.size], vals[:row.size]


def tree_pruning(node_size, cc, num_child, child, tol, p) -> list:
    """tree_pruning_m.f90:13-155: subtree roots (1-based) for p workers."""
    ns = i32(node_size)
    roots = np.zeros(max(1, ns.size), np.int32)
    ch = i32(child) if len(child) else np.zeros(1, np.int32)
    k = lib().orc_tree_pruning(int(ns.size), ns, i32(cc), i32(num_child), ch, float(tol), int(p), roots)
    return roots[:k].tolist()


def compute_tree(num_col, col) -> np.ndarray:
    n = len(num_col)
    out = np.zeros(n, np.int32)
    lib().orc_t_compute_tree(n, sets_from_lengths(num_col), i32(col), out)
    return out


def column_count(num_row, row, parent) -> np.ndarray:
    n = len(num_row)
    out = np.zeros(n, np.int32)
    lib().orc_t_column_count(n, sets_from_lengths(num_row), i32(row), i32(parent), out)
    return out


def postorder(parent):
    n = len(parent)
    perm, sub = np.zeros(n, np.int32), np.zeros(n, np.int32)
    lib().orc_t_postorder(n, i32(parent), perm, sub)
    return perm, sub


def parent_in_postordering_tree(num_child) -> np.ndarray:
    n = len(num_child)
    out = np.zeros(n, np.int32)
    lib().orc_t_parent_in_postordering_tree(n, i32(num_child), out)
    return out


def finding_leaves(subtree, num_row, row) -> np.ndarray:
    n = len(num_row)
    out = np.zeros(n, np.int32)
    lib().orc_t_finding_leaves(n, i32(subtree), sets_from_lengths(num_row), i32(row), out)
    return out


def search_node_sets(isleaf, num_child, child_val) -> np.ndarray:
    n = len(isleaf)
    out = np.zeros(n + 1, np.int32)
    ns = lib().orc_t_search_node_sets(n, i32(isleaf), i32(num_child), i32(child_val), out)
    return out[: ns + 1]


def merge_lists(cc, num_child, child_val, node_size, max_zero):
    n = len(cc)
    out = np.zeros(2 * n + 1, np.int32)
    lib().orc_t_merge_lists(n, i32(cc), i32(num_child), i32(child_val), i32(node_size), int(max_zero), out)
    lists, cur = [], []
    for v in out[: 2 * n]:
        if v == 0:
            lists.append(cur)
            cur = []
            if len(lists) == n:
                break
        else:
            cur.append(int(v))
    return lists


def symbolic_factorize(a_len, a_val, cc, node_size, num_child, child_val) -> np.ndarray:
    out = np.zeros(int(np.sum(cc)), np.int32)
    lib().orc_t_symbolic_factorize(len(a_len), i32(a_len), i32(a_val), i32(cc), i32(node_size),
                                   i32(num_child), i32(child_val), out)
    return out


def supernodal_ccs(num_row, row, sets):
    n = len(num_row)
    ns = len(sets) - 1
    lens = np.zeros(ns, np.int32)
    vals = np.zeros(len(row), np.int32)
    t = lib().orc_t_supernodal_ccs(n, sets_from_lengths(num_row), i32(row), ns, i32(sets), lens, vals)
    return lens, vals[:t]


def supernodal_index(node_size, l_len, l_val, a_len, a_val) -> np.ndarray:
    out = np.zeros(len(a_val), np.int32)
    lib().orc_t_supernodal_index(len(node_size), i32(node_size), i32(l_len), i32(l_val), len(a_len),
                                 i32(a_len), i32(a_val), out)
    return out


def local_index(node_size, l_len, l_val, num_child, child_val) -> np.ndarray:
    out = np.zeros(len(l_val), np.int32)
    lib().orc_t_local_index(len(node_size), i32(node_size), i32(l_len), i32(l_val), i32(num_child),
                            i32(child_val), out)
    return out


def block_local_index(nc, nr, nb, l_len, l_val) -> dict:
    nn = len(nc)
    tot = int(np.sum(l_len))
    cap = max(tot, 1)
    node_ptr = np.zeros(nn + 1, np.int32)
    block_ptr = np.zeros(cap + 1, np.int32)
    pnum, cnum, off, start = (np.zeros(cap, np.int32) for _ in range(4))
    val = np.zeros(cap, np.int32)
    ng = lib().orc_t_block_local_index(nn, i32(nc), i32(nr), int(nb), i32(l_len), i32(l_val),
                                       node_ptr, block_ptr, pnum, cnum, off, start, val)
    return {"node_ptr": node_ptr, "block_ptr": block_ptr[: ng + 1], "parent_num": pnum[:ng],
            "child_num": cnum[:ng], "offset": off[:ng], "start_row": start[:ng], "val": val[:tot],
            "num_groups": ng}


def node_geometry(nc, nr, nb) -> dict:
    nn = len(nc)
    ws, nblk, ss, wsz = (np.zeros(nn, np.int32) for _ in range(4))
    tot = np.zeros(3, np.int64)
    lib().orc_t_node_geometry(nn, i32(nc), i32(nr), int(nb), ws, nblk, ss, wsz, tot)
    return {"work_start": ws, "num_block": nblk, "ssize": ss, "wsize": wsz, "totals": tot}


def tile_start(nc, nr, nb, kind, node, i, j) -> int:
    return int(lib().orc_t_tile_start(len(nc), i32(nc), i32(nr), int(nb), kind, node, i, j))
