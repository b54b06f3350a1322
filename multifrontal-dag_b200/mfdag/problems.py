"""Synthetic SPD test problems and their fill-reducing orderings.

Matrices are returned in the reference solver's input format: the symmetric
lower triangle in CCS with 1-based int32 column pointers and row indices, rows
ascending inside each column and the diagonal first (the order example.f90's
coo_to_ccs produces and that the reference's analysis relies on).

Orderings are geometric nested dissection on the grid: they are passed to the
analysis in place of METIS_NodeND's output (the reference's use_metis = 1
branch, hppllt.f90:47-51), so the CPU oracle and the GPU path consume the
identical permutation.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Problem:
    name: str
    n: int
    col: np.ndarray          # int32, n+1, 1-based
    row: np.ndarray          # int32, nnz, 1-based
    val: np.ndarray          # float64, nnz
    order: np.ndarray | None = None   # int32 new->old, 1-based (None: natural order)
    rhs: np.ndarray | None = None     # float64 (n,) or (n, nrhs) column-major
    x_true: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.col[-1] - 1)


def _lower_ccs(n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray):
    """Sort 0-based (row >= col) triplets into lower CCS, rows ascending per column."""
    order = np.lexsort((rows, cols))
    rows, cols, vals = rows[order], cols[order], vals[order]
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(ptr, cols + 1, 1)
    ptr = np.cumsum(ptr) + 1
    return ptr.astype(np.int32), (rows + 1).astype(np.int32), vals.astype(np.float64)


def grid_laplacian(dims, diag=None, off=-1.0, shift=0.0):
    """5-point (2D) / 7-point (3D) Laplacian, lexicographic numbering x fastest."""
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    if diag is None:
        diag = 2.0 * len(dims)
    idx = np.arange(n)
    coords = np.unravel_index(idx, dims[::-1])[::-1]      # x, y, (z)
    rows, cols, vals = [idx], [idx], [np.full(n, diag + shift)]
    stride = 1
    for ax, d in enumerate(dims):
        mask = coords[ax] < d - 1
        c = idx[mask]
        rows.append(c + stride); cols.append(c); vals.append(np.full(c.size, off))
        stride *= d
    return _lower_ccs(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def nested_dissection(dims, dof: int = 1, leaf: int = 8) -> np.ndarray:
    """Geometric nested dissection of a structured grid (x fastest numbering).

    Boxes are split across their longest axis by a one-cell-thick separator
    plane; both halves are ordered first, then the separator.  Inside a
    separator, cells that touch an ancestor separator (a box face that is not
    the domain boundary) are ordered last, corner lines after edge lines: each
    such cell brings new rows into the factor's column structure, so placing
    them last keeps the rest of the separator one fundamental supernode.
    Boxes with at most ``leaf`` cells are ordered lexicographically.  With
    dof > 1 the dofs of a cell stay contiguous.  Returns new->old, 1-based int32.
    """
    dims = tuple(int(d) for d in dims)
    nd = len(dims)
    grid = np.arange(int(np.prod(dims))).reshape(dims[::-1])   # [z][y][x] or [y][x]
    out = []

    def emit(lo, hi, is_sep):
        sl = tuple(slice(l, h) for l, h in zip(lo[::-1], hi[::-1]))
        cells = grid[sl].ravel()
        if not is_sep or cells.size <= 1:
            out.append(cells)
            return
        # count, per cell, the box faces it lies on that border an ancestor separator
        coords = np.unravel_index(cells, dims[::-1])[::-1]
        touch = np.zeros(cells.size, dtype=np.int64)
        for ax in range(nd):
            if hi[ax] - lo[ax] == 1:           # the separator's own thin axis
                continue
            if lo[ax] > 0:
                touch += coords[ax] == lo[ax]
            if hi[ax] < dims[ax]:
                touch += coords[ax] == hi[ax] - 1
        out.append(cells[np.argsort(touch, kind="stable")])

    work = [("box", tuple(0 for _ in dims), dims)]
    while work:
        kind, lo, hi = work.pop()
        size = [h - l for l, h in zip(lo, hi)]
        if kind == "sep":
            emit(lo, hi, True)
            continue
        if np.prod(size) <= leaf or max(size) <= 2:
            emit(lo, hi, False)
            continue
        ax = int(np.argmax(size))
        m = lo[ax] + size[ax] // 2
        left_hi = list(hi); left_hi[ax] = m
        right_lo = list(lo); right_lo[ax] = m + 1
        sep_lo = list(lo); sep_lo[ax] = m
        sep_hi = list(hi); sep_hi[ax] = m + 1
        # popped in reverse: left half, right half, then the separator
        work.append(("sep", tuple(sep_lo), tuple(sep_hi)))
        if right_lo[ax] < hi[ax]:
            work.append(("box", tuple(right_lo), tuple(hi)))
        work.append(("box", tuple(lo), tuple(left_hi)))
    cells = np.concatenate(out)
    if dof > 1:
        cells = (cells[:, None] * dof + np.arange(dof)[None, :]).ravel()
    return (cells + 1).astype(np.int32)


def _rhs_for(n, ptr, row, val, x):
    """b = A x for the symmetric matrix stored as its lower CCS."""
    return sym_matvec(n, ptr, row, val, x)


def sym_matvec(n, ptr, row, val, x):
    cols = np.repeat(np.arange(n), np.diff(ptr))
    r = row - 1
    x = np.asarray(x, dtype=np.float64)
    if x.ndim == 1:
        y = np.zeros(n)
        np.add.at(y, r, val * x[cols])
        off = r != cols
        np.add.at(y, cols[off], val[off] * x[r[off]])
        return y
    y = np.zeros_like(x)
    np.add.at(y, r, val[:, None] * x[cols])
    off = r != cols
    np.add.at(y, cols[off], val[off][:, None] * x[r[off]])
    return y


def laplace2d(side: int = 100, seed: int = 0, nd: bool = True) -> Problem:
    """2D 5-point Laplacian (diag 4, off -1); x* ~ U[-1,1] from ``seed``; b = A x*."""
    ptr, row, val = grid_laplacian((side, side), diag=4.0)
    n = side * side
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, n)
    b = sym_matvec(n, ptr, row, val, x)
    order = nested_dissection((side, side)) if nd else None
    return Problem(f"laplace2d_{side}x{side}", n, ptr, row, val, order, b, x, {"dims": (side, side)})


def laplace3d(side: int = 64, seed: int = 1, nd: bool = True) -> Problem:
    """3D 7-point Laplacian (diag 6, off -1); x* ~ U[-1,1] from ``seed``; b = A x*."""
    dims = (side, side, side)
    ptr, row, val = grid_laplacian(dims, diag=6.0)
    n = side ** 3
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, n)
    b = sym_matvec(n, ptr, row, val, x)
    order = nested_dissection(dims) if nd else None
    return Problem(f"laplace3d_{side}^3", n, ptr, row, val, order, b, x, {"dims": dims})


def diffusion3d(side: int = 80, seed: int = 2, nd: bool = True) -> Problem:
    """3D 7-point variable-coefficient diffusion with Dirichlet boundaries.

    Per-cell conductivity k = 10^U[-2,2] (seed); interior face coefficient is
    the harmonic mean 2 k1 k2 / (k1 + k2); a boundary face adds 2 k_cell to the
    diagonal only; A_ii is the sum of the cell's face coefficients and
    A_ij = -a_face.
    """
    dims = (side, side, side)
    n = side ** 3
    rng = np.random.default_rng(seed)
    k = 10.0 ** rng.uniform(-2.0, 2.0, n)
    idx = np.arange(n)
    coords = np.unravel_index(idx, dims[::-1])[::-1]
    diag = np.zeros(n)
    rows, cols, vals = [], [], []
    stride = 1
    for ax in range(3):
        lo_b = coords[ax] == 0
        hi_b = coords[ax] == side - 1
        diag[lo_b] += 2.0 * k[lo_b]
        diag[hi_b] += 2.0 * k[hi_b]
        m = coords[ax] < side - 1
        c = idx[m]
        a = 2.0 * k[c] * k[c + stride] / (k[c] + k[c + stride])
        diag[c] += a
        diag[c + stride] += a
        rows.append(c + stride); cols.append(c); vals.append(-a)
        stride *= side
    rows.append(idx); cols.append(idx); vals.append(diag)
    ptr, row, val = _lower_ccs(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))
    x = rng.uniform(-1.0, 1.0, n)
    b = sym_matvec(n, ptr, row, val, x)
    order = nested_dissection(dims) if nd else None
    return Problem(f"diffusion3d_{side}^3", n, ptr, row, val, order, b, x, {"dims": dims})


_GRID2D_CACHE: dict = {}


def _grid2d(side: int, nd: bool):
    """5-point structure, unshifted values and ordering of one side (memoized:
    a 2,000-system batch has at most 113 distinct sides)."""
    key = (side, nd)
    if key not in _GRID2D_CACHE:
        ptr, row, val = grid_laplacian((side, side), diag=4.0)
        order = nested_dissection((side, side)) if nd else None
        diag_pos = (ptr[:-1] - 1).astype(np.int64)        # the diagonal leads each column
        _GRID2D_CACHE[key] = (ptr, row, val, order, diag_pos)
    return _GRID2D_CACHE[key]


def laplace2d_batch(count: int = 2000, seed: int = 3, lo: int = 16, hi: int = 128, nd: bool = True):
    """Uneven batch of shifted 2D 5-point Laplacians.

    From one generator seeded with ``seed``: sides ~ randint[lo, hi] (inclusive),
    then shifts ~ U[0, 0.1], then each system's RHS ~ U[-1, 1] in system order.
    A_i = 5-point(s_i) + shift_i I.  Systems of equal side share their
    structure and ordering arrays (read-only).
    """
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=count)
    shifts = rng.uniform(0.0, 0.1, size=count)
    out = []
    for i in range(count):
        s = int(sides[i])
        ptr, row, val0, order, diag_pos = _grid2d(s, nd)
        val = val0.copy()
        val[diag_pos] += float(shifts[i])
        b = rng.uniform(-1.0, 1.0, s * s)
        out.append(Problem(f"batch_{i}_{s}", s * s, ptr, row, val, order, b, None,
                           {"dims": (s, s), "shift": float(shifts[i])}))
    return out


def _hex_stiffness_parts():
    """Q1 (trilinear) hexahedron on the unit cube, 2x2x2 Gauss quadrature.

    Returns (K_lambda, K_mu), 24 x 24, such that an isotropic element's
    stiffness is lambda * K_lambda + mu * K_mu.  Local nodes are the cube's
    corners in lexicographic order (x fastest), dofs node-major (ux, uy, uz).
    Strain rows: xx, yy, zz, xy, yz, zx (engineering shear).
    """
    corners = np.array([[a, b, c] for c in (0, 1) for b in (0, 1) for a in (0, 1)], dtype=np.float64)
    gp = np.array([0.5 - 0.5 / np.sqrt(3.0), 0.5 + 0.5 / np.sqrt(3.0)])
    m = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
    Dl = np.outer(m, m)
    Dm = np.diag([2.0, 2.0, 2.0, 1.0, 1.0, 1.0])
    Kl = np.zeros((24, 24))
    Km = np.zeros((24, 24))
    for z in gp:
        for y in gp:
            for x in gp:
                pt = (x, y, z)
                lin = np.where(corners == 1.0, np.array(pt)[None, :], 1.0 - np.array(pt)[None, :])   # 8 x 3 factors
                sgn = np.where(corners == 1.0, 1.0, -1.0)
                grad = np.empty((8, 3))
                for d in range(3):
                    others = [e for e in range(3) if e != d]
                    grad[:, d] = sgn[:, d] * lin[:, others[0]] * lin[:, others[1]]
                B = np.zeros((6, 24))
                for k in range(8):
                    gx, gy, gz = grad[k]
                    c = 3 * k
                    B[0, c] = gx
                    B[1, c + 1] = gy
                    B[2, c + 2] = gz
                    B[3, c], B[3, c + 1] = gy, gx
                    B[4, c + 1], B[4, c + 2] = gz, gy
                    B[5, c], B[5, c + 2] = gz, gx
                w = 1.0 / 8.0
                Kl += w * B.T @ Dl @ B
                Km += w * B.T @ Dm @ B
    return Kl, Km


def elasticity3d(ne: int = 40, seed: int = 4, nrhs: int = 64, nd: bool = True) -> Problem:
    """3D linear elasticity, Q1 hexahedra on an ne^3 unit-element mesh, 3 dofs
    per node, the face x = 0 clamped (its nodes removed).

    From one generator seeded with ``seed``, per element (x fastest):
    E = 10^U[-1, 1], then nu ~ U[0.25, 0.35]; then the nrhs right-hand sides
    ~ U[-1, 1] as an (n, nrhs) Fortran-ordered array.  Free nodes are the
    (ne) x (ne+1) x (ne+1) grid x = 1..ne, numbered x fastest, dofs node-major.
    """
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    nel = ne ** 3
    E = 10.0 ** rng.uniform(-1.0, 1.0, nel)
    nu = rng.uniform(0.25, 0.35, nel)
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    Kl, Km = _hex_stiffness_parts()
    nx, ny, nz = ne, ne + 1, ne + 1               # free-node grid
    n = 3 * nx * ny * nz
    e = np.arange(nel)
    ex, ey, ez = e % ne, (e // ne) % ne, e // (ne * ne)
    corners = [(a, b, c) for c in (0, 1) for b in (0, 1) for a in (0, 1)]
    gd = np.empty((nel, 24), dtype=np.int64)
    for k, (a, b, c) in enumerate(corners):
        x = ex + a
        node = (x - 1) + nx * ((ey + b) + ny * (ez + c))
        for d in range(3):
            gd[:, 3 * k + d] = np.where(x >= 1, 3 * node + d, -1)
    r = np.repeat(gd, 24, axis=1).reshape(nel, 24, 24)
    cidx = np.tile(gd, (1, 24)).reshape(nel, 24, 24)
    keep = (r >= cidx) & (cidx >= 0)
    vals = (lam[:, None, None] * Kl[None] + mu[:, None, None] * Km[None])[keep]
    A = sp.coo_matrix((vals, (r[keep], cidx[keep])), shape=(n, n)).tocsc()
    A.sum_duplicates()
    A.sort_indices()
    ptr = (A.indptr + 1).astype(np.int32)
    row = (A.indices + 1).astype(np.int32)
    val = A.data.astype(np.float64)
    b = np.asfortranarray(rng.uniform(-1.0, 1.0, (n, nrhs)))
    order = nested_dissection((nx, ny, nz), dof=3) if nd else None
    return Problem(f"elasticity3d_{ne}^3", n, ptr, row, val, order, b, None,
                   {"dims": (nx, ny, nz), "dof": 3, "elements": nel})


def backward_error(n, ptr, row, val, x, b) -> float:
    """Normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)."""
    r = np.asarray(b) - sym_matvec(n, ptr, row, val, x)
    absrow = sym_matvec(n, ptr, row, np.abs(val), np.ones(n))
    anorm = float(absrow.max())
    return float(np.abs(r).max() / (anorm * np.abs(x).max() + np.abs(b).max()))
