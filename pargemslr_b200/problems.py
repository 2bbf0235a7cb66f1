"""Synthetic test matrices of the benchmark workloads.

``laplacian`` restates the reference's 5-/7-point stencil generator
(CooMatrixClass::Laplacian, ParGeMSLR SRC/matrices/coo_matrix.cpp:519-614):
diagonal 4 (2D) or 6 (3D) minus ``shift``, off-diagonals -1 -/+ alpha in each
direction, Dirichlet boundary by truncation, rows in natural (x fastest)
order with columns sorted.
"""
from __future__ import annotations

import numpy as np


def laplacian(nx: int, ny: int, nz: int, alphax: float = 0.0, alphay: float = 0.0, alphaz: float = 0.0,
              shift: float = 0.0):
    """(rowptr, colidx, values) of the reference stencil, int32/int32/float64.

    Within a row the entries come in the reference's insertion order:
    z-, z+, y-, y+, x-, x+, diagonal.
    """
    n = nx * ny * nz
    is2d = (nx == 1) + (ny == 1) + (nz == 1) > 0
    vd = (4.0 if is2d else 6.0) - shift
    idx = np.arange(n, dtype=np.int64)
    k = idx // (nx * ny)
    i = (idx - k * nx * ny) // nx
    j = idx - k * nx * ny - i * nx
    rows, cols, vals, slot = [], [], [], []
    stencil = ((k > 0, -nx * ny, -1.0 + alphaz), (k < nz - 1, nx * ny, -1.0 - alphaz),
               (i > 0, -nx, -1.0 + alphay), (i < ny - 1, nx, -1.0 - alphay),
               (j > 0, -1, -1.0 + alphax), (j < nx - 1, 1, -1.0 - alphax),
               (np.ones(n, bool), 0, vd))
    for s, (cond, off, v) in enumerate(stencil):
        r = idx[cond]
        rows.append(r)
        cols.append(r + off)
        vals.append(np.full(r.size, v))
        slot.append(np.full(r.size, s))
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    order = np.lexsort((np.concatenate(slot), r))
    r, c, v = r[order], c[order], v[order]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, r + 1, 1)
    rp = np.cumsum(rp)
    return rp.astype(np.int32), c.astype(np.int32), v.astype(np.float64)


def x_true(n: int, seed: int) -> np.ndarray:
    """x_true = 2u - 1 with u ~ U[0, 1) from a seeded generator."""
    rng = np.random.default_rng(seed)
    return 2.0 * rng.random(n) - 1.0


def spmv(A, x: np.ndarray) -> np.ndarray:
    rp, cj, va = A
    y = np.zeros(len(rp) - 1)
    np.add.at(y, np.repeat(np.arange(len(rp) - 1), np.diff(rp)), va * x[cj])
    return y


def _csr_from_rows(n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray):
    order = np.lexsort((cols, rows))
    r, c, v = rows[order], cols[order], vals[order]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp).astype(np.int32), c.astype(np.int32), v.astype(np.float64)


def upwind_convdiff_2d(nx: int, ny: int, beta_x: float, beta_y: float):
    """-Laplace(u) + beta . grad(u) on an nx x ny grid, h = 1/(n+1), first-order
    upwind convection, Dirichlet boundary by truncation, scaled by h^2.

    Nonsymmetric for beta != 0.  The reference's stencil is central, so this
    generator is the project's own (rows in natural order, columns sorted).
    """
    n = nx * ny
    hx, hy = 1.0 / (nx + 1), 1.0 / (ny + 1)
    idx = np.arange(n, dtype=np.int64)
    i = idx // nx
    j = idx - i * nx
    # upwind: for beta > 0 the convection term couples to the west/south neighbour
    wx, wy = abs(beta_x) * hx, abs(beta_y) * hy
    west = -1.0 - (wx if beta_x > 0 else 0.0)
    east = -1.0 - (wx if beta_x < 0 else 0.0)
    south = -1.0 - (wy if beta_y > 0 else 0.0)
    north = -1.0 - (wy if beta_y < 0 else 0.0)
    diag = 4.0 + wx + wy
    parts = ((j > 0, -1, west), (j < nx - 1, 1, east), (i > 0, -nx, south), (i < ny - 1, nx, north),
             (np.ones(n, bool), 0, diag))
    rows = np.concatenate([idx[c] for c, _, _ in parts])
    cols = np.concatenate([idx[c] + off for c, off, _ in parts])
    vals = np.concatenate([np.full(int(c.sum()), v) for c, _, v in parts])
    return _csr_from_rows(n, rows, cols, vals)


def random_diag_dominant(n: int, seed: int, nnz_min: int = 7, nnz_max: int = 27, factor: float = 1.2):
    """Nonsymmetric random sparse matrix: each row has a uniform number of
    nonzeros in [nnz_min, nnz_max] (diagonal included) at random columns,
    off-diagonal values ~ N(0, 1), and the diagonal set to `factor` times
    the row's absolute off-diagonal sum."""
    rng = np.random.default_rng(seed)
    per_row = rng.integers(nnz_min - 1, nnz_max, size=n)  # off-diagonals per row
    rows = np.repeat(np.arange(n, dtype=np.int64), per_row)
    cols = rng.integers(0, n - 1, size=rows.size)
    cols = cols + (cols >= rows)  # never the diagonal
    vals = rng.standard_normal(rows.size)
    # merge duplicate (row, col) pairs
    key = rows * n + cols
    key, inv = np.unique(key, return_inverse=True)
    vals = np.bincount(inv, weights=vals)
    rows, cols = key // n, key % n
    diag = factor * np.bincount(rows, weights=np.abs(vals), minlength=n)
    diag[diag == 0] = 1.0
    allr = np.concatenate([rows, np.arange(n)])
    allc = np.concatenate([cols, np.arange(n)])
    allv = np.concatenate([vals, diag])
    return _csr_from_rows(n, allr, allc, allv)


def random_skewed(n: int, seed: int, heavy_frac: float = 0.02, heavy=(200, 2000), light=(3, 9), factor: float = 1.2):
    """Random sparse matrix with skewed row lengths: a fraction `heavy_frac` of the rows (at random positions) holds
    `heavy` = [lo, hi) nonzeros each, the others `light` = [lo, hi); values and diagonal as random_diag_dominant.
    The long rows carry most of the nonzeros, the case the merge-path SpMV is for."""
    rng = np.random.default_rng(seed)
    per_row = rng.integers(light[0] - 1, light[1] - 1, size=n)
    hv = rng.random(n) < heavy_frac
    per_row[hv] = rng.integers(heavy[0] - 1, heavy[1] - 1, size=int(hv.sum()))
    per_row = np.minimum(per_row, n - 1)
    rows = np.repeat(np.arange(n, dtype=np.int64), per_row)
    cols = rng.integers(0, n - 1, size=rows.size)
    cols = cols + (cols >= rows)
    vals = rng.standard_normal(rows.size)
    key = rows * n + cols
    key, inv = np.unique(key, return_inverse=True)
    vals = np.bincount(inv, weights=vals)
    rows, cols = key // n, key % n
    diag = factor * np.bincount(rows, weights=np.abs(vals), minlength=n)
    diag[diag == 0] = 1.0
    allr = np.concatenate([rows, np.arange(n)])
    allc = np.concatenate([cols, np.arange(n)])
    allv = np.concatenate([vals, diag])
    return _csr_from_rows(n, allr, allc, allv)
