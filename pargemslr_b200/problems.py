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
