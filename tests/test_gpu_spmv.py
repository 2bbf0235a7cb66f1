"""GPU CSR SpMV variants against the oracle's CsrMatrixPMatVecHostTemplate restatement (matrixops.cpp:5139).

Both variants (S lanes per row; merge path) and the histogram's choice are run on device arrays through the C ABI on
a regular matrix (3D Laplacian), the serving workload's uniform random matrix (7-27 per row) and a matrix with
skewed rows, and compared with the oracle in FP64: y = alpha A x + beta y within 1e-13 relative (the variants sum
a row in different orders).  Empty rows and a zero-row matrix are covered.  The lanes-per-row kernel loads whole
aligned 4-entry blocks (128-bit loads) when the arrays allow it (16-byte aligned, nonzeros a multiple of 4) and single
entries otherwise; the "blocks" cases trim the last row so that the nonzeros fill whole blocks.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from pargemslr_b200 import _abi
from pargemslr_b200 import problems

pytestmark = pytest.mark.gpu

MATRICES = {
    "lap3d_32": lambda: problems.laplacian(32, 32, 32),
    "random_7_27": lambda: problems.random_diag_dominant(60000, 7),
    "skewed": lambda: problems.random_skewed(60000, 8),
}


def _device_csr(A, keep):
    import torch
    rp, cj, va = A
    t = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (rp, cj, va)]
    keep.extend(t)
    n = rp.size - 1
    return _abi.Csr(n, n, cj.size, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr())


def _with_empty_rows(A, every=97):
    rp, cj, va = A
    lens = np.diff(rp)
    keep = np.repeat(np.arange(rp.size - 1) % every != 0, lens)
    lens = np.where(np.arange(rp.size - 1) % every != 0, lens, 0)
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.int32), cj[keep], va[keep]


def _whole_blocks(A):
    rp, cj, va = A
    cut = cj.size % 4
    if cut == 0:
        return A
    rp = rp.copy()
    rp[-1] -= cut
    return rp, cj[:rp[-1]], va[:rp[-1]]


@pytest.mark.parametrize("name", sorted(MATRICES))
@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("shape", ["plain", "empty_rows", "blocks"])
def test_spmv_matches_oracle(name, variant, shape):
    import torch
    A = MATRICES[name]()
    if shape == "empty_rows":
        A = _with_empty_rows(A)
    if shape in ("empty_rows", "blocks"):
        A = _whole_blocks(A)
    rp, cj, va = A
    n = rp.size - 1
    rng = np.random.default_rng(1)
    x = rng.standard_normal(n)
    y0 = rng.standard_normal(n)
    for alpha, beta in ((1.0, 0.0), (-0.5, 2.0)):
        y_ref = y0.copy()
        O.csr_matvec(O.Csr(rp, cj, va, n, n), alpha, x, beta, y_ref)
        keep = []
        Ad = _device_csr(A, keep)
        xd = torch.from_numpy(x).cuda()
        yd = torch.from_numpy(y0.copy()).cuda()
        _abi.check(_abi.lib().pgx_csr_spmv_device_variant(C.byref(Ad), variant, alpha, xd.data_ptr(), beta,
                                                          yd.data_ptr()))
        y = yd.cpu().numpy()
        err = np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref)
        assert err <= 1e-13, (name, variant, alpha, beta, err)


def test_zero_row_matrix_is_a_no_op():
    import torch
    Ad = _abi.Csr(0, 0, 0, None, None, None)
    y = torch.ones(4, dtype=torch.float64, device="cuda")
    _abi.check(_abi.lib().pgx_csr_spmv_device_variant(C.byref(Ad), 2, 1.0, y.data_ptr(), 0.0, y.data_ptr()))
    assert torch.all(y == 1)
