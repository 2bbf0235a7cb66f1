"""The hypre plugin interface (include/pgx_hypre.h) through the C ABI.

HYPRE_pargemslr.cpp unpacks a hypre ParCSR matrix into diag/offd CSR arrays
(hypre keeps each row's diagonal entry first) and calls the plugin's matrix
create, preconditioner create / SetParams / Setup / Solve and the parameter
file reader.  Without a GPU: the matrix is taken in with sorted rows, matrices
of more than one rank are refused, the parameter file equals the reference
parser's result, and calls made out of order fail cleanly.  On a GPU: Solve
is one preconditioner application, bit for bit the one the Python front end
computes from the same matrix and parameters.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from pargemslr_b200 import _abi
from pargemslr_b200 import params as P
from pargemslr_b200 import problems
from oracle.paths import REFERENCE_TESTS

HERE = os.path.dirname(os.path.abspath(__file__))
REF_HYPRE_INPUTS = os.path.join(REFERENCE_TESTS, "hypre", "inputs")


def _diag_first(A):
    """A's rows with the diagonal entry moved to the front, as hypre stores them."""
    rp, cj, va = (np.array(a) for a in A)
    for r in range(rp.size - 1):
        b, e = rp[r], rp[r + 1]
        k = b + int(np.nonzero(cj[b:e] == r)[0][0])
        cj[b:k + 1] = np.roll(cj[b:k + 1], 1)
        va[b:k + 1] = np.roll(va[b:k + 1], 1)
    return rp.astype(np.int32), cj.astype(np.int32), va.astype(np.float64)


def _sorted(A):
    rp, cj, va = A
    n = rp.size - 1
    M = sp.csr_matrix((va, cj, rp), shape=(n, n))
    M.sort_indices()
    return M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data.astype(np.float64)


def _create(A, nrow_global=None, nrow_start=0, offd_i=None, location=0):
    rp, cj, va = A
    n = rp.size - 1
    ng = n if nrow_global is None else nrow_global
    return _abi.lib().pgx_hypre_csr_matrix_create(ng, ng, nrow_start, nrow_start, n, n, _abi.ptr(rp), _abi.ptr(cj),
                                                   _abi.ptr(va), _abi.ptr(offd_i), None, None, 0, None, location)


def test_matrix_is_taken_in_with_sorted_rows():
    L = _abi.lib()
    A = problems.laplacian(9, 7, 3)
    H = _diag_first(A)
    assert not np.array_equal(H[1], A[1])
    m = _create(H, offd_i=np.zeros(A[0].size, np.int32))
    assert m
    v = _abi.Csr()
    _abi.check(L.pgx_hypre_csr_matrix_view(m, C.byref(v)))
    n = A[0].size - 1
    S = _sorted(A)
    assert (v.rows, v.cols, v.nnz) == (n, n, S[1].size)
    np.testing.assert_array_equal(np.ctypeslib.as_array(C.cast(v.rowptr, C.POINTER(C.c_int32)), (n + 1,)), S[0])
    np.testing.assert_array_equal(np.ctypeslib.as_array(C.cast(v.colidx, C.POINTER(C.c_int32)), (v.nnz,)), S[1])
    np.testing.assert_array_equal(np.ctypeslib.as_array(C.cast(v.values, C.POINTER(C.c_double)), (v.nnz,)), S[2])
    assert L.pgx_hypre_csr_matrix_destroy(m) == 0


def test_matrices_of_more_than_one_rank_are_refused():
    L = _abi.lib()
    A = problems.laplacian(6, 6, 1)
    n = A[0].size - 1
    assert not _create(A, nrow_global=2 * n)
    assert b"one rank" in L.pgx_last_error()
    assert not _create(A, nrow_global=2 * n, nrow_start=n)
    offd = np.zeros(n + 1, np.int32)
    offd[1:] = 1  # one off-rank entry in row 0
    assert not _create(A, offd_i=offd)
    assert b"off-diagonal" in L.pgx_last_error()
    assert not _create(A, location=2)
    bad = (A[0], A[1].copy(), A[2])
    bad[1][3] = n
    assert not _create(bad)
    assert b"out of range" in L.pgx_last_error()
    assert L.pgx_hypre_csr_matrix_destroy(None) == 0


def test_parameter_file():
    L = _abi.lib()
    p = L.pgx_hypre_params_from_file(None)
    np.testing.assert_array_equal(np.ctypeslib.as_array(p, (180,)), _abi.params_default())
    L.pgx_hypre_params_destroy(p)
    # as in the reference, a file that cannot be read leaves the defaults
    p = L.pgx_hypre_params_from_file(b"/nonexistent/inputs")
    np.testing.assert_array_equal(np.ctypeslib.as_array(p, (180,)), _abi.params_default())
    L.pgx_hypre_params_destroy(p)
    if os.path.exists(REF_HYPRE_INPUTS):
        golden = json.load(open(os.path.join(HERE, "golden", "params_files.json")))["reference_inputs"]["hypre/inputs"]
        p = L.pgx_hypre_params_from_file(REF_HYPRE_INPUTS.encode())
        np.testing.assert_array_equal(np.ctypeslib.as_array(p, (180,)), np.array(golden["values"]))
        L.pgx_hypre_params_destroy(p)


def test_calls_out_of_order():
    L = _abi.lib()
    g = L.pgx_hypre_gemslr_create()
    assert g
    x = np.zeros(4)
    assert L.pgx_hypre_gemslr_solve(g, None, _abi.ptr(x), _abi.ptr(x)) == _abi.ERROR_FUNCTION_CALL
    assert L.pgx_hypre_gemslr_set_precision(g, 7) == _abi.ERROR_INVALID_OPTION
    assert L.pgx_hypre_gemslr_set_precision(g, _abi.PRECISION_MIXED) == 0
    assert L.pgx_hypre_gemslr_set_params(g, None) == _abi.ERROR_INVALID_PARAM
    assert L.pgx_hypre_gemslr_setup(g, None, None, None) == _abi.ERROR_INVALID_PARAM
    assert not L.pgx_hypre_gemslr_handle(g)
    assert L.pgx_hypre_gemslr_destroy(g) == 0
    assert L.pgx_hypre_gemslr_destroy(None) == 0


def test_setup_without_a_device_fails_cleanly():
    """On a machine without a GPU the host setup runs and the move to the device is refused."""
    from tests.conftest import _has_gpu
    if _has_gpu():
        pytest.skip("a GPU is present")
    L = _abi.lib()
    A = problems.laplacian(12, 12, 1)
    m = _create(A)
    g = L.pgx_hypre_gemslr_create()
    p = P.workload_params("lap2d_256")
    _abi.check(L.pgx_hypre_gemslr_set_params(g, _abi.ptr(p)))
    assert L.pgx_hypre_gemslr_setup(g, m, None, None) != 0
    assert not L.pgx_hypre_gemslr_handle(g)
    x = np.zeros(A[0].size - 1)
    assert L.pgx_hypre_gemslr_solve(g, m, _abi.ptr(x), _abi.ptr(x)) == _abi.ERROR_FUNCTION_CALL
    L.pgx_hypre_gemslr_destroy(g)
    L.pgx_hypre_csr_matrix_destroy(m)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_is_one_preconditioner_application(precision):
    from pargemslr_b200.handle import GemslrHandle, init
    init(0)
    L = _abi.lib()
    A = _sorted(problems.laplacian(96, 96, 1))
    n = A[0].size - 1
    p = P.workload_params("lap2d_256")
    m = _create(_diag_first(A))
    g = L.pgx_hypre_gemslr_create()
    _abi.check(L.pgx_hypre_gemslr_set_params(g, _abi.ptr(p)))
    _abi.check(L.pgx_hypre_gemslr_set_precision(g, {"fp64": 0, "mixed": 1}[precision]))
    _abi.check(L.pgx_hypre_gemslr_setup(g, m, None, None))
    _abi.check(L.pgx_hypre_gemslr_setup(g, m, None, None))  # set up once
    b = problems.x_true(n, 9)
    x = np.zeros(n)
    _abi.check(L.pgx_hypre_gemslr_solve(g, m, _abi.ptr(x), _abi.ptr(b)))
    h = GemslrHandle.from_matrix(A, p, precision=precision)
    np.testing.assert_array_equal(x, h.apply(b))
    h.close()
    L.pgx_hypre_gemslr_destroy(g)
    L.pgx_hypre_csr_matrix_destroy(m)
