"""Complex systems on the host side: the reference's complexd dump, its import
through the C ABI (no device needed before commit) and the refusals.

The fixture tests/golden/zlap3d_12 comes from the reference's own complex
solver (oracle/_ref/pgx_ref_driver_z over GemslrClass<..., complexd>): a 12^3
Laplacian shifted by 0.3 + 0.05i, 5 levels, two complex-Gaussian right-hand
sides.
"""
import ctypes as C
import os

import numpy as np
import pytest

from pargemslr_b200 import _abi, pgxd
from pargemslr_b200.handle import import_structures
from pargemslr_b200.structures import from_dump

CASE = os.path.join(os.path.dirname(__file__), "golden", "zlap3d_12")


def test_complex_dump_loads_as_complex_structures():
    st = from_dump(os.path.join(CASE, "setup.bin"))
    assert st.complex and st.n == 12 ** 3 and st.nlev == 5
    assert st.A[2].dtype == np.complex128
    for l, lv in enumerate(st.levels):
        assert lv.L[2].dtype == np.complex128 and lv.dinv.dtype == np.complex128
        assert lv.dinv.size == lv.L[3]
        if lv.rank:
            m = st.n - int(st.lev_ptr[l + 1])
            assert lv.W.dtype == np.complex128 and lv.W.size == m * lv.rank
    # the matrix is the reference's shifted stencil: diagonal 6 - (0.3 + 0.05i)
    rp, cj, va = st.A[0], st.A[1], st.A[2]
    diag = np.array([va[k] for r in range(st.n) for k in range(rp[r], rp[r + 1]) if cj[k] == r])
    np.testing.assert_allclose(diag, 6.0 - (0.3 + 0.05j))
    prob = pgxd.read(os.path.join(CASE, "problem.bin"))
    assert int(prob["nrhs"][0]) == 2 and prob["B"].view(np.complex128).size == 2 * st.n


def test_complex_structures_import_through_the_abi():
    st = from_dump(os.path.join(CASE, "setup.bin"))
    for precision in ("fp64", "mixed"):
        h = import_structures(st, precision)
        assert h
        _abi.lib().pgx_gemslr_destroy(h)


def test_complex_import_checks_sizes_and_refuses_the_host_setup():
    L = _abi.lib()
    h = C.c_void_p()
    assert L.pgx_gemslr_create(C.byref(h), 8, 7) == _abi.ERROR_INVALID_OPTION
    _abi.check(L.pgx_gemslr_create(C.byref(h), 4, _abi.PRECISION_COMPLEX_FP64))
    try:
        # a 4 x 4 complex diagonal: 4 values are 8 doubles
        keep = []
        rp = np.arange(5, dtype=np.int32)
        cj = np.arange(4, dtype=np.int32)
        va = np.array([1 + 1j, 2, 3 - 1j, 4], np.complex128)
        A = _abi.csr_struct(rp, cj, va, 4, 4, keep=keep)
        assert A.nnz == 4
        _abi.check(L.pgx_gemslr_set_matrix(h, C.byref(A)))
    finally:
        L.pgx_gemslr_destroy(h)
    # this library's host setup is real; a complex preconditioner is imported
    keep = []
    A = _abi.csr_struct(np.arange(5, dtype=np.int32), np.arange(4, dtype=np.int32), np.ones(4), 4, 4, keep=keep)
    p = np.zeros(180)
    h2 = C.c_void_p()
    rc = L.pgx_gemslr_setup(C.byref(h2), C.byref(A), _abi.ptr(p), _abi.PRECISION_COMPLEX_MIXED)
    assert rc == _abi.ERROR_INVALID_OPTION
    assert b"real" in L.pgx_last_error()
