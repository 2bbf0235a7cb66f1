"""Matrix Market ingestion (pgx_csr_read_mm) on the host; no GPU needed.

The reader follows CooMatrixReadFromFile (coordinate, real or integer,
general or symmetric with off-diagonal entries mirrored) and returns CSR with
sorted columns and summed duplicates; scipy's reader is the independent check.
The reference's own test matrices are used when its sources are present.
"""
import os

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from pargemslr_b200 import _abi

REF_MATRICES = "/root/reference/ParGeMSLR/TESTS/sequential/Matrices"


def _check_against_scipy(path):
    rp, cj, va, shape = _abi.read_mm(path)
    ref = sp.csr_matrix(scipy.io.mmread(path))
    ref.sum_duplicates()
    ref.sort_indices()
    assert shape == ref.shape
    np.testing.assert_array_equal(rp, ref.indptr)
    np.testing.assert_array_equal(cj, ref.indices)
    np.testing.assert_allclose(va, ref.data, rtol=0, atol=0)


@pytest.mark.parametrize("symmetric", [False, True])
def test_reader_matches_scipy_on_written_files(tmp_path, symmetric):
    rng = np.random.default_rng(4)
    M = sp.random(300, 300, density=0.02, random_state=5, format="coo")
    M = M + sp.eye(300)
    if symmetric:
        M = sp.tril(M + M.T).tocoo()
    path = str(tmp_path / "m.mtx")
    scipy.io.mmwrite(path, M, symmetry="symmetric" if symmetric else "general")
    _check_against_scipy(path)


def test_duplicates_are_summed(tmp_path):
    path = tmp_path / "d.mtx"
    path.write_text("%%MatrixMarket matrix coordinate real general\n% c\n3 3 4\n1 1 1.5\n2 3 2\n1 1 0.25\n3 2 -1\n")
    rp, cj, va, shape = _abi.read_mm(str(path))
    assert shape == (3, 3)
    np.testing.assert_array_equal(rp, [0, 1, 2, 3])
    np.testing.assert_array_equal(cj, [0, 2, 1])
    np.testing.assert_array_equal(va, [1.75, 2.0, -1.0])


def test_unsupported_files_fail_cleanly(tmp_path):
    bad = tmp_path / "p.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate pattern general\n2 2 1\n1 1\n")
    with pytest.raises(_abi.PgxError):
        _abi.read_mm(str(bad))
    with pytest.raises(_abi.PgxError):
        _abi.read_mm(str(tmp_path / "missing.mtx"))


@pytest.mark.skipif(not os.path.isdir(REF_MATRICES), reason="reference sources not present")
@pytest.mark.parametrize("name", ["gr_30_30.mtx", "test_small.mtx", "test_sym_small.mtx"])
def test_reference_test_matrices(name):
    _check_against_scipy(os.path.join(REF_MATRICES, name))
