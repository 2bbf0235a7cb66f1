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

from oracle.paths import REFERENCE_TESTS
from pargemslr_b200 import _abi

REF_MATRICES = os.path.join(REFERENCE_TESTS, "sequential", "Matrices")


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


VECTOR_REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "vector_ref")


def _vector_reference(path, idxin):
    import subprocess
    out = subprocess.run([VECTOR_REF, path, str(idxin)], capture_output=True, text=True, check=True).stdout.split()
    k = out.index("rc")
    rc = int(out[k + 1])
    if rc:
        return rc, None
    n = int(out[k + 3])
    return 0, np.array([float.fromhex(v) for v in out[k + 4:k + 4 + n]])


VECTOR_FILES = {
    # name: (text, idxin, expected values by index or None for an error)
    "plain": ("%%MatrixMarket matrix coordinate real general\n% c\n5 1 3\n1 1 2.5\n4 1 -1\n5 1 3e-2\n", 1,
              {0: 2.5, 3: -1.0, 4: 0.03}),
    "later_entry_wins": ("%%MatrixMarket matrix coordinate real general\n4 1 3\n2 1 1\n3 1 7\n2 1 -4\n", 1,
                         {1: -4.0, 2: 7.0}),
    "zero_based": ("%%MatrixMarket matrix coordinate integer general\n3 1 2\n0 0 5\n2 0 6\n", 0, {0: 5.0, 2: 6.0}),
    "column_ignored": ("%%MatrixMarket matrix coordinate real general\n3 2 2\n1 2 1.5\n3 1 2\n", 1,
                       {0: 1.5, 2: 2.0}),
    "out_of_range": ("%%MatrixMarket matrix coordinate real general\n3 1 1\n4 1 1\n", 1, None),
    "array_format": ("%%MatrixMarket matrix array real general\n2 1\n1\n2\n", 1, None),
}


@pytest.mark.parametrize("name", sorted(VECTOR_FILES))
def test_vector_reader(tmp_path, name):
    text, idxin, want = VECTOR_FILES[name]
    path = tmp_path / f"{name}.mtx"
    path.write_text(text)
    if want is None:
        with pytest.raises(_abi.PgxError):
            _abi.read_mm_vector(str(path), idxin)
    else:
        x = _abi.read_mm_vector(str(path), idxin)
        size_line = next(line for line in text.split("\n") if line and line[0] != "%")
        expect = np.zeros(int(size_line.split()[0]))
        for i, v in want.items():
            expect[i] = v
        np.testing.assert_array_equal(x, expect)
    # the reference's reader agrees where it is defined (it does not check the index range)
    if os.path.exists(VECTOR_REF) and name != "out_of_range":
        rc, ref = _vector_reference(str(path), idxin)
        if want is None:
            assert rc != 0
        else:
            assert rc == 0
            np.testing.assert_array_equal(x, ref)


@pytest.mark.skipif(not os.path.isdir(REF_MATRICES), reason="reference sources not present")
def test_reference_right_hand_side_file():
    path = os.path.join(REF_MATRICES, "gr_30_30_b.mtx")
    x = _abi.read_mm_vector(path, 1)
    ref = np.asarray(scipy.io.mmread(path).todense()).ravel()
    np.testing.assert_array_equal(x, ref)
    if os.path.exists(VECTOR_REF):
        rc, r = _vector_reference(path, 1)
        assert rc == 0
        np.testing.assert_array_equal(x, r)


def test_vector_capacity_is_checked(tmp_path):
    import ctypes as C
    path = tmp_path / "v.mtx"
    path.write_text("%%MatrixMarket matrix coordinate real general\n6 1 1\n2 1 1\n")
    n = C.c_int32(0)
    x = np.zeros(3)
    rc = _abi.lib().pgx_vector_read_mm(str(path).encode(), 1, 3, _abi.ptr(x), C.byref(n))
    assert rc == _abi.ERROR_INVALID_PARAM and n.value == 6


def test_headers_that_promise_more_than_the_file_holds(tmp_path):
    """A header's counts size nothing by themselves: a file claiming 10^15 entries, or a vector of 2^31 - 1 rows,
    fails at its first missing or bad entry with the I/O error, without allocating for the claim."""
    big = tmp_path / "big.mtx"
    big.write_text("%%MatrixMarket matrix coordinate real general\n2000000000 2000000000 1000000000000000\n")
    with pytest.raises(_abi.PgxError) as e:
        _abi.read_mm(str(big))
    assert e.value.code == _abi.ERROR_IO and "entry 1" in str(e.value)
    vec = tmp_path / "vec.mtx"
    vec.write_text("%%MatrixMarket matrix coordinate real general\n2147483647 1 2\n1 1 1.0\nx\n")
    with pytest.raises(_abi.PgxError) as e:
        _abi.read_mm_vector(str(vec))
    assert e.value.code == _abi.ERROR_IO and "entry 2" in str(e.value)
