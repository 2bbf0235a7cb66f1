"""Host setup routines (pargemslr_b200/csrc/setup.cpp) checked on the CPU.

The C++ harness tests/setup_harness.cpp is compiled against setup.cpp with
g++ and checks the nested-dissection level structure (a permutation whose
levels have uncoupled subdomains), ILUT (exact LU without dropping, the fill
limit with it), the Matrix Market reader, and the multicolor order inside
subdomains (same levels, uncoupled runs of rows, far fewer factor levels,
and the red-black split of its factors, which solves as the plain factors do).
"""
import os
import shutil
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_setup_routines(tmp_path):
    exe = str(tmp_path / "setup_harness")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-o", exe, os.path.join(HERE, "setup_harness.cpp"),
                    os.path.join(ROOT, "pargemslr_b200", "csrc", "setup.cpp")], check=True)
    mm = tmp_path / "s.mtx"
    # lower triangle of a symmetric matrix, one entry given twice: (1,1) = 1.5 + 2
    mm.write_text("%%MatrixMarket matrix coordinate real symmetric\n"
                  "3 3 5\n1 1 1.5\n1 1 2\n3 1 -1\n2 2 2\n3 3 4\n")
    out = subprocess.run([exe, str(mm)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count("ok") == 6, out.stdout


EDGE_SCRIPT = r'''
import ctypes as C, sys
import numpy as np
import scipy.sparse as sp
sys.path.insert(0, sys.argv[2])
from pargemslr_b200 import _abi, problems, params as P
L = _abi.lib()
p = P.workload_params("lap2d_256")
def lap(nx, ny):
    a = problems.laplacian(nx, ny, 1)
    return sp.csr_matrix((a[2], a[1], a[0]), shape=(nx * ny, nx * ny))
case = sys.argv[1]
if case == "one":
    M = sp.csr_matrix(np.array([[4.0]]))
elif case == "diagonal":
    M = sp.diags(np.arange(1, 51, dtype=float))
elif case == "two_blocks":
    M = sp.block_diag([lap(10, 10), lap(7, 9)])
elif case == "path3":
    M = sp.diags([-1.0, 4.0, -1.0], [-1, 0, 1], shape=(3, 3))
elif case == "star":
    M = sp.lil_matrix((60, 60)); M.setdiag(60.0)
    for i in range(1, 60):
        M[0, i] = -1.0; M[i, 0] = -1.0
elif case == "nonsymmetric_pattern":
    M = sp.random(300, 300, density=0.02, random_state=2) + sp.eye(300) * 5
elif case == "more_levels_than_rows":
    p[P.PREPOSS_NLEV_GLOBAL] = 12
    M = lap(6, 6)
elif case == "rank_above_size":
    p[P.LR_RANK1_GLOBAL] = p[P.LR_RANK2_GLOBAL] = 500
    M = lap(12, 12)
elif case == "multicolor_order":
    p[P.ILU_PERM_OPTION_GLOBAL] = 6
    a = problems.laplacian(20, 20, 20)
    M = sp.csr_matrix((a[2], a[1], a[0]), shape=(8000, 8000))
elif case == "empty_row":
    M = sp.lil_matrix((20, 20)); M.setdiag(2.0); M[5, 5] = 0.0
M = sp.csr_matrix(M); M.eliminate_zeros(); M.sort_indices()
n = M.shape[0]
keep = []
arrs = (M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data.astype(np.float64))
A = _abi.csr_struct(*arrs, n, n, keep=keep)
h = C.c_void_p()
print("rc", L.pgx_gemslr_setup(C.byref(h), C.byref(A), _abi.ptr(p), 0), L.pgx_last_error().decode())
'''


@pytest.mark.parametrize("case,expect", [("one", 200), ("diagonal", 200), ("two_blocks", 200), ("path3", 200),
                                         ("star", 200), ("nonsymmetric_pattern", 200),
                                         ("more_levels_than_rows", 200), ("rank_above_size", 200),
                                         ("multicolor_order", 200),
                                         ("empty_row", 103)])
def test_host_setup_of_awkward_matrices(tmp_path, case, expect):
    """pgx_gemslr_setup on matrices a file could hold: the host part (levels, ILUT, coupling blocks) completes and
    the call stops at the first device step (200 without a GPU), or fails with the reference's code (103: an empty
    row in ILUT).  Each case runs in its own process, so a crash fails the test instead of the session."""
    from tests.conftest import _has_gpu
    if _has_gpu():
        pytest.skip("checks the host part, which ends at the device step on a machine without a GPU")
    script = tmp_path / "edge.py"
    script.write_text(EDGE_SCRIPT)
    out = subprocess.run([sys.executable, str(script), case, ROOT], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.split()[:2] == ["rc", str(expect)], out.stdout
