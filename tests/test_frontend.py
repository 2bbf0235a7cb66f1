"""The C++ front end (include/pgx_pargemslr.hpp): the reference's class names over the C ABI.

tests/frontend_driver.cpp is a driver written like the reference's parallel
Laplacian driver (build A, b = A x_true, SetMatrixP / SetWithParameterArray /
SetPreconditionerP, Setup(x, b), Solve(x, b), the getters), compiled with g++
as C++11 against the header and linked with libpgx.so.  Without a GPU it
checks the host side: the matrix is the reference stencil byte for byte, the
right-hand side is A x_true, a driver parameter file is read, and calls made
out of order return the reference's status codes.  On a GPU, the driver's
solution and preconditioner application equal those of the same setup made
through the Python front end, bit for bit.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from pargemslr_b200 import _abi
from pargemslr_b200 import params as P
from pargemslr_b200 import problems

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")

# sequential-format lines (TESTS/sequential/io.cpp:336-725): the slot each line sets, and
# for keyword lines the words by value
_B = ["ILUT", "ILUK", "GEMSLR"]
_SEQ = [(1, _B), 2, (3, _B), 11, 12, 13, 14, 20, 21, 22, 23, (24, ["ND", "RKWAY"]), (25, ["ND", "RKWAY"]),
        40, 44, 48, 50, 52, 54, (58, ["NO", "RCM", "AMD", "ND"]), (70, ["STD", "TR", "SUB"]),
        (71, ["STD", "TR", "SUB"]), 74, 75, 86, 87, 78, 79, 82, 83, 90, 91, 130, 131, 132, 142,
        (141, ["LU", "U", "MUL"]), 150]


def write_sequential(path, p):
    """A sequential-format parameter file holding p's values in the slots the format sets."""
    out = []
    for k, line in enumerate(_SEQ):
        if isinstance(line, tuple):
            slot, words = line
            out.append(f" {words[int(p[slot])]}   {k + 1}. keyword\n")
        else:
            out.append(f" {float(p[line])!r}   {k + 1}. value\n")
    with open(path, "w") as f:
        f.write("".join(out))


def _build(tmp_path):
    exe = str(tmp_path / "frontend_driver")
    lib = os.path.dirname(_abi.LIB_PATH)
    subprocess.run(["g++", "-O2", "-std=c++11", "-Wall", "-Wextra", "-Werror", "-ffp-contract=off",
                    "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "frontend_driver.cpp"), "-o", exe,
                    "-L", lib, "-lpgx", f"-Wl,-rpath,{lib}"], check=True)
    return exe


def _run(exe, out, nx, ny, nz, params_file="-", fmt=0, precision=0):
    r = subprocess.run([exe, str(nx), str(ny), str(nz), params_file, str(fmt), str(precision), str(out)],
                       capture_output=True, text=True, timeout=600)
    kv = {}
    for line in r.stdout.split("\n"):
        for tok in line.split(" "):
            if "=" in tok:
                k, v = tok.split("=", 1)
                kv.setdefault(k, v)
    return r.returncode, kv, r.stdout


def _load(out, name, dtype):
    return np.fromfile(os.path.join(out, name), dtype=dtype)


def test_driver_host_side(tmp_path):
    exe = _build(tmp_path)
    out = tmp_path / "o"
    out.mkdir()
    xt = problems.x_true(14 * 9 * 3, 4)
    xt.tofile(str(out / "xtrue.bin"))
    p = P.workload_params("lap2d_256")
    pf = str(tmp_path / "inputs")
    write_sequential(pf, p)
    rc, kv, text = _run(exe, out, 14, 9, 3, pf, 0)
    assert rc == 0, text
    assert kv["params"] == "0" and kv["laplacian"] == "0" and kv["matvec"] == "0", text
    # the parameter file round-trips every slot it names
    got = _load(out, "params.bin", np.float64)
    for line in _SEQ:
        slot = line[0] if isinstance(line, tuple) else line
        assert got[slot] == p[slot], slot
    # the reference stencil, byte for byte, and b = A x_true in the reference's row order
    A = problems.laplacian(14, 9, 3)
    np.testing.assert_array_equal(_load(out, "A_rp.bin", np.int32), A[0])
    np.testing.assert_array_equal(_load(out, "A_cj.bin", np.int32), A[1])
    np.testing.assert_array_equal(_load(out, "A_va.bin", np.float64), A[2])
    np.testing.assert_array_equal(_load(out, "b.bin", np.float64), problems.spmv(A, xt))
    # calls out of order: the reference's codes
    assert kv["solve_before_setup"] == str(_abi.ERROR_FUNCTION_CALL)
    assert kv["apply_before_setup"] == str(_abi.ERROR_FUNCTION_CALL)
    assert kv["nnz_before_setup"] == "-1"
    assert kv["matvec_trans"] == str(_abi.ERROR_INVALID_OPTION)
    assert kv["mm_zero_based"] == str(_abi.ERROR_INVALID_OPTION)
    assert kv["precision"] == "0"
    assert kv.get("device") == "none" or kv.get("solve") == "0", text


def test_driver_rejects_a_bad_parameter_file(tmp_path):
    exe = _build(tmp_path)
    bad = tmp_path / "inputs"
    bad.write_text(" ILUT c\n 1 c\n NOPE c\n")
    rc, kv, text = _run(exe, tmp_path, 4, 4, 1, str(bad), 0)
    assert rc == 1 and kv["params"] == str(_abi.ERROR_IO) and "line 3" in text


def test_vector_from_matrix_market(tmp_path):
    """ParallelVectorClass::ReadFromMMFile reads a right-hand-side file as the reference's vector reader does."""
    vec = tmp_path / "b.mtx"
    vec.write_text("%%MatrixMarket matrix coordinate real general\n5 1 3\n2 1 0.5\n5 1 -2\n2 1 4\n")
    src = tmp_path / "v.cpp"
    src.write_text('#include <cstdio>\n#include "pgx_pargemslr.hpp"\n'
                   "int main(int, char** argv) { pgx::ParallelVectorClass<double> b;\n"
                   "  int rc = b.ReadFromMMFile(argv[1], 1); printf(\"%d %d\", rc, b.GetLengthLocal());\n"
                   "  for (int i = 0; i < b.GetLengthLocal(); i++) printf(\" %g\", b.GetData()[i]);\n"
                   "  printf(\" %d\\n\", b.ReadFromMMFile(\"/nonexistent.mtx\", 1)); return 0; }\n")
    exe = str(tmp_path / "v")
    lib = os.path.dirname(_abi.LIB_PATH)
    subprocess.run(["g++", "-std=c++11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", exe,
                    "-L", lib, "-lpgx", f"-Wl,-rpath,{lib}"], check=True)
    out = subprocess.run([exe, str(vec)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["0", "5", "0", "4", "0", "0", "-2", str(_abi.ERROR_IO)]


def test_single_precision_types_do_not_compile(tmp_path):
    src = tmp_path / "f.cpp"
    src.write_text('#include "pgx_pargemslr.hpp"\nint main() { pgx::ParallelVectorClass<float> v; return 0; }\n')
    r = subprocess.run(["g++", "-std=c++11", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "FP64" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_driver_solve_equals_python_front_end(tmp_path, precision):
    from pargemslr_b200.handle import GemslrHandle
    exe = _build(tmp_path)
    out = tmp_path / "o"
    out.mkdir()
    nx, ny = 96, 96
    xt = problems.x_true(nx * ny, 6)
    xt.tofile(str(out / "xtrue.bin"))
    pf = str(tmp_path / "inputs")
    write_sequential(pf, P.workload_params("lap2d_256"))
    prec = {"fp64": 0, "mixed": 1}[precision]
    rc, kv, text = _run(exe, out, nx, ny, 1, pf, 0, prec)
    assert rc == 0 and kv["setup"] == "0" and kv["solve"] == "0" and kv["apply"] == "0", text
    assert float(kv["true_rel_res"]) <= 1e-8, text
    p = _load(out, "params.bin", np.float64)
    A = problems.laplacian(nx, ny, 1)
    b = _load(out, "b.bin", np.float64)
    h = GemslrHandle.from_matrix(A, p, precision=precision)
    x, r = h.solve(b, params=p)
    assert int(kv["iters"]) == r["iters"]
    np.testing.assert_array_equal(_load(out, "x.bin", np.float64), x)
    np.testing.assert_array_equal(_load(out, "z.bin", np.float64), h.apply(b))
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) <= 1e-5  # this library's own setup, as in test_gpu_setup
    nb, nl = C.c_int64(), C.c_int64()
    _abi.check(_abi.lib().pgx_gemslr_nnz(h._h, C.byref(nb), C.byref(nl)))
    assert int(kv["nnz_bsolver"]) == nb.value and int(kv["nnz_lr"]) == nl.value
    assert int(kv["nnz_total"]) == nb.value + nl.value and nb.value > A[1].size
    h.close()
