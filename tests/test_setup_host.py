"""Host setup routines (pargemslr_b200/csrc/setup.cpp) checked on the CPU.

The C++ harness tests/setup_harness.cpp is compiled against setup.cpp with
g++ and checks the nested-dissection level structure (a permutation whose
levels have uncoupled subdomains), ILUT (exact LU without dropping, the fill
limit with it) and the Matrix Market reader.
"""
import os
import shutil
import subprocess

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
    assert out.stdout.count("ok") == 4, out.stdout
