"""Parameter arrays on the host (pgx_params_default / pgx_params_read_file); no GPU needed.

The reference's drivers fill the double[180] array that SetWithParameterArray
reads from PargemslrSetDefaultParameterArray and then from a parameter file,
in one of three line-oriented formats (sequential, parallel, hypre).  The
library's reader is pinned to the reference's own three parsers: bit for bit
on every slot, and on the status, over seeded random files
(tests/params_fuzz.py) whose reference results are in
tests/golden/params_files.json, over the reference's own driver parameter
files, and, when oracle/_ref holds the parsers, over further random files
compared live.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from pargemslr_b200 import _abi
from pargemslr_b200 import params as P
from oracle.paths import REFERENCE_TESTS
from tests import params_fuzz as F

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "params_files.json")))
REF_TESTS = REFERENCE_TESTS


def _write(tmp_path, name, text):
    path = tmp_path / name
    path.write_text(text)
    return str(path)


def _read(path, fmt, base):
    """(status, array) of the library's reader, as the reference parser reports them."""
    p = np.array(base, dtype=np.float64)
    rc = _abi.lib().pgx_params_read_file(path.encode(), _abi.INPUTS_FORMATS[fmt], _abi.ptr(p))
    return rc, p


def test_defaults_match_the_reference():
    ref = np.array(GOLDEN["reference_inputs"]["defaults"]["values"])
    np.testing.assert_array_equal(_abi.params_default(), ref)
    np.testing.assert_array_equal(P.default_params(), ref)


@pytest.mark.parametrize("fmt", list(F.FORMATS))
def test_random_files_match_the_reference_parser(tmp_path, fmt):
    fill = GOLDEN["fill"]
    cases = [c for c in GOLDEN["cases"] if c["format"] == fmt]
    assert len(cases) >= 40 and any(c["status"] != 0 for c in cases) and any(c["status"] == 0 for c in cases)
    for c in cases:
        text = F.random_file(fmt, c["seed"])
        assert hashlib.sha256(text.encode()).hexdigest() == c["sha256"], "the file generator changed"
        rc, got = _read(_write(tmp_path, f"{fmt}_{c['seed']}", text), fmt, np.full(180, fill))
        want = np.full(180, fill)
        for i, v in c["changed"]:
            want[i] = v
        assert rc == c["status"], (fmt, c["seed"], rc, _abi.lib().pgx_last_error())
        np.testing.assert_array_equal(got, want, err_msg=f"{fmt} seed {c['seed']}")


def test_python_mirror_of_the_sequential_file():
    """params.sequential_inputs_params() restates TESTS/sequential/inputs by hand; it must equal what
    the reference parser builds from that file."""
    ref = np.array(GOLDEN["reference_inputs"]["sequential/inputs"]["values"])
    np.testing.assert_array_equal(P.sequential_inputs_params(), ref)


@pytest.mark.skipif(not os.path.isdir(REF_TESTS), reason="reference sources not present")
@pytest.mark.parametrize("rel", [k for k in GOLDEN["reference_inputs"] if k != "defaults"])
def test_reference_driver_files(rel):
    g = GOLDEN["reference_inputs"][rel]
    got = _abi.params_read_file(os.path.join(REF_TESTS, rel), g["format"])
    np.testing.assert_array_equal(got, np.array(g["values"]))


@pytest.mark.parametrize("fmt", list(F.FORMATS))
def test_further_random_files_live(tmp_path, fmt):
    if not F.reference_available(fmt):
        pytest.skip("oracle/_ref parsers not built")
    for seed in range(1000, 1100):
        path = _write(tmp_path, f"{fmt}_{seed}", F.random_file(fmt, seed))
        for base in (None, -2.25):
            rc_ref, want = F.run_reference(fmt, path, base)
            start = _abi.params_default() if base is None else np.full(180, base)
            rc, got = _read(path, fmt, start)
            assert rc == rc_ref, (fmt, seed)
            np.testing.assert_array_equal(got, want, err_msg=f"{fmt} seed {seed}")


def test_hypre_file_line_by_line(tmp_path):
    """Each line of a hypre-format file, as the reference parser reads it (a line's numbers stop at the
    first token that is not one; a trailing comment that starts with a number is read as one; an exponent
    marker without digits is taken into the number before it, "1e 2" being 1 then 2), up to an unknown
    keyword, which stops the read with the I/O error and leaves the later lines unread."""
    lines = ["gemslr c", "1 c", "ILUK c", "4. levels", "Gemslr c", "BJILUK c", "2", "1e 2 c", "7 x 9",
             "ND c", "rkway c", "1e-3 2E+ 3 .5e1 c", "10 20", "1 2 3", "amd c", "QQ c", "STD c"]
    path = _write(tmp_path, "h", "\n".join(lines) + "\n")
    rc, p = _read(path, "hypre", np.full(180, -1.0))
    assert rc == _abi.ERROR_IO
    assert "line 16" in _abi.lib().pgx_last_error().decode()
    want = np.full(180, -1.0)
    for slot, v in [(P.PRECOND_GLOBAL_PRECOND, 2), (P.PREPOSS_GLOBAL_PARTITION, 1), (P.PRECOND_LOCAL_REPCOND1, 1),
                    (P.PRECOND_LOCAL_REPCOND1_LEVEL, 4), (P.PRECOND_LOCAL_REPCOND2, 2), (P.PRECOND_LOCAL_REPCOND3, 3),
                    (P.POLY_ORDER, 2), (P.PREPOSS_NLEV_GLOBAL, 1), (P.PREPOSS_NLEV_LOCAL, 2),
                    (P.PREPOSS_NCOMP_GLOBAL, 7), (P.PREPOSS_PARTITION_GLOBAL, 0), (P.PREPOSS_PARTITION_LOCAL, 1),
                    (P.ILU_DROPTOL_B_GLOBAL, 1e-3), (P.ILU_DROPTOL_B_LOCAL, 1e-3), (P.ILU_DROPTOL_EF_GLOBAL, 2),
                    (P.ILU_DROPTOL_EF_LOCAL, 2), (P.ILU_DROPTOL_S_GLOBAL, 3), (P.ILU_DROPTOL_S_LOCAL, 3),
                    (P.ILU_DROPTOL_C_GLOBAL, 5), (P.ILU_DROPTOL_C_LOCAL, 5), (P.ILU_ROWNNZ_B_GLOBAL, 10),
                    (P.ILU_ROWNNZ_B_LOCAL, 10), (P.ILU_ROWNNZ_S_GLOBAL, 20), (P.ILU_ROWNNZ_S_LOCAL, 20),
                    (P.ILU_LFIL_B_GLOBAL, 1), (P.ILU_LFIL_B_LOCAL, 1), (P.ILU_LFIL_C_GLOBAL, 3),
                    (P.ILU_LFIL_C_LOCAL, 3), (P.ILU_PERM_OPTION_GLOBAL, 2), (P.ILU_PERM_OPTION_LOCAL, 2)]:
        want[slot] = v
    np.testing.assert_array_equal(p, want)
    if F.reference_available("hypre"):
        rc_ref, v_ref = F.run_reference("hypre", path, -1.0)
        assert rc_ref == rc
        np.testing.assert_array_equal(v_ref, want)


def test_errors(tmp_path):
    L = _abi.lib()
    p = _abi.params_default()
    assert L.pgx_params_read_file(str(tmp_path / "missing").encode(), 0, _abi.ptr(p)) == _abi.ERROR_IO
    path = _write(tmp_path, "s", "ILUT c\n")
    assert L.pgx_params_read_file(path.encode(), 3, _abi.ptr(p)) == _abi.ERROR_INVALID_PARAM
    assert L.pgx_params_read_file(None, 0, _abi.ptr(p)) == _abi.ERROR_INVALID_PARAM
    assert L.pgx_params_read_file(path.encode(), 0, None) == _abi.ERROR_INVALID_PARAM
    assert L.pgx_params_default(None) == _abi.ERROR_INVALID_PARAM
    np.testing.assert_array_equal(p, _abi.params_default())
    # an empty file changes nothing
    empty = _write(tmp_path, "e", "")
    for fmt in F.FORMATS:
        np.testing.assert_array_equal(_abi.params_read_file(empty, fmt), _abi.params_default())


ARG_CASES = [
    # (argv, {slot: value}) as the drivers' read_inputs applies them
    (["-tol", "1e-3", "-kdim", "30", "-maxits", "77"], {13: 1e-3, 11: 30, 12: 77}),
    (["-maxits", "-5", "x", "-maxits", "12"], {12: 12}),  # a value starting with '-' is skipped
    (["-kdim", "2.9e1", "-kdim", "40"], {11: 2}),  # atoi reads the leading digits; the first use wins
    (["--tol", "5", "tol", "6", "-tol"], {}),  # neither "--tol" nor a bare name nor a trailing flag counts
    (["-tol", "abc"], {13: 0.0}),  # atof of a non-number
    ([], {}),
]


@pytest.mark.parametrize("argv,changed", ARG_CASES)
def test_command_line_arguments(argv, changed):
    want = _abi.params_default()
    for slot, v in changed.items():
        want[slot] = v
    np.testing.assert_array_equal(_abi.params_read_args(argv), want)
    if F.reference_available("sequential"):
        rc, ref = F.run_reference_args(argv)
        assert rc == 0
        np.testing.assert_array_equal(ref, want)


def test_random_command_lines_live():
    if not F.reference_available("sequential"):
        pytest.skip("oracle/_ref parsers not built")
    import random
    rng = random.Random(17)
    toks = ["-tol", "-kdim", "-maxits", "-x", "--tol", "tol", "1e-3", "-1", "42", "3.5", "abc", "", "7e", "0x10"]
    for _ in range(200):
        argv = [rng.choice(toks) for _ in range(rng.randint(0, 8))]
        rc, ref = F.run_reference_args(argv)
        np.testing.assert_array_equal(_abi.params_read_args(argv), ref, err_msg=repr(argv))
