"""The C-ABI library loads and exports every symbol include/pgx.h and include/pgx_hypre.h declare (no GPU)."""
import os
import re

from pargemslr_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header="pgx.h"):
    with open(os.path.join(ROOT, "include", header)) as f:
        text = f.read()
    return sorted(set(re.findall(r"^(?:int|const char \*|void \*|double \*|pgx_handle)\s*(pgx_\w+)\s*\(", text, re.M)))


def test_header_and_binding_agree():
    assert declared() == sorted(_abi.EXPORTS)
    assert declared("pgx_hypre.h") == sorted(_abi.HYPRE_EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _abi.lib()
    missing = [s for s in declared() + declared("pgx_hypre.h") if not hasattr(L, s)]
    assert not missing, missing


def test_calls_without_device_fail_cleanly():
    import ctypes as C
    L = _abi.lib()
    h = C.c_void_p()
    assert L.pgx_gemslr_create(C.byref(h), 0, 0) == _abi.ERROR_INVALID_PARAM
    assert L.pgx_gemslr_create(C.byref(h), 4, 7) == _abi.ERROR_INVALID_OPTION
    assert L.pgx_gemslr_solve(None, None, None, 0, None, None) == _abi.ERROR_INVALID_PARAM
    assert b"null" in L.pgx_last_error()


def test_level_schedule_rejects_non_triangular_factor():
    import numpy as np
    import pytest
    rp = np.array([0, 1, 2], np.int32)
    cj = np.array([1, 0], np.int32)  # row 0 depends on row 1: not lower triangular
    with pytest.raises(_abi.PgxError):
        _abi.build_levels("L", rp, cj)
