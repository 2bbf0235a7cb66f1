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
    assert L.pgx_gemslr_set_wait_limit(None, 5) == _abi.ERROR_INVALID_PARAM
    st = C.c_int32(0)
    assert L.pgx_wait_selfcheck(0, C.byref(st), None) == _abi.ERROR_INVALID_PARAM
    assert L.pgx_wait_selfcheck(5, None, None) == _abi.ERROR_INVALID_PARAM
    sy = C.c_void_p()
    assert L.pgx_systems_create(C.byref(sy), None, 0) == _abi.ERROR_INVALID_PARAM
    hs = (C.c_void_p * 2)(None, None)
    assert L.pgx_systems_create(C.byref(sy), C.cast(hs, C.c_void_p), 2) == _abi.ERROR_FUNCTION_CALL
    assert L.pgx_systems_solve(None, None, None, 0, None, None) == _abi.ERROR_INVALID_PARAM
    assert L.pgx_systems_set_schedule(None, 512, 2, 4, 2) == _abi.ERROR_INVALID_PARAM
    assert L.pgx_systems_destroy(None) == 0
    assert L.pgx_gemslr_set_solve_option(None, 1) == _abi.ERROR_INVALID_PARAM


def test_level_schedule_rejects_non_triangular_factor():
    import numpy as np
    import pytest
    rp = np.array([0, 1, 2], np.int32)
    cj = np.array([1, 0], np.int32)  # row 0 depends on row 1: not lower triangular
    with pytest.raises(_abi.PgxError):
        _abi.build_levels("L", rp, cj)


def test_a_c_program_links_and_calls_the_library(tmp_path):
    """The C ABI is usable from C: a C99 program that includes include/pgx.h and include/pgx_hypre.h, links
    libpgx.so and calls host-side entry points."""
    import shutil
    import subprocess

    import pytest
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    src = tmp_path / "host.c"
    src.write_text(r'''
#include <stdio.h>
#include "pgx.h"
#include "pgx_hypre.h"
int main(void) {
  double params[PGX_PARAMS_SIZE];
  const char *argv[] = {"-kdim", "30"};
  int32_t lp[2] = {0, 0}, order[1] = {0}, nlev = 0;
  const int32_t rp[2] = {0, 0};
  void *g;
  if (pgx_params_default(params) != PGX_SUCCESS) return 1;
  if (pgx_params_read_args(2, argv, params) != PGX_SUCCESS || params[11] != 30.0) return 2;
  if (pgx_build_levels('L', 1, rp, NULL, &nlev, lp, order) != PGX_SUCCESS || nlev != 1) return 3;
  g = pgx_hypre_gemslr_create();
  if (!g || pgx_hypre_gemslr_destroy(g) != PGX_SUCCESS) return 4;
  printf("version %d\n", pgx_version());
  return 0;
}
''')
    exe = str(tmp_path / "host")
    lib = os.path.dirname(_abi.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", exe, "-L", lib, "-lpgx", f"-Wl,-rpath,{lib}"], check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "version 200", (out.returncode, out.stdout, out.stderr)
