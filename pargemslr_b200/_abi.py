"""ctypes binding of the C ABI declared in ``include/pgx.h``.

The library is the in-tree ``pargemslr_b200/_lib/libpgx.so``.  There is no
fallback: if the library cannot be loaded, :func:`lib` raises, so a missing or
broken CUDA build fails loudly instead of silently computing elsewhere.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libpgx.so")

SUCCESS = 0
ERROR_INVALID_OPTION = 100
ERROR_INVALID_PARAM = 101
ERROR_IO = 102
ERROR_FUNCTION_CALL = 106
ERROR_MEMORY_LOCATION = 107
ERROR_CUDA = 200
ERROR_OOM = 201
ERROR_TIMEOUT = 202
ERROR_NOT_FINITE = 203
ERROR_NO_DEVICE = 204

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_COMPLEX_FP64 = 2
PRECISION_COMPLEX_MIXED = 3
LOCATION_HOST = 0
LOCATION_DEVICE = 1

# every symbol include/pgx.h declares
EXPORTS = (
    "pgx_init", "pgx_finalize", "pgx_last_error", "pgx_version",
    "pgx_gemslr_create", "pgx_gemslr_set_matrix", "pgx_gemslr_set_perm",
    "pgx_gemslr_set_levels", "pgx_gemslr_set_level", "pgx_gemslr_set_inner",
    "pgx_gemslr_commit", "pgx_gemslr_destroy", "pgx_gemslr_device_bytes",
    "pgx_gemslr_solve", "pgx_gemslr_precond_apply", "pgx_build_levels",
    "pgx_csr_spmv_device", "pgx_gemslr_setup", "pgx_gemslr_kernel_stats",
    "pgx_gemslr_set_slots", "pgx_gemslr_slot_bytes", "pgx_gemslr_solve_batch",
    "pgx_server_create", "pgx_server_submit", "pgx_server_step", "pgx_server_collect", "pgx_server_destroy",
    "pgx_gemslr_solve_static", "pgx_gemslr_set_lanes", "pgx_csr_read_mm", "pgx_csr_free",
    "pgx_server_start", "pgx_server_stop", "pgx_params_default", "pgx_params_read_file",
    "pgx_gemslr_nnz", "pgx_params_read_args", "pgx_vector_read_mm",
    "pgx_gemslr_set_wait_limit", "pgx_wait_selfcheck", "pgx_gemslr_residual_history",
    "pgx_csr_spmv_plan", "pgx_csr_spmv_device_variant", "pgx_gemslr_describe",
    "pgx_pool_create", "pgx_pool_add", "pgx_pool_submit", "pgx_pool_step", "pgx_pool_start", "pgx_pool_stop",
    "pgx_pool_collect", "pgx_pool_stats", "pgx_pool_destroy", "pgx_lowrank_block_apply_c64",
    "pgx_systems_create", "pgx_systems_solve", "pgx_systems_tune", "pgx_systems_tune_table",
    "pgx_systems_set_schedule", "pgx_systems_get_schedule", "pgx_systems_timing", "pgx_systems_device_bytes",
    "pgx_systems_last_ms", "pgx_gemslr_set_solve_option",
    "pgx_systems_destroy",
)

# every symbol include/pgx_hypre.h declares (the reference's hypre plugin interface)
HYPRE_EXPORTS = (
    "pgx_hypre_init_gpu", "pgx_hypre_finalize_gpu", "pgx_hypre_csr_matrix_create", "pgx_hypre_csr_matrix_destroy",
    "pgx_hypre_csr_matrix_view", "pgx_hypre_gemslr_create", "pgx_hypre_gemslr_destroy",
    "pgx_hypre_gemslr_set_params", "pgx_hypre_gemslr_set_precision", "pgx_hypre_gemslr_setup",
    "pgx_hypre_gemslr_solve", "pgx_hypre_gemslr_handle", "pgx_hypre_params_from_file", "pgx_hypre_params_destroy",
)


class PgxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pgx error {code}: {msg}")
        self.code = code


class Csr(C.Structure):
    _fields_ = [
        ("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int64),
        ("rowptr", C.c_void_p), ("colidx", C.c_void_p), ("values", C.c_void_p),
    ]


class Level(C.Structure):
    _fields_ = [
        ("ncomp", C.c_int32), ("dom_ptr", C.c_void_p),
        ("L", Csr), ("U", Csr), ("dinv", C.c_void_p), ("B", Csr), ("E", Csr), ("F", Csr),
        ("rank", C.c_int32), ("W", C.c_void_p), ("WH", C.c_void_p),
    ]


class Result(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("iters", C.c_int32), ("rel_res", C.c_double),
        ("true_rel_res", C.c_double), ("solve_ms", C.c_double), ("launches", C.c_int32),
    ]


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load libpgx.so (once).  Raises if it is missing: no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pargemslr_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    L.pgx_init.argtypes = [C.c_int]
    L.pgx_lowrank_block_apply_c64.argtypes = [i32, i32, i32, vp, vp, vp, C.c_int64]
    L.pgx_last_error.restype = C.c_char_p
    L.pgx_gemslr_create.argtypes = [C.POINTER(vp), i32, i32]
    L.pgx_gemslr_set_matrix.argtypes = [vp, C.POINTER(Csr)]
    L.pgx_gemslr_set_perm.argtypes = [vp, vp, vp]
    L.pgx_gemslr_set_levels.argtypes = [vp, i32, vp]
    L.pgx_gemslr_set_level.argtypes = [vp, i32, C.POINTER(Level)]
    L.pgx_gemslr_set_inner.argtypes = [vp, i32, i32, dbl]
    L.pgx_gemslr_set_solve_option.argtypes = [vp, i32]
    L.pgx_gemslr_commit.argtypes = [vp]
    L.pgx_gemslr_destroy.argtypes = [vp]
    L.pgx_gemslr_device_bytes.argtypes = [vp, i32, C.POINTER(i64)]
    L.pgx_gemslr_solve.argtypes = [vp, vp, vp, i32, vp, C.POINTER(Result)]
    L.pgx_gemslr_precond_apply.argtypes = [vp, vp, vp, i32]
    L.pgx_build_levels.argtypes = [C.c_char, i32, vp, vp, C.POINTER(i32), vp, vp]
    L.pgx_csr_spmv_device.argtypes = [C.POINTER(Csr), dbl, vp, dbl, vp]
    L.pgx_gemslr_setup.argtypes = [C.POINTER(vp), C.POINTER(Csr), vp, i32]
    L.pgx_gemslr_kernel_stats.argtypes = [vp, i32, i32, i32, C.POINTER(dbl), C.POINTER(dbl)]
    L.pgx_gemslr_set_slots.argtypes = [vp, i32]
    L.pgx_gemslr_set_lanes.argtypes = [vp, i32]
    L.pgx_csr_read_mm.argtypes = [C.c_char_p, C.POINTER(Csr)]
    L.pgx_csr_free.argtypes = [C.POINTER(Csr)]
    L.pgx_gemslr_slot_bytes.argtypes = [vp, i32, C.POINTER(i64)]
    L.pgx_gemslr_solve_batch.argtypes = [vp, i32, vp, i64, vp, i64, i32, vp, vp]
    L.pgx_server_create.argtypes = [vp, vp, C.POINTER(vp)]
    L.pgx_server_submit.argtypes = [vp, vp, vp, i32, i64]
    L.pgx_server_step.argtypes = [vp, C.POINTER(i32), C.POINTER(i32)]
    L.pgx_server_collect.argtypes = [vp, i32, vp, vp, C.POINTER(i32)]
    L.pgx_server_destroy.argtypes = [vp]
    L.pgx_server_start.argtypes = [vp]
    L.pgx_server_stop.argtypes = [vp]
    L.pgx_gemslr_solve_static.argtypes = [vp, vp, vp, i32, vp, vp]
    L.pgx_params_default.argtypes = [vp]
    L.pgx_gemslr_nnz.argtypes = [vp, C.POINTER(i64), C.POINTER(i64)]
    L.pgx_params_read_file.argtypes = [C.c_char_p, i32, vp]
    L.pgx_params_read_args.argtypes = [i32, C.POINTER(C.c_char_p), vp]
    L.pgx_vector_read_mm.argtypes = [C.c_char_p, i32, i32, vp, C.POINTER(i32)]
    L.pgx_gemslr_set_wait_limit.argtypes = [vp, i64]
    L.pgx_wait_selfcheck.argtypes = [i64, C.POINTER(i32), C.POINTER(dbl)]
    L.pgx_gemslr_residual_history.argtypes = [vp, i32, vp, C.POINTER(i32)]
    L.pgx_pool_create.argtypes = [i64, vp, C.POINTER(vp)]
    L.pgx_pool_add.argtypes = [vp, vp, C.POINTER(i32)]
    L.pgx_pool_submit.argtypes = [vp, i32, vp, vp, i32, i64]
    L.pgx_pool_step.argtypes = [vp, C.POINTER(i32), C.POINTER(i32)]
    L.pgx_pool_start.argtypes = [vp]
    L.pgx_pool_stop.argtypes = [vp]
    L.pgx_pool_collect.argtypes = [vp, i32, vp, vp, C.POINTER(i32)]
    L.pgx_pool_stats.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i32)]
    L.pgx_pool_destroy.argtypes = [vp]
    L.pgx_gemslr_describe.argtypes = [vp, i32, C.c_char_p, i32, C.POINTER(i32)]
    L.pgx_systems_create.argtypes = [C.POINTER(vp), vp, i32]
    L.pgx_systems_solve.argtypes = [vp, vp, vp, i32, vp, vp]
    L.pgx_systems_tune.argtypes = [vp, vp, i32, vp, i32, C.POINTER(dbl)]
    L.pgx_systems_tune_table.argtypes = [vp, i32, vp, C.POINTER(i32)]
    L.pgx_systems_set_schedule.argtypes = [vp, i32, i32, i32, i32]
    L.pgx_systems_get_schedule.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.pgx_systems_timing.argtypes = [vp, i32, vp, vp, vp]
    L.pgx_systems_device_bytes.argtypes = [vp, C.POINTER(i64)]
    L.pgx_systems_last_ms.argtypes = [vp, C.POINTER(dbl)]
    L.pgx_systems_destroy.argtypes = [vp]
    L.pgx_csr_spmv_plan.argtypes = [C.POINTER(Csr), C.POINTER(i32), C.POINTER(i32)]
    L.pgx_csr_spmv_device_variant.argtypes = [C.POINTER(Csr), i32, dbl, vp, dbl, vp]
    for name in EXPORTS + HYPRE_EXPORTS:
        if name != "pgx_last_error":
            getattr(L, name).restype = C.c_int
    lg = C.c_long
    L.pgx_hypre_init_gpu.argtypes = [C.c_int]
    L.pgx_hypre_finalize_gpu.argtypes = []
    L.pgx_hypre_csr_matrix_create.argtypes = [lg, lg, lg, lg, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, vp,
                                              C.c_int]
    L.pgx_hypre_csr_matrix_create.restype = vp
    L.pgx_hypre_csr_matrix_destroy.argtypes = [vp]
    L.pgx_hypre_csr_matrix_view.argtypes = [vp, C.POINTER(Csr)]
    L.pgx_hypre_gemslr_create.argtypes = []
    L.pgx_hypre_gemslr_create.restype = vp
    L.pgx_hypre_gemslr_destroy.argtypes = [vp]
    L.pgx_hypre_gemslr_set_params.argtypes = [vp, vp]
    L.pgx_hypre_gemslr_set_precision.argtypes = [vp, C.c_int]
    L.pgx_hypre_gemslr_setup.argtypes = [vp, vp, vp, vp]
    L.pgx_hypre_gemslr_solve.argtypes = [vp, vp, vp, vp]
    L.pgx_hypre_gemslr_handle.argtypes = [vp]
    L.pgx_hypre_gemslr_handle.restype = vp
    L.pgx_hypre_params_from_file.argtypes = [C.c_char_p]
    L.pgx_hypre_params_from_file.restype = C.POINTER(C.c_double)
    L.pgx_hypre_params_destroy.argtypes = [vp]
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != SUCCESS:
        msg = lib().pgx_last_error()
        raise PgxError(rc, msg.decode() if msg else "")


def ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


def doubles(a: Optional[np.ndarray]) -> Optional[np.ndarray]:
    """Values as the C ABI takes them: float64, or a complex array as interleaved {re, im} float64."""
    if a is None:
        return None
    if np.iscomplexobj(a):
        return np.ascontiguousarray(a, np.complex128).view(np.float64)
    return np.ascontiguousarray(a, np.float64)


def csr_struct(rp: Optional[np.ndarray], cj: Optional[np.ndarray], va: Optional[np.ndarray], rows: int,
               cols: int, keep: list) -> Csr:
    """A pgx_csr view over numpy arrays (kept alive through `keep`)."""
    if rp is None or rows == 0:
        return Csr(0, 0, 0, None, None, None)
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    cj = np.ascontiguousarray(cj, dtype=np.int32)
    va = doubles(va)
    keep.extend([rp, cj, va])
    return Csr(rows, cols, int(cj.size), ptr(rp), ptr(cj) if cj.size else None, ptr(va) if va.size else None)


def build_levels(uplo: str, rp: np.ndarray, cj: np.ndarray):
    """Level-set schedule of a triangular factor (pgx_build_levels)."""
    n = rp.size - 1
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    cj = np.ascontiguousarray(cj, dtype=np.int32)
    nlev = C.c_int32(0)
    lptr = np.zeros(n + 1, dtype=np.int32)
    order = np.zeros(max(n, 1), dtype=np.int32)
    check(lib().pgx_build_levels(uplo.encode(), n, ptr(rp), ptr(cj) if cj.size else None, C.byref(nlev),
                                 ptr(lptr), ptr(order)))
    return lptr[: nlev.value + 1].copy(), order[:n].copy()


INPUTS_FORMATS = {"sequential": 0, "parallel": 1, "hypre": 2}


def params_default() -> np.ndarray:
    """The default parameter array built by the library (pgx_params_default)."""
    p = np.zeros(180, dtype=np.float64)
    check(lib().pgx_params_default(ptr(p)))
    return p


def params_read_file(path: str, fmt: str, base: np.ndarray = None) -> np.ndarray:
    """`base` (default: the library's defaults) with the slots a parameter file names overwritten
    (pgx_params_read_file); fmt is "sequential", "parallel" or "hypre"."""
    p = params_default() if base is None else np.array(base, dtype=np.float64, copy=True)
    check(lib().pgx_params_read_file(path.encode(), INPUTS_FORMATS[fmt], ptr(p)))
    return p


def params_read_args(args, base: np.ndarray = None) -> np.ndarray:
    """`base` (default: the library's defaults) with a driver's -tol / -kdim / -maxits arguments applied
    (pgx_params_read_args)."""
    p = params_default() if base is None else np.array(base, dtype=np.float64, copy=True)
    argv = (C.c_char_p * max(len(args), 1))(*[a.encode() for a in args])
    check(lib().pgx_params_read_args(len(args), argv, ptr(p)))
    return p


def read_mm_vector(path: str, idxin: int = 1) -> np.ndarray:
    """A vector stored as a coordinate Matrix Market file, read by the library (pgx_vector_read_mm)."""
    L = lib()
    n = C.c_int32(0)
    check(L.pgx_vector_read_mm(path.encode(), idxin, 0, None, C.byref(n)))
    x = np.zeros(n.value)
    check(L.pgx_vector_read_mm(path.encode(), idxin, n.value, ptr(x), C.byref(n)))
    return x


def read_mm(path: str):
    """(rowptr, colidx, values) of a Matrix Market file read by the library (pgx_csr_read_mm)."""
    L = lib()
    A = Csr()
    check(L.pgx_csr_read_mm(path.encode(), C.byref(A)))
    try:
        n, nnz = A.rows, A.nnz
        rp = np.ctypeslib.as_array(C.cast(A.rowptr, C.POINTER(C.c_int32)), (n + 1,)).copy()
        cj = np.ctypeslib.as_array(C.cast(A.colidx, C.POINTER(C.c_int32)), (max(nnz, 1),))[:nnz].copy()
        va = np.ctypeslib.as_array(C.cast(A.values, C.POINTER(C.c_double)), (max(nnz, 1),))[:nnz].copy()
        return rp, cj, va, (A.rows, A.cols)
    finally:
        L.pgx_csr_free(C.byref(A))
