"""The import route's refusals on the host: pgx_gemslr_create / set_* / commit and the solve side, no GPU needed.

Every structure a caller hands over is checked before anything reaches the
device, and a refusal returns the reference's error codes (101 invalid
parameter, 100 invalid option, 106 a call out of order) with a message, and
leaves the handle usable: the correct call afterwards succeeds.  The
structures are the reference's own setup of the 32x32 Laplacian
(tests/golden/lap2d_32).
"""
import ctypes as C
import os

import numpy as np
import pytest

from pargemslr_b200 import _abi
from pargemslr_b200.handle import import_structures
from pargemslr_b200.structures import from_dump

HERE = os.path.dirname(os.path.abspath(__file__))
ST = from_dump(os.path.join(HERE, "golden", "lap2d_32", "setup.bin"))
KMAX = 128
L = _abi.lib()


def _desc(lv, keep):
    d = _abi.Level()
    dom = np.ascontiguousarray(lv.dom_ptr, np.int32)
    dinv = np.ascontiguousarray(lv.dinv, np.float64)
    keep.extend([dom, dinv])
    d.ncomp = lv.ncomp
    d.dom_ptr = _abi.ptr(dom)
    d.L = _abi.csr_struct(*lv.L, keep=keep)
    d.U = _abi.csr_struct(*lv.U, keep=keep)
    d.dinv = _abi.ptr(dinv)
    d.B = _abi.csr_struct(*lv.B, keep=keep)
    if lv.E is not None:
        d.E = _abi.csr_struct(*lv.E, keep=keep)
        d.F = _abi.csr_struct(*lv.F, keep=keep)
    d.rank = lv.rank
    if lv.rank > 0:
        W = np.ascontiguousarray(lv.W, np.float64)
        WH = np.ascontiguousarray(lv.WH, np.float64)
        keep.extend([W, WH])
        d.W, d.WH = _abi.ptr(W), _abi.ptr(WH)
    return d


@pytest.fixture
def handle():
    h = C.c_void_p()
    _abi.check(L.pgx_gemslr_create(C.byref(h), ST.n, _abi.PRECISION_FP64))
    yield h
    L.pgx_gemslr_destroy(h)


def _refused(rc, code, words):
    assert rc == code, (rc, L.pgx_last_error())
    assert words in L.pgx_last_error().decode(), L.pgx_last_error()


def test_create():
    h = C.c_void_p()
    _refused(L.pgx_gemslr_create(C.byref(h), 0, 0), _abi.ERROR_INVALID_PARAM, "positive")
    _refused(L.pgx_gemslr_create(C.byref(h), 10, 7), _abi.ERROR_INVALID_OPTION, "precision")
    _refused(L.pgx_gemslr_create(None, 10, 0), _abi.ERROR_INVALID_PARAM, "null")


def test_matrix(handle):
    keep = []
    rp, cj, va, n, _ = ST.A
    _refused(L.pgx_gemslr_set_matrix(handle, C.byref(_abi.csr_struct(rp[:-1], cj, va, n - 1, n - 1, keep))),
             _abi.ERROR_INVALID_PARAM, "n x n")
    bad = cj.copy()
    bad[5] = n
    _refused(L.pgx_gemslr_set_matrix(handle, C.byref(_abi.csr_struct(rp, bad, va, n, n, keep))),
             _abi.ERROR_INVALID_PARAM, "out of range")
    _abi.check(L.pgx_gemslr_set_matrix(handle, C.byref(_abi.csr_struct(rp, cj, va, n, n, keep))))


def test_permutations(handle):
    p = np.ascontiguousarray(ST.pperm, np.int32).copy()
    q = p.copy()
    q[0] = q[1]
    _refused(L.pgx_gemslr_set_perm(handle, _abi.ptr(q), None), _abi.ERROR_INVALID_PARAM, "not a permutation")
    q = p.copy()
    q[3] = ST.n
    _refused(L.pgx_gemslr_set_perm(handle, _abi.ptr(p), _abi.ptr(q)), _abi.ERROR_INVALID_PARAM, "qperm")
    _abi.check(L.pgx_gemslr_set_perm(handle, _abi.ptr(p), None))


def test_level_pointers(handle):
    lp = np.ascontiguousarray(ST.lev_ptr, np.int32)
    _refused(L.pgx_gemslr_set_levels(handle, 0, _abi.ptr(lp)), _abi.ERROR_INVALID_PARAM, "nlev")
    short = lp.copy()
    short[-1] -= 1
    _refused(L.pgx_gemslr_set_levels(handle, ST.nlev, _abi.ptr(short)), _abi.ERROR_INVALID_PARAM, "span")
    empty = lp.copy()
    empty[1] = empty[0]
    _refused(L.pgx_gemslr_set_levels(handle, ST.nlev, _abi.ptr(empty)), _abi.ERROR_INVALID_PARAM, "empty")
    _abi.check(L.pgx_gemslr_set_levels(handle, ST.nlev, _abi.ptr(lp)))


def test_levels(handle):
    lp = np.ascontiguousarray(ST.lev_ptr, np.int32)
    _abi.check(L.pgx_gemslr_set_levels(handle, ST.nlev, _abi.ptr(lp)))
    keep = []
    lv = ST.levels[0]
    good = _desc(lv, keep)
    _refused(L.pgx_gemslr_set_level(handle, ST.nlev, C.byref(good)), _abi.ERROR_INVALID_PARAM, "out of range")
    d = _desc(lv, keep)
    d.L = _abi.csr_struct(*ST.levels[1].L, keep=keep)
    _refused(L.pgx_gemslr_set_level(handle, 0, C.byref(d)), _abi.ERROR_INVALID_PARAM, "L/U must be")
    d = _desc(lv, keep)
    d.dinv = None
    _refused(L.pgx_gemslr_set_level(handle, 0, C.byref(d)), _abi.ERROR_INVALID_PARAM, "dinv")
    d = _desc(lv, keep)
    d.E = _abi.csr_struct(*lv.F, keep=keep)
    _refused(L.pgx_gemslr_set_level(handle, 0, C.byref(d)), _abi.ERROR_INVALID_PARAM, "E must be")
    d = _desc(lv, keep)
    d.rank = KMAX + 1
    _refused(L.pgx_gemslr_set_level(handle, 0, C.byref(d)), _abi.ERROR_INVALID_PARAM, "rank")
    d = _desc(lv, keep)
    d.rank = max(lv.rank, 1)
    d.W = None
    _refused(L.pgx_gemslr_set_level(handle, 0, C.byref(d)), _abi.ERROR_INVALID_PARAM, "W/WH")
    _abi.check(L.pgx_gemslr_set_level(handle, 0, C.byref(good)))


def test_inner_settings(handle):
    _refused(L.pgx_gemslr_set_inner(handle, 1, 0, 1e-2), _abi.ERROR_INVALID_PARAM, "inner maxits")
    _refused(L.pgx_gemslr_set_inner(handle, 1, KMAX + 1, 1e-2), _abi.ERROR_INVALID_PARAM, "inner maxits")
    _abi.check(L.pgx_gemslr_set_inner(handle, 1, 5, 1e-2))
    _abi.check(L.pgx_gemslr_set_inner(handle, 0, 0, 0.0))  # off: the count is not used


def test_calls_out_of_order(handle):
    _refused(L.pgx_gemslr_commit(handle), _abi.ERROR_FUNCTION_CALL, "set_matrix")
    keep = []
    _abi.check(L.pgx_gemslr_set_matrix(handle, C.byref(_abi.csr_struct(*ST.A, keep=keep))))
    _refused(L.pgx_gemslr_commit(handle), _abi.ERROR_FUNCTION_CALL, "set_levels")
    nb = C.c_int64()
    _refused(L.pgx_gemslr_nnz(handle, C.byref(nb), None), _abi.ERROR_FUNCTION_CALL, "levels not set")
    lp = np.ascontiguousarray(ST.lev_ptr, np.int32)
    _abi.check(L.pgx_gemslr_set_levels(handle, ST.nlev, _abi.ptr(lp)))
    _refused(L.pgx_gemslr_commit(handle), _abi.ERROR_FUNCTION_CALL, "level 0 not set")
    for l, lv in enumerate(ST.levels):
        _abi.check(L.pgx_gemslr_set_level(handle, l, C.byref(_desc(lv, keep))))
    _abi.check(L.pgx_gemslr_nnz(handle, C.byref(nb), None))


def test_whole_import_succeeds_up_to_the_device():
    h = import_structures(ST)
    try:
        nb, nl = C.c_int64(), C.c_int64()
        _abi.check(L.pgx_gemslr_nnz(h, C.byref(nb), C.byref(nl)))
        assert nb.value > 0
    finally:
        L.pgx_gemslr_destroy(h)


@pytest.mark.parametrize("call", ["solve", "apply", "static", "slots", "lanes", "device_bytes", "slot_bytes", "batch",
                                  "server", "kernel_stats"])
def test_solve_side_calls_before_commit(call):
    """Every solve-side entry point refuses a handle whose structures are set but not committed (106)."""
    h = import_structures(ST)
    n = ST.n
    x, b, res = np.zeros(n), np.ones(n), _abi.Result()
    v, ms, by, s = C.c_int64(), C.c_double(), C.c_double(), C.c_void_p()
    calls = {
        "solve": lambda: L.pgx_gemslr_solve(h, _abi.ptr(x), _abi.ptr(b), 0, None, C.byref(res)),
        "apply": lambda: L.pgx_gemslr_precond_apply(h, _abi.ptr(x), _abi.ptr(b), 0),
        "static": lambda: L.pgx_gemslr_solve_static(h, _abi.ptr(x), _abi.ptr(b), 0, None, C.byref(res)),
        "slots": lambda: L.pgx_gemslr_set_slots(h, 2),
        "lanes": lambda: L.pgx_gemslr_set_lanes(h, 2),
        "device_bytes": lambda: L.pgx_gemslr_device_bytes(h, 50, C.byref(v)),
        "slot_bytes": lambda: L.pgx_gemslr_slot_bytes(h, 50, C.byref(v)),
        "batch": lambda: L.pgx_gemslr_solve_batch(h, 1, _abi.ptr(x), n, _abi.ptr(b), n, 0, None, None),
        "server": lambda: L.pgx_server_create(h, None, C.byref(s)),
        "kernel_stats": lambda: L.pgx_gemslr_kernel_stats(h, 0, 0, 1, C.byref(ms), C.byref(by)),
    }
    try:
        _refused(calls[call](), _abi.ERROR_FUNCTION_CALL, "commit")
    finally:
        L.pgx_gemslr_destroy(h)
