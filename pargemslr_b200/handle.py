"""Device solve handle: the Python face of the pgx_gemslr_* C ABI."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from .structures import GemslrStructures

_initialized_device: Optional[int] = None


def _result(res) -> dict:
    return {"iters": res.iters, "rel_res": res.rel_res, "true_rel_res": res.true_rel_res,
            "solve_ms": res.solve_ms, "status": res.status, "launches": res.launches}


def init(device: int = 0) -> None:
    global _initialized_device
    if _initialized_device != device:
        _abi.check(_abi.lib().pgx_init(device))
        _initialized_device = device


def _precision_code(precision: str, cplx: bool) -> int:
    """The C ABI's precision code: FP64 or mixed, over real or complex values."""
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"unknown precision {precision!r}")
    if cplx:
        return _abi.PRECISION_COMPLEX_FP64 if precision == "fp64" else _abi.PRECISION_COMPLEX_MIXED
    return _abi.PRECISION_FP64 if precision == "fp64" else _abi.PRECISION_MIXED


def import_structures(st: GemslrStructures, precision: str = "fp64") -> C.c_void_p:
    """A handle holding the structures, set level by level (pgx_gemslr_create / set_*), not yet committed
    to the device; the caller commits or destroys it."""
    prec = _precision_code(precision, st.complex)
    L = _abi.lib()
    h = C.c_void_p()
    _abi.check(L.pgx_gemslr_create(C.byref(h), st.n, prec))
    keep: list = []
    try:
        A = _abi.csr_struct(*st.A, keep=keep)
        _abi.check(L.pgx_gemslr_set_matrix(h, C.byref(A)))
        pp = np.ascontiguousarray(st.pperm, np.int32)
        qp = None if st.qperm is None else np.ascontiguousarray(st.qperm, np.int32)
        keep.extend([pp, qp])
        _abi.check(L.pgx_gemslr_set_perm(h, _abi.ptr(pp), _abi.ptr(qp)))
        lp = np.ascontiguousarray(st.lev_ptr, np.int32)
        keep.append(lp)
        _abi.check(L.pgx_gemslr_set_levels(h, st.nlev, _abi.ptr(lp)))
        for l, lv in enumerate(st.levels):
            desc = _abi.Level()
            dom = np.ascontiguousarray(lv.dom_ptr, np.int32)
            dinv = _abi.doubles(lv.dinv)
            keep.extend([dom, dinv])
            desc.ncomp = lv.ncomp
            desc.dom_ptr = _abi.ptr(dom)
            desc.L = _abi.csr_struct(*lv.L, keep=keep)
            desc.U = _abi.csr_struct(*lv.U, keep=keep)
            desc.dinv = _abi.ptr(dinv)
            desc.B = _abi.csr_struct(*lv.B, keep=keep)
            if lv.E is not None:
                desc.E = _abi.csr_struct(*lv.E, keep=keep)
                desc.F = _abi.csr_struct(*lv.F, keep=keep)
            desc.rank = lv.rank
            if lv.rank > 0:
                W = _abi.doubles(lv.W)
                WH = _abi.doubles(lv.WH)
                keep.extend([W, WH])
                desc.W = _abi.ptr(W)
                desc.WH = _abi.ptr(WH)
            _abi.check(L.pgx_gemslr_set_level(h, l, C.byref(desc)))
        _abi.check(L.pgx_gemslr_set_inner(h, st.inner_enable, st.inner_maxits, st.inner_tol))
        if st.solve_option:
            _abi.check(L.pgx_gemslr_set_solve_option(h, st.solve_option))
    except Exception:
        L.pgx_gemslr_destroy(h)
        raise
    return h


class GemslrHandle:
    """GeMSLR-preconditioned FGMRES on one GPU, built from post-setup structures.

    precision: ``"fp64"`` (the reference's arithmetic) or ``"mixed"`` (FP32
    preconditioner apply inside FP64 FGMRES).  Complex structures (the
    reference's complexd instantiation) give a complex handle: complex128
    throughout, or a complex64 preconditioner inside complex128 FGMRES; its
    vectors are complex128 arrays.
    """

    def __init__(self, st: GemslrStructures, precision: str = "fp64", device: int = 0):
        init(device)
        self.n = st.n
        self.complex = st.complex
        self.precision = precision
        self._h = None
        self._h = import_structures(st, precision)
        try:
            _abi.check(_abi.lib().pgx_gemslr_commit(self._h))
        except Exception:
            _abi.lib().pgx_gemslr_destroy(self._h)
            self._h = None
            raise

    @classmethod
    def from_matrix(cls, A, params: np.ndarray, precision: str = "fp64", device: int = 0) -> "GemslrHandle":
        """Set up GeMSLR for A with this library's host setup (pgx_gemslr_setup).

        A is (rowptr, colidx, values) or a scipy-style CSR object; params is
        the reference's double[180] parameter array.
        """
        init(device)
        if hasattr(A, "indptr"):
            rp, cj, va, n = A.indptr, A.indices, A.data, A.shape[0]
        else:
            rp, cj, va = A
            n = len(rp) - 1
        keep: list = []
        Ac = _abi.csr_struct(rp, cj, va, n, n, keep=keep)
        p = np.ascontiguousarray(params, np.float64)
        prec = {"fp64": _abi.PRECISION_FP64, "mixed": _abi.PRECISION_MIXED}[precision]
        h = C.c_void_p()
        _abi.check(_abi.lib().pgx_gemslr_setup(C.byref(h), C.byref(Ac), _abi.ptr(p), prec))
        self = cls.__new__(cls)
        self.n = n
        self.complex = False
        self.precision = precision
        self._h = h
        return self

    @property
    def _dtype(self):
        return np.complex128 if getattr(self, "complex", False) else np.float64

    def close(self) -> None:
        if getattr(self, "_h", None):
            _abi.lib().pgx_gemslr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self, kdim: int) -> int:
        b = C.c_int64(0)
        _abi.check(_abi.lib().pgx_gemslr_device_bytes(self._h, kdim, C.byref(b)))
        return int(b.value)

    def solve(self, b: np.ndarray, x0: Optional[np.ndarray] = None, params: Optional[np.ndarray] = None):
        """Host-array solve; returns (x, result dict)."""
        b = np.ascontiguousarray(b, self._dtype)
        x = np.zeros(self.n, self._dtype) if x0 is None else np.array(x0, dtype=self._dtype, copy=True)
        p = None if params is None else np.ascontiguousarray(params, np.float64)
        res = _abi.Result()
        rc = _abi.lib().pgx_gemslr_solve(self._h, _abi.ptr(x), _abi.ptr(b), _abi.LOCATION_HOST, _abi.ptr(p),
                                         C.byref(res))
        _abi.check(rc)
        return x, _result(res)

    def solve_device(self, x_ptr: int, b_ptr: int, params: Optional[np.ndarray] = None):
        """Solve on device pointers (e.g. torch tensors' data_ptr())."""
        p = None if params is None else np.ascontiguousarray(params, np.float64)
        res = _abi.Result()
        _abi.check(_abi.lib().pgx_gemslr_solve(self._h, x_ptr, b_ptr, _abi.LOCATION_DEVICE, _abi.ptr(p),
                                               C.byref(res)))
        return _result(res)

    def solve_host_ptr(self, x_ptr: int, b_ptr: int, params: Optional[np.ndarray] = None):
        """Solve on host pointers (e.g. pinned torch tensors): the copies are part of the call."""
        p = None if params is None else np.ascontiguousarray(params, np.float64)
        res = _abi.Result()
        _abi.check(_abi.lib().pgx_gemslr_solve(self._h, x_ptr, b_ptr, _abi.LOCATION_HOST, _abi.ptr(p),
                                               C.byref(res)))
        return _result(res)

    def set_slots(self, nslots: int) -> None:
        """Solve slots for concurrent solves (pgx_gemslr_set_slots); slot 0 is the handle."""
        _abi.check(_abi.lib().pgx_gemslr_set_slots(self._h, nslots))

    def set_lanes(self, lanes: int) -> None:
        """Right-hand sides each additional slot advances together (1, 2 or 4; pgx_gemslr_set_lanes)."""
        _abi.check(_abi.lib().pgx_gemslr_set_lanes(self._h, lanes))

    def slot_bytes(self, kdim: int) -> int:
        """Device bytes of one additional slot for FGMRES(kdim)."""
        b = C.c_int64(0)
        _abi.check(_abi.lib().pgx_gemslr_slot_bytes(self._h, kdim, C.byref(b)))
        return int(b.value)

    def solve_batch_ptr(self, nrhs: int, x_ptr: int, ldx: int, b_ptr: int, ldb: int, location: int,
                        params: Optional[np.ndarray] = None):
        """Solve nrhs column systems spread over the slots; returns one result dict per column."""
        p = None if params is None else np.ascontiguousarray(params, np.float64)
        res = (_abi.Result * max(nrhs, 1))()
        rc = _abi.lib().pgx_gemslr_solve_batch(self._h, nrhs, x_ptr, ldx, b_ptr, ldb, location, _abi.ptr(p),
                                               C.cast(res, C.c_void_p))
        _abi.check(rc)
        return [_result(res[i]) for i in range(nrhs)]

    def solve_batch(self, B: np.ndarray, X0: Optional[np.ndarray] = None, params: Optional[np.ndarray] = None):
        """Host-array batch solve: B is (nrhs, n), one right-hand side per row; returns (X, results)."""
        B = np.ascontiguousarray(B, self._dtype)
        X = np.zeros_like(B) if X0 is None else np.array(X0, dtype=self._dtype, copy=True, order="C")
        res = self.solve_batch_ptr(B.shape[0], _abi.ptr(X), self.n, _abi.ptr(B), self.n, _abi.LOCATION_HOST,
                                   params)
        return X, res

    def server(self, params: Optional[np.ndarray] = None) -> "Server":
        """A serving loop over this handle's slots (pgx_server_*)."""
        return Server(self, params)

    def kernel_stats(self, which: int, level: int = 0, reps: int = 5):
        """(average ms, algorithmic bytes) of one building block (pgx_gemslr_kernel_stats)."""
        ms = C.c_double(0)
        b = C.c_double(0)
        _abi.check(_abi.lib().pgx_gemslr_kernel_stats(self._h, which, level, reps, C.byref(ms), C.byref(b)))
        return ms.value, b.value

    def describe(self, slot: int = 0) -> str:
        """Which kernel and layout every pass and SpMV of a slot uses (pgx_gemslr_describe)."""
        ln = C.c_int32(0)
        _abi.check(_abi.lib().pgx_gemslr_describe(self._h, slot, None, 0, C.byref(ln)))
        buf = C.create_string_buffer(ln.value + 1)
        _abi.check(_abi.lib().pgx_gemslr_describe(self._h, slot, buf, ln.value + 1, C.byref(ln)))
        return buf.value.decode()

    def residual_history(self) -> np.ndarray:
        """Relative Givens residual estimates of the last solve on the handle (FlexGmresClass::GetRelativeResidual):
        ||r0||/||b|| first, then one per iteration."""
        cnt = C.c_int32(0)
        _abi.check(_abi.lib().pgx_gemslr_residual_history(self._h, 0, None, C.byref(cnt)))
        out = np.zeros(cnt.value)
        _abi.check(_abi.lib().pgx_gemslr_residual_history(self._h, cnt.value, _abi.ptr(out), C.byref(cnt)))
        return out

    def apply(self, v: np.ndarray) -> np.ndarray:
        """z = M^-1 v (one preconditioner application) on host arrays."""
        v = np.ascontiguousarray(v, self._dtype)
        z = np.zeros(self.n, self._dtype)
        _abi.check(_abi.lib().pgx_gemslr_precond_apply(self._h, _abi.ptr(z), _abi.ptr(v), _abi.LOCATION_HOST))
        return z


class Server:
    """Serving loop over one resident preconditioned matrix (pgx_server_*).

    Requests queue in submission order; step() admits waiting requests into
    free slots and advances the in-flight solves without blocking; collect()
    returns finished (request id, result) pairs.  The arrays given to submit()
    are kept alive here until their request is collected.
    """

    def __init__(self, handle: GemslrHandle, params: Optional[np.ndarray] = None):
        self.handle = handle
        self._params = None if params is None else np.ascontiguousarray(params, np.float64)
        self._keep: dict = {}
        s = C.c_void_p()
        _abi.check(_abi.lib().pgx_server_create(handle._h, _abi.ptr(self._params), C.byref(s)))
        self._s = s

    def submit(self, x: np.ndarray, b: np.ndarray, request_id: int) -> None:
        """Queue a host-array solve; x (contiguous float64, the initial guess) receives the solution."""
        if x.dtype != np.float64 or not x.flags.c_contiguous or x.size != self.handle.n:
            raise ValueError("x must be a contiguous float64 array of length n")
        b = np.ascontiguousarray(b, np.float64)
        _abi.check(_abi.lib().pgx_server_submit(self._s, _abi.ptr(x), _abi.ptr(b), _abi.LOCATION_HOST,
                                                request_id))
        self._keep[request_id] = (x, b)

    def submit_ptr(self, x_ptr: int, b_ptr: int, location: int, request_id: int) -> None:
        """Queue a solve on raw pointers (host or device, per location)."""
        _abi.check(_abi.lib().pgx_server_submit(self._s, x_ptr, b_ptr, location, request_id))

    def step(self):
        """Advance every slot once without blocking; returns (active, queued)."""
        a = C.c_int32(0)
        q = C.c_int32(0)
        _abi.check(_abi.lib().pgx_server_step(self._s, C.byref(a), C.byref(q)))
        return a.value, q.value

    def collect(self, max_n: int = 256):
        ids = (C.c_int64 * max_n)()
        res = (_abi.Result * max_n)()
        n = C.c_int32(0)
        _abi.check(_abi.lib().pgx_server_collect(self._s, max_n, C.cast(ids, C.c_void_p),
                                                 C.cast(res, C.c_void_p), C.byref(n)))
        out = []
        for i in range(n.value):
            self._keep.pop(int(ids[i]), None)
            out.append((int(ids[i]), _result(res[i])))
        return out

    def start(self) -> None:
        """Serve on a background thread of the library (pgx_server_start): submit/collect from any thread."""
        _abi.check(_abi.lib().pgx_server_start(self._s))

    def stop(self) -> None:
        """Stop the background thread (pgx_server_stop); in-flight solves can be finished with step/run."""
        _abi.check(_abi.lib().pgx_server_stop(self._s))

    def run(self):
        """Step until the queue and the slots are empty; returns every collected (id, result)."""
        done = []
        while True:
            a, q = self.step()
            done.extend(self.collect())
            if a == 0 and q == 0:
                break
        done.extend(self.collect())
        return done

    def close(self) -> None:
        if getattr(self, "_s", None):
            _abi.lib().pgx_server_destroy(self._s)
            self._s = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
