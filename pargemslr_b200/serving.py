"""Serving pool: many resident preconditioned matrices behind one request queue and one device-memory budget.

The Python face of the pgx_pool_* C ABI.  Members are committed handles; requests name their member.  A request is
admitted when an idle slot of its member exists or a new slot (work space and FGMRES(kdim) Krylov basis) fits the
budget, after releasing idle slots of other members if need be; otherwise it waits.  Admission is first fit in
arrival order.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _abi
from .handle import GemslrHandle, _result


class Pool:
    def __init__(self, budget_bytes: int, params: Optional[np.ndarray] = None):
        self._params = None if params is None else np.ascontiguousarray(params, np.float64)
        p = C.c_void_p()
        _abi.check(_abi.lib().pgx_pool_create(int(budget_bytes), _abi.ptr(self._params), C.byref(p)))
        self._p = p
        self._members: List[GemslrHandle] = []
        self._keep: Dict[int, Tuple[np.ndarray, np.ndarray]] = {}

    def add(self, handle: GemslrHandle) -> int:
        """Make a committed handle a member; returns its index (PgxError ERROR_OOM if its factors do not fit)."""
        idx = C.c_int32(-1)
        _abi.check(_abi.lib().pgx_pool_add(self._p, handle._h, C.byref(idx)))
        self._members.append(handle)
        return idx.value

    def submit(self, index: int, x: np.ndarray, b: np.ndarray, request_id: int) -> None:
        """Queue a host-array solve for member `index`; x (contiguous float64, the initial guess) receives the
        solution.  The arrays are kept alive here until the request is collected."""
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("x must be a contiguous float64 array")
        b = np.ascontiguousarray(b, np.float64)
        _abi.check(_abi.lib().pgx_pool_submit(self._p, index, _abi.ptr(x), _abi.ptr(b), _abi.LOCATION_HOST,
                                              request_id))
        self._keep[request_id] = (x, b)

    def submit_ptr(self, index: int, x_ptr: int, b_ptr: int, location: int, request_id: int) -> None:
        _abi.check(_abi.lib().pgx_pool_submit(self._p, index, x_ptr, b_ptr, location, request_id))

    def step(self) -> Tuple[int, int]:
        a, q = C.c_int32(0), C.c_int32(0)
        _abi.check(_abi.lib().pgx_pool_step(self._p, C.byref(a), C.byref(q)))
        return a.value, q.value

    def collect(self, max_n: int = 1024):
        ids = (C.c_int64 * max_n)()
        res = (_abi.Result * max_n)()
        n = C.c_int32(0)
        _abi.check(_abi.lib().pgx_pool_collect(self._p, max_n, C.cast(ids, C.c_void_p), C.cast(res, C.c_void_p),
                                               C.byref(n)))
        out = []
        for i in range(n.value):
            self._keep.pop(int(ids[i]), None)
            out.append((int(ids[i]), _result(res[i])))
        return out

    def start(self) -> None:
        _abi.check(_abi.lib().pgx_pool_start(self._p))

    def stop(self) -> None:
        _abi.check(_abi.lib().pgx_pool_stop(self._p))

    def stats(self) -> Dict[str, int]:
        used, peak, slots = C.c_int64(0), C.c_int64(0), C.c_int32(0)
        _abi.check(_abi.lib().pgx_pool_stats(self._p, C.byref(used), C.byref(peak), C.byref(slots)))
        return {"bytes_in_use": used.value, "peak_bytes": peak.value, "slots": slots.value}

    def run(self):
        """Step until nothing is queued or in flight; returns every collected (id, result)."""
        done = []
        while True:
            a, q = self.step()
            done.extend(self.collect())
            if a == 0 and q == 0:
                break
        done.extend(self.collect())
        return done

    def close(self) -> None:
        if getattr(self, "_p", None):
            _abi.lib().pgx_pool_destroy(self._p)
            self._p = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
