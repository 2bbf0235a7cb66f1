"""Many systems of uneven sizes solved by one persistent kernel launch.

The Python face of the pgx_systems_* C ABI.  A :class:`SystemsBatch` packs the
preconditioners of committed real handles (each its own matrix, levels,
factors and low-rank bases) and solves every system's FGMRES with its GeMSLR
preconditioner in ONE launch: each CTA takes the next system of a work list
ordered by estimated cost, largest first, and runs that system's whole solve.
The reference solves one system per ``FlexGmresClass::Solve`` call
(SRC/solvers/fgmres.hpp:263-558); this batch has no counterpart there.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _abi
from .handle import GemslrHandle, _result


def shard_systems(costs: Sequence[float], world: int) -> List[List[int]]:
    """Split systems over `world` GPUs so that their estimated costs balance: largest first, each to the GPU whose
    total is smallest so far (ties to the lower rank).  The split depends only on the costs, so every rank computes
    the same one and no exchange is needed; independent systems never talk to each other."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda j: (load[j], j))
        out[r].append(k)
        load[r] += float(costs[k])
    for part in out:
        part.sort()
    return out


class SystemsBatch:
    def __init__(self, handles: Sequence[GemslrHandle]):
        if not handles:
            raise ValueError("no handles")
        hs = (C.c_void_p * len(handles))(*[h._h.value if isinstance(h._h, C.c_void_p) else h._h for h in handles])
        p = C.c_void_p()
        _abi.check(_abi.lib().pgx_systems_create(C.byref(p), C.cast(hs, C.c_void_p), len(handles)))
        self._p = p
        self.count = len(handles)
        self.sizes = [h.n for h in handles]

    @staticmethod
    def _ptrs(arrays) -> C.Array:
        return (C.c_void_p * len(arrays))(*[_abi.ptr(a) if isinstance(a, np.ndarray) else int(a) for a in arrays])

    def solve(self, B: Sequence[np.ndarray], X0: Optional[Sequence[np.ndarray]] = None,
              params: Optional[np.ndarray] = None) -> Tuple[List[np.ndarray], List[dict]]:
        """Solve A_i x_i = b_i for every system from host arrays; X0 (default zeros) is the initial guess.
        Returns the solutions and one result dict per system."""
        if len(B) != self.count:
            raise ValueError(f"{len(B)} right-hand sides for {self.count} systems")
        Bc = [np.ascontiguousarray(b, np.float64) for b in B]
        X = [np.zeros(n) if X0 is None else np.array(X0[i], np.float64, copy=True) for i, n in enumerate(self.sizes)]
        for i, (b, x) in enumerate(zip(Bc, X)):
            if b.shape != (self.sizes[i],) or x.shape != (self.sizes[i],):
                raise ValueError(f"system {i}: vectors of length {self.sizes[i]} expected")
        res = (_abi.Result * self.count)()
        prm = None if params is None else np.ascontiguousarray(params, np.float64)
        _abi.check(_abi.lib().pgx_systems_solve(self._p, C.cast(self._ptrs(X), C.c_void_p),
                                                C.cast(self._ptrs(Bc), C.c_void_p), _abi.LOCATION_HOST,
                                                _abi.ptr(prm), C.cast(res, C.c_void_p)))
        return X, [_result(r) for r in res]

    def solve_ptrs(self, x_ptrs: Sequence[int], b_ptrs: Sequence[int], location: int,
                   params: Optional[np.ndarray] = None) -> List[dict]:
        """Solve with raw pointers (all host or all device memory), x holding the initial guesses."""
        res = (_abi.Result * self.count)()
        prm = None if params is None else np.ascontiguousarray(params, np.float64)
        xs = (C.c_void_p * self.count)(*[int(p) for p in x_ptrs])
        bs = (C.c_void_p * self.count)(*[int(p) for p in b_ptrs])
        _abi.check(_abi.lib().pgx_systems_solve(self._p, C.cast(xs, C.c_void_p), C.cast(bs, C.c_void_p), location,
                                                _abi.ptr(prm), C.cast(res, C.c_void_p)))
        return [_result(r) for r in res]

    def tune(self, B: Sequence[np.ndarray], params: Optional[np.ndarray] = None, stride: int = 1) -> float:
        """Run the schedule autotuner on these right-hand sides (every stride-th system of the work list); returns
        the best launch time in ms."""
        Bc = [np.ascontiguousarray(b, np.float64) for b in B]
        prm = None if params is None else np.ascontiguousarray(params, np.float64)
        best = C.c_double(0.0)
        _abi.check(_abi.lib().pgx_systems_tune(self._p, C.cast(self._ptrs(Bc), C.c_void_p), _abi.LOCATION_HOST,
                                               _abi.ptr(prm), int(stride), C.byref(best)))
        return best.value

    def tune_table(self) -> List[Tuple[int, int, int, int, float]]:
        """The candidates the last tune tried: (threads, CTAs per SM, SpMV lanes, prefetch depth, ms)."""
        rows = C.c_int32(0)
        _abi.check(_abi.lib().pgx_systems_tune_table(self._p, 0, None, C.byref(rows)))
        t = np.zeros(5 * max(rows.value, 1))
        _abi.check(_abi.lib().pgx_systems_tune_table(self._p, rows.value, _abi.ptr(t), C.byref(rows)))
        return [(int(t[5 * i]), int(t[5 * i + 1]), int(t[5 * i + 2]), int(t[5 * i + 3]), float(t[5 * i + 4]))
                for i in range(rows.value)]

    @property
    def schedule(self) -> Tuple[int, int, int, int]:
        """(threads per CTA, CTAs per SM, SpMV lanes per row, levels the triangular passes fetch ahead)."""
        a, b, c, d = C.c_int32(0), C.c_int32(0), C.c_int32(0), C.c_int32(0)
        _abi.check(_abi.lib().pgx_systems_get_schedule(self._p, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return a.value, b.value, c.value, d.value

    def set_schedule(self, threads: int, ctas_per_sm: int, lanes: int, depth: int = 2) -> None:
        _abi.check(_abi.lib().pgx_systems_set_schedule(self._p, threads, ctas_per_sm, lanes, depth))

    def timing(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Per system: start and end of its solve in the last launch (ms from the first start), and its time in
        the triangular (B-block) solves."""
        s, e, t = np.zeros(self.count), np.zeros(self.count), np.zeros(self.count)
        _abi.check(_abi.lib().pgx_systems_timing(self._p, self.count, _abi.ptr(s), _abi.ptr(e), _abi.ptr(t)))
        return s, e, t

    def last_launch_ms(self) -> float:
        """Device time of the last solve's launch (CUDA events around the kernel)."""
        ms = C.c_double(0.0)
        _abi.check(_abi.lib().pgx_systems_last_ms(self._p, C.byref(ms)))
        return ms.value

    def device_bytes(self) -> int:
        b = C.c_int64(0)
        _abi.check(_abi.lib().pgx_systems_device_bytes(self._p, C.byref(b)))
        return b.value

    def close(self) -> None:
        if getattr(self, "_p", None):
            _abi.lib().pgx_systems_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
