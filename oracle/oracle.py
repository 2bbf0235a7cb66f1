"""CPU restatement of the reference GeMSLR-FGMRES solve phase — the ORACLE.

Test infrastructure: only tests/, __graft_entry__.smoke() and the CPU
baseline of bench.py use this module; the product path never does.

The numerical kernels live in restate.c (built into oracle/_build/
liboracle.so by `make -C oracle oracle`), each repeating the loop order of the
reference routine it names; this module repeats the reference's call
sequence on top of them:

  GemslrOracle.solve          GemslrClass::Solve         gemslr.cpp:3431-3472
  GemslrOracle.solve_level    GemslrClass::SolveLevel    gemslr.cpp:3474-3630
  GemslrOracle.solve_b        GemslrClass::SolveB        gemslr.cpp:3632-3678
  GemslrOracle.lowrank        SolveApplyLowRankLevel     gemslr.cpp:3681-3722
  GemslrOracle.schur_matvec   GemslrClass::SchurMatVec   gemslr.cpp:3799-3960
  GemslrOracle.schur_solve    GemslrSchurMatrixClass::Solve  gemslr.cpp:294-330
  fgmres                      FlexGmresClass::Solve      fgmres.hpp:263-558

On the reference's own post-setup structures (the PGXD dump written by
oracle/ref_driver.cpp) the results agree with the reference binary bit for
bit; tests/test_oracle.py checks that against committed golden outputs of
the reference, which pins this oracle.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from typing import Callable, Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
EPS = np.finfo(np.float64).eps

_lib = None


def build() -> str:
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    src = os.path.join(HERE, "restate.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-o", LIB, src, "-lm"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        L.oracle_csr_matvec.argtypes = [C.c_int, P, P, P, C.c_double, P, C.c_double, P]
        L.oracle_ilu_solve.argtypes = [C.c_int, P, P, P, P, P, P, P, P, P]
        L.oracle_build_levels.argtypes = [C.c_char, C.c_int, P, P, P, P]
        L.oracle_build_levels.restype = C.c_int
        L.oracle_dense_matvec_t.argtypes = [C.c_int, C.c_int, P, P, P]
        L.oracle_dense_matvec_n.argtypes = [C.c_int, C.c_int, P, P, P]
        L.oracle_dot.argtypes = [C.c_int, P, P]
        L.oracle_dot.restype = C.c_double
        L.oracle_axpy.argtypes = [C.c_int, C.c_double, P, P]
        L.oracle_scale.argtypes = [C.c_int, C.c_double, P]
        L.oracle_mgs.argtypes = [C.c_int, P, C.c_int, P, C.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class Csr:
    """CSR matrix held as three contiguous numpy arrays."""

    def __init__(self, rp, cj, va, rows: int, cols: int):
        self.rp = np.ascontiguousarray(rp, np.int32)
        self.cj = np.ascontiguousarray(cj, np.int32)
        self.va = np.ascontiguousarray(va, np.float64)
        self.rows, self.cols = rows, cols

    def matvec(self, alpha: float, x: np.ndarray, beta: float, y: np.ndarray) -> None:
        assert x.flags.c_contiguous and y.flags.c_contiguous
        if self.rows == 0:
            return
        lib().oracle_csr_matvec(self.rows, _p(self.rp), _p(self.cj), _p(self.va), alpha, _p(x), beta, _p(y))


def csr_matvec(A: Csr, alpha, x, beta, y):
    A.matvec(alpha, x, beta, y)


def ilu_solve(L: Csr, U: Csr, d: np.ndarray, rhs: np.ndarray, x: np.ndarray) -> None:
    n = L.rows
    if n == 0:
        return
    lib().oracle_ilu_solve(n, _p(L.rp), _p(L.cj), _p(L.va), _p(U.rp), _p(U.cj), _p(U.va), _p(d), _p(rhs), _p(x))


def build_levels(uplo: str, rp: np.ndarray, cj: np.ndarray):
    n = rp.size - 1
    rp = np.ascontiguousarray(rp, np.int32)
    cj = np.ascontiguousarray(cj, np.int32)
    lptr = np.zeros(n + 1, np.int32)
    order = np.zeros(max(n, 1), np.int32)
    nlev = lib().oracle_build_levels(uplo.encode(), n, _p(rp), _p(cj) if cj.size else None, _p(lptr), _p(order))
    if nlev < 0:
        raise ValueError("factor is not strictly triangular")
    return lptr[: nlev + 1].copy(), order[:n].copy()


def dot(x, y) -> float:
    return lib().oracle_dot(x.size, _p(x), _p(y))


def axpy(a: float, x, y) -> None:
    lib().oracle_axpy(x.size, a, _p(x), _p(y))


def scale(a: float, x) -> None:
    lib().oracle_scale(x.size, a, _p(x))


def norm2(x) -> float:
    return math.sqrt(abs(dot(x, x)))


def fgmres(matvec: Callable, precond: Optional[Callable], x: np.ndarray, rhs: np.ndarray, kdim: int, maxits: int,
           tol: float, absolute: bool = False) -> Dict[str, object]:
    """FlexGmresClass::Solve (fgmres.hpp:263-558), MGS without re-orthogonalisation.

    matvec(alpha, x, beta, y): y = alpha*A*x + beta*y; precond(z, v): z = M^-1 v.
    Returns iterations, the Givens relative residual and its history; x is
    updated in place.
    """
    n = x.size
    V = np.zeros((kdim + 1) * n)
    Z = np.zeros((kdim + 1) * n)
    H = np.zeros((kdim + 1) * kdim)  # column-major, leading dimension kdim+1
    ldh = kdim + 1
    c = [0.0] * kdim
    s = [0.0] * kdim
    rs = [0.0] * (kdim + 1)

    def col(M, j):
        return M[j * n:(j + 1) * n]

    def h(i, j):
        return H[i + j * ldh]

    def set_h(i, j, v):
        H[i + j * ldh] = v

    normb = norm2(rhs)
    if normb < EPS:
        x[:] = 0.0
        return {"iters": 0, "rel_res": 0.0, "hist": [1.0]}
    v = col(V, 0)
    v[:] = rhs
    matvec(-1.0, x, 1.0, v)
    normr = norm2(v)
    if normr < EPS:
        return {"iters": 0, "rel_res": 0.0, "hist": [1.0]}
    tolr = tol if absolute else tol * normb
    hist = [normr / normb]
    r0 = normr
    sines = []  # the Givens sine of every iteration, in order
    it = 0
    i = 0
    broke = False
    while it < maxits:
        rs[0] = normr
        scale(1.0 / normr, col(V, 0))
        i = 0
        while i < kdim and it < maxits:
            i += 1
            it += 1
            vv, z, w = col(V, i - 1), col(Z, i - 1), col(V, i)
            if precond is not None:
                precond(z, vv)
                matvec(1.0, z, 0.0, w)
            else:
                z[:] = vv
                matvec(1.0, vv, 0.0, w)
            lib().oracle_mgs(n, _p(V), i - 1, _p(H), ldh)
            for j in range(1, i):
                hii = h(j - 1, i - 1)
                set_h(j - 1, i - 1, c[j - 1] * hii + s[j - 1] * h(j, i - 1))
                set_h(j, i - 1, -s[j - 1] * hii + c[j - 1] * h(j, i - 1))
            hii = h(i - 1, i - 1)
            hii1 = h(i, i - 1)
            gam = math.sqrt(abs(hii) * abs(hii) + abs(hii1) * abs(hii1))
            if abs(gam) < EPS:
                broke = True
                break
            c[i - 1] = hii / gam
            s[i - 1] = hii1 / gam
            sines.append(s[i - 1])
            rs[i] = -s[i - 1] * rs[i - 1]
            rs[i - 1] = c[i - 1] * rs[i - 1]
            set_h(i - 1, i - 1, c[i - 1] * hii + s[i - 1] * hii1)
            normr = abs(rs[i])
            hist.append(normr / normb)
            if normr <= tolr:
                break
        if broke:
            break
        rs[i - 1] /= h(i - 1, i - 1)
        for k in range(i - 2, -1, -1):
            for j in range(k + 1, i):
                rs[k] -= h(k, j) * rs[j]
            rs[k] /= h(k, k)
        for j in range(i):
            axpy(rs[j], col(Z, j), x)
        if normr <= tolr:
            break
        v = col(V, 0)
        v[:] = rhs
        w = col(V, i)
        matvec(1.0, x, 0.0, w)
        axpy(-1.0, w, v)
    return {"iters": it, "rel_res": normr / normb, "hist": hist, "r0": r0, "normb": normb, "givens_s": sines}


class GemslrOracle:
    """The reference's GeMSLR solve phase on a PGXD setup dump."""

    def __init__(self, setup: Dict[str, np.ndarray]):
        d = setup
        self.n = int(d["n"][0])
        self.nlev = int(d["nlev"][0])
        self.lev_ptr = d["lev_ptr"].astype(np.int64)
        self.pperm = d["pperm"].astype(np.int64)
        self.qperm = d["qperm"].astype(np.int64) if d["qperm"].size else None
        self.A = self._csr(d, "A")
        self.inner = int(d["inner.enable"][0]) != 0
        self.inner_maxits = int(d["inner.maxits"][0])
        self.inner_tol = float(d["inner.tol"][0])
        # solve option 1, the U solve (gemslr.cpp:3527-3532): in the solve phase a
        # level skips its block-L part and starts from z = rhs
        self.usolve = "solve_option" in d and int(d["solve_option"][0]) == 1
        # solve option 2, the multiplicative solve of ParallelGemslrClass
        # (SolveLevelGemslrMul, parallel_gemslr.cpp:5816-6050), with the inner
        # iteration on the RAP operator (RAPMatVec, parallel_gemslr.cpp:7194)
        self.mul = "solve_option" in d and int(d["solve_option"][0]) == 2
        self.lv: List[dict] = []
        for l in range(self.nlev):
            pre = f"L{l}."
            ncomp = int(d[pre + "ncomp"][0])
            lv = {"ncomp": ncomp, "dom": d[pre + "dom_ptr"].astype(np.int64), "L": [], "U": [], "D": [], "B": []}
            for c in range(ncomp):
                pc = f"{pre}B{c}."
                lv["L"].append(self._csr(d, pc + "L"))
                lv["U"].append(self._csr(d, pc + "U"))
                lv["D"].append(np.ascontiguousarray(d[pc + "D"], np.float64))
                lv["B"].append(self._csr(d, pc + "A"))
            if l < self.nlev - 1:
                lv["E"] = self._csr(d, pre + "E")
                lv["F"] = self._csr(d, pre + "F")
                lv["lrc"] = int(d[pre + "lrc"][0])
                if lv["lrc"] > 0:
                    lv["W"] = np.ascontiguousarray(d[pre + "W"], np.float64)
                    lv["WH"] = np.ascontiguousarray(d[pre + "WH"], np.float64)
            m = self.n - int(self.lev_ptr[l])
            lv["z"] = np.zeros(m)
            lv["w"] = np.zeros(m)
            lv["v"] = np.zeros(m)
            lv["xlr"] = np.zeros(self.n - int(self.lev_ptr[l + 1]))
            self.lv.append(lv)

    @staticmethod
    def _csr(d, name) -> Csr:
        shape = d[name + ".shape"]
        return Csr(d[name + ".i"], d[name + ".j"], d[name + ".a"], int(shape[0]), int(shape[1]))

    # -------------------------------------------------------------- solve
    def solve(self, rhs: np.ndarray) -> np.ndarray:
        """z = M^-1 rhs (GemslrClass::Solve)."""
        rhs_t = np.ascontiguousarray(rhs[self.pperm])       # GatherPerm
        x_t = np.zeros(self.n)
        if self.mul:
            self.solve_level_mul(x_t, rhs_t, 0)
        else:
            self.solve_level(x_t, rhs_t, 0)
        out = np.empty(self.n)
        out[self.qperm if self.qperm is not None else self.pperm] = x_t  # ScatterRperm
        return out

    def solve_b(self, x: np.ndarray, rhs: np.ndarray, level: int) -> None:
        lv = self.lv[level]
        start = int(self.lev_ptr[level])
        for c in range(lv["ncomp"]):
            a, b = int(lv["dom"][c]) - start, int(lv["dom"][c + 1]) - start
            ilu_solve(lv["L"][c], lv["U"][c], lv["D"][c], rhs[a:b], x[a:b])

    def lowrank(self, out: np.ndarray, rhs: np.ndarray, level: int) -> None:
        lv = self.lv[level]
        m, r = rhs.size, lv["lrc"]
        t = np.zeros(r)
        lib().oracle_dense_matvec_t(m, r, _p(lv["W"]), _p(rhs), _p(t))
        lib().oracle_dense_matvec_n(m, r, _p(lv["WH"]), _p(t), _p(out))

    def solve_level(self, x: np.ndarray, rhs: np.ndarray, level: int) -> None:
        if level == self.nlev - 1:
            self.solve_b(x, rhs, level)
            return
        lv = self.lv[level]
        nl = int(self.lev_ptr[level + 1] - self.lev_ptr[level])
        rhsu, rhsl = rhs[:nl], rhs[nl:]
        xu, xl = x[:nl], x[nl:]
        zu, zl = lv["z"][:nl], lv["z"][nl:]
        if self.usolve:
            zl[:] = rhsl
        else:
            self.solve_b(zu, rhsu, level)
            lv["E"].matvec(-1.0, zu, 0.0, zl)
            axpy(1.0, rhsl, zl)
        if self.inner and level == 0:
            xl[:] = 0.0
            fgmres(self.schur_matvec, self.schur_solve, xl, zl, self.inner_maxits, self.inner_maxits, self.inner_tol)
        else:
            if lv["lrc"] > 0:
                self.lowrank(lv["xlr"], zl, level)
                axpy(1.0, lv["xlr"], zl)
            self.solve_level(xl, zl, level + 1)
        lv["F"].matvec(-1.0, xl, 0.0, zu)
        axpy(1.0, rhsu, zu)
        self.solve_b(xu, zu, level)

    def b_matvec(self, level: int, alpha: float, x: np.ndarray, beta: float, y: np.ndarray) -> None:
        """y = alpha B_l x + beta y over the level's subdomain blocks (BMatVec)."""
        lv = self.lv[level]
        start = int(self.lev_ptr[level])
        for c in range(lv["ncomp"]):
            a, b = int(lv["dom"][c]) - start, int(lv["dom"][c + 1]) - start
            yc = np.ascontiguousarray(y[a:b])
            lv["B"][c].matvec(alpha, np.ascontiguousarray(x[a:b]), beta, yc)
            y[a:b] = yc

    def solve_level_mul(self, x: np.ndarray, rhs: np.ndarray, level: int) -> None:
        """ParallelGemslrClass::SolveLevelGemslrMul (parallel_gemslr.cpp:5816-6050): the smoothing
        x_u = B^-1 b_u, the residual r = b - A [x_u; 0], its restriction r_l - E B^-1 r_u, the Schur solve
        (inner FGMRES on RAP at level 0, else low rank and the next level) and x = x + [-B^-1 F; I] x_l."""
        if level == self.nlev - 1:
            self.solve_b(x, rhs, level)
            return
        lv = self.lv[level]
        nl = int(self.lev_ptr[level + 1] - self.lev_ptr[level])
        rhsu, rhsl = rhs[:nl], rhs[nl:]
        xu, xl = x[:nl], x[nl:]
        y = np.zeros(x.size)
        z = np.zeros(x.size)
        yu, zu, zl = y[:nl], z[:nl], z[nl:]
        self.solve_b(xu, rhsu, level)                      # 1. x_u = B^-1 b_u
        zu[:] = rhsu                                       # 2. z = b - A [x_u; 0]
        self.b_matvec(level, -1.0, xu, 1.0, zu)
        zl[:] = rhsl
        lv["E"].matvec(-1.0, xu, 1.0, zl)
        self.solve_b(yu, zu, level)                        # 3. z_l -= E B^-1 z_u
        lv["E"].matvec(-1.0, yu, 1.0, zl)
        if self.inner and level == 0:                      # 4. Schur solve
            xl[:] = 0.0
            fgmres(self.rap_matvec, self.schur_solve, xl, zl, self.inner_maxits, self.inner_maxits, self.inner_tol)
        else:
            if lv["lrc"] > 0:
                self.lowrank(lv["xlr"], zl, level)
                axpy(1.0, lv["xlr"], zl)
            self.solve_level_mul(xl, zl, level + 1)
        lv["F"].matvec(-1.0, xl, 0.0, yu)                  # 5. x_u += -B^-1 F x_l
        self.solve_b(zu, yu, level)
        axpy(1.0, zu, xu)

    def rap_matvec(self, alpha: float, x: np.ndarray, beta: float, y: np.ndarray) -> None:
        """y = alpha R A P x + beta y at level 0 (RAPMatVec, parallel_gemslr.cpp:7194): P x = [-B^-1 F x; x],
        A P x through B, F, E and C, R = [-E B^-1, I]."""
        level = 0
        lv = self.lv[level]
        nl = int(self.lev_ptr[level + 1] - self.lev_ptr[level])
        vu = np.zeros(nl)
        wu = np.zeros(nl)
        vl = np.array(x, copy=True)
        lv["F"].matvec(-1.0, x, 0.0, wu)
        self.solve_b(vu, wu, level)
        self.b_matvec(level, 1.0, vu, 0.0, wu)
        lv["F"].matvec(1.0, vl, 1.0, wu)
        wl = np.zeros(x.size)
        lv["E"].matvec(1.0, vu, 0.0, wl)
        wl += self.c_matvec(vl)
        self.solve_b(vu, wu, level)
        lv["E"].matvec(-alpha, vu, beta, y)
        axpy(alpha, wl, y)

    def c_matvec(self, x: np.ndarray) -> np.ndarray:
        """C_0 x: the blocks of the levels below level 0 (CMatVec)."""
        level = 0
        n_start = int(self.lev_ptr[level])
        nl = int(self.lev_ptr[level + 1] - self.lev_ptr[level])
        w = np.zeros(self.n - n_start)
        for j in range(level + 1, self.nlev):
            lj = self.lv[j]
            sj = int(self.lev_ptr[j])
            ej = int(self.lev_ptr[j + 1])
            for c in range(lj["ncomp"]):
                a, b = int(lj["dom"][c]), int(lj["dom"][c + 1])
                xi = x[a - n_start - nl:b - n_start - nl]
                zi = np.ascontiguousarray(w[a - n_start:b - n_start])
                lj["B"][c].matvec(1.0, np.ascontiguousarray(xi), 1.0, zi)
                w[a - n_start:b - n_start] = zi
            if j == self.nlev - 1:
                break
            nli = ej - sj
            ziu = np.ascontiguousarray(w[sj - n_start:sj - n_start + nli])
            lj["F"].matvec(1.0, np.ascontiguousarray(x[ej - n_start - nl:]), 1.0, ziu)
            w[sj - n_start:sj - n_start + nli] = ziu
            zil = np.ascontiguousarray(w[ej - n_start:])
            lj["E"].matvec(1.0, np.ascontiguousarray(x[sj - n_start - nl:sj - n_start - nl + nli]), 1.0, zil)
            w[ej - n_start:] = zil
        return w[nl:]

    def schur_solve(self, x: np.ndarray, rhs: np.ndarray) -> None:
        lv = self.lv[0]
        if lv["lrc"] > 0:
            self.lowrank(lv["xlr"], rhs, 0)
            axpy(1.0, rhs, lv["xlr"])
            self.solve_level(x, lv["xlr"], 1)
        else:
            self.solve_level(x, rhs, 1)

    def schur_matvec(self, alpha: float, x: np.ndarray, beta: float, y: np.ndarray) -> None:
        level = 0
        lv = self.lv[level]
        n_start = int(self.lev_ptr[level])
        nl = int(self.lev_ptr[level + 1] - self.lev_ptr[level])
        worku = lv["v"][:nl]
        zu, zl = lv["w"][:nl], lv["w"][nl:]
        lv["F"].matvec(1.0, x, 0.0, zu)
        self.solve_b(worku, zu, level)
        lv["E"].matvec(-alpha, worku, beta, y)
        zl[:] = 0.0
        for j in range(level + 1, self.nlev):
            lj = self.lv[j]
            sj = int(self.lev_ptr[j])
            ej = int(self.lev_ptr[j + 1])
            for c in range(lj["ncomp"]):
                a, b = int(lj["dom"][c]), int(lj["dom"][c + 1])
                xi = x[a - n_start - nl:b - n_start - nl]
                zi = lv["w"][a - n_start:b - n_start]
                lj["B"][c].matvec(1.0, np.ascontiguousarray(xi), 1.0, zi)
            if j == self.nlev - 1:
                break
            nli = ej - sj
            xil = x[ej - n_start - nl:]
            ziu = lv["w"][sj - n_start:sj - n_start + nli]
            lj["F"].matvec(1.0, xil, 1.0, ziu)
            xiu = x[sj - n_start - nl:sj - n_start - nl + nli]
            zil = lv["w"][ej - n_start:]
            lj["E"].matvec(1.0, xiu, 1.0, zil)
        axpy(alpha, zl, y)

    def matvec_a(self, alpha: float, x: np.ndarray, beta: float, y: np.ndarray) -> None:
        self.A.matvec(alpha, x, beta, y)

    def fgmres_solve(self, b: np.ndarray, kdim: int, maxits: int, tol: float, absolute: bool = False):
        """FlexGmres + GeMSLR from x0 = 0: returns (x, result)."""
        x = np.zeros(self.n)

        def precond(z, v):
            z[:] = self.solve(v)

        res = fgmres(self.matvec_a, precond, x, np.ascontiguousarray(b, np.float64), kdim, maxits, tol, absolute)
        return x, res
