"""Post-setup GeMSLR structures, as the solve phase consumes them.

``GemslrStructures`` holds exactly what GemslrClass::Setup leaves behind for
the solve (ParGeMSLR SRC/preconditioners/gemslr.cpp:1602-1711): the symmetric
permutation ``pperm`` (and ``qperm`` when unsymmetric), the level pointers
``lev_ptr``, per level the subdomain pointers and ILU factors of the block-
diagonal B_l (L strictly lower, U strictly upper, ``dinv`` the inverse
diagonal), the unfactored B_l, the coupling blocks E_l / F_l, the low-rank
bases W_l / WH_l, and the settings of the level-0 inner FGMRES.

Per-subdomain factors are concatenated block-diagonally per level here, which
is the layout the device solve uses (one level = one triangular system).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import pgxd

CsrT = Tuple[np.ndarray, np.ndarray, np.ndarray, int, int]  # rowptr, colidx, values, rows, cols


def _values(a: np.ndarray, cplx: bool) -> np.ndarray:
    """A dumped value array: doubles, or for a complex dump {re, im} pairs as complex128."""
    a = np.ascontiguousarray(a, np.float64)
    return a.view(np.complex128) if cplx else a


def empty_csr(rows: int, cols: int) -> CsrT:
    return (np.zeros(rows + 1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float64), rows, cols)


def block_diag(blocks: List[CsrT], offsets: List[int], n: int) -> CsrT:
    """Concatenate square CSR blocks on the diagonal at the given offsets."""
    rp = np.zeros(n + 1, np.int64)
    cjs, vas = [], []
    for (brp, bcj, bva, br, _), off in zip(blocks, offsets):
        rp[off + 1: off + br + 1] = np.diff(brp)
        cjs.append(bcj.astype(np.int64) + off)
        vas.append(bva)
    rp = np.cumsum(rp)
    cj = np.concatenate(cjs) if cjs else np.zeros(0, np.int64)
    dt = np.result_type(*[v.dtype for v in vas]) if vas else np.float64
    va = np.concatenate(vas).astype(dt) if vas else np.zeros(0)
    # blocks are visited in offset order, so rows come out contiguous
    return (rp.astype(np.int32), cj.astype(np.int32), va, n, n)


@dataclass
class LevelStructures:
    ncomp: int
    dom_ptr: np.ndarray           # relative to the level start, ncomp + 1 entries
    L: CsrT
    U: CsrT
    dinv: np.ndarray
    B: CsrT
    E: Optional[CsrT] = None
    F: Optional[CsrT] = None
    rank: int = 0
    W: Optional[np.ndarray] = None   # m x rank, column-major (flattened)
    WH: Optional[np.ndarray] = None


@dataclass
class GemslrStructures:
    n: int
    A: CsrT
    pperm: np.ndarray
    qperm: Optional[np.ndarray]
    lev_ptr: np.ndarray
    levels: List[LevelStructures] = field(default_factory=list)
    inner_enable: int = 1
    inner_maxits: int = 5
    inner_tol: float = 1e-2
    solve_option: int = 0  # GemslrClass solve option: 0 LU, 1 U (gemslr.hpp:120-128)

    @property
    def nlev(self) -> int:
        return len(self.levels)

    @property
    def complex(self) -> bool:
        """Complex values (the reference's complexd instantiation)."""
        return np.iscomplexobj(self.A[2])

    def nnz_factors(self) -> int:
        return int(sum(lv.L[1].size + lv.U[1].size for lv in self.levels))


def _csr(d: Dict[str, np.ndarray], name: str, cplx: bool = False) -> CsrT:
    shape = d[name + ".shape"]
    return (d[name + ".i"].astype(np.int32), d[name + ".j"].astype(np.int32), _values(d[name + ".a"], cplx),
            int(shape[0]), int(shape[1]))


def from_dump(path: str) -> GemslrStructures:
    """Load the structures a reference GemslrClass exported (PGXD container)."""
    d = pgxd.read(path)
    z = "complex" in d and int(d["complex"][0]) == 1
    n = int(d["n"][0])
    nlev = int(d["nlev"][0])
    lev_ptr = d["lev_ptr"].astype(np.int32)
    qperm = d["qperm"].astype(np.int32) if d["qperm"].size else None
    st = GemslrStructures(n=n, A=_csr(d, "A", z), pperm=d["pperm"].astype(np.int32), qperm=qperm, lev_ptr=lev_ptr,
                          inner_enable=int(d["inner.enable"][0]), inner_maxits=int(d["inner.maxits"][0]),
                          inner_tol=float(d["inner.tol"][0]),
                          solve_option=int(d["solve_option"][0]) if "solve_option" in d else 0)
    if "solve_class" not in d and st.solve_option in (2, 3):
        # GemslrClass checks only the U option (gemslr.cpp:3527): it solves 2 and 3 with the LU sequence
        st.solve_option = 0
    if st.solve_option not in (0, 1, 2):
        raise ValueError("solve option %d: the LU (0), U (1) and multiplicative (2) solves are built"
                         % st.solve_option)
    for l in range(nlev):
        pre = f"L{l}."
        ncomp = int(d[pre + "ncomp"][0])
        start, end = int(lev_ptr[l]), int(lev_ptr[l + 1])
        nl = end - start
        dom = d[pre + "dom_ptr"].astype(np.int64) - start
        offs = [int(dom[c]) for c in range(ncomp)]
        Ls, Us, Bs, Ds = [], [], [], []
        for c in range(ncomp):
            pc = f"{pre}B{c}."
            if d[pc + "rperm"].size or d[pc + "cperm"].size:
                raise ValueError("ILU factors with an internal permutation are not supported")
            Ls.append(_csr(d, pc + "L", z))
            Us.append(_csr(d, pc + "U", z))
            Bs.append(_csr(d, pc + "A", z))
            Ds.append(_values(d[pc + "D"], z))
        lv = LevelStructures(ncomp=ncomp, dom_ptr=dom.astype(np.int32), L=block_diag(Ls, offs, nl),
                             U=block_diag(Us, offs, nl), dinv=np.concatenate(Ds), B=block_diag(Bs, offs, nl))
        if l < nlev - 1:
            lv.E = _csr(d, pre + "E", z)
            lv.F = _csr(d, pre + "F", z)
            lv.rank = int(d[pre + "lrc"][0])
            if lv.rank > 0:
                lv.W = _values(d[pre + "W"], z)
                lv.WH = _values(d[pre + "WH"], z)
        st.levels.append(lv)
    return st


def _permute_rows(d: Dict[str, np.ndarray], name: str, src: np.ndarray) -> None:
    """Rows of CSR `name` reordered in place: new row p is old row src[p] (entry order within a row kept)."""
    rp, cj, va = d[name + ".i"].astype(np.int64), d[name + ".j"], d[name + ".a"]
    lens = np.diff(rp)[src]
    nrp = np.zeros(src.size + 1, np.int64)
    nrp[1:] = np.cumsum(lens)
    idx = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in src]) if src.size else np.zeros(0, np.int64)
    d[name + ".i"] = nrp.astype(np.int32)
    d[name + ".j"] = cj[idx].astype(np.int32)
    d[name + ".a"] = va[idx]


def parallel_to_sequential_dump(d: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """The structures a reference ParallelGemslrClass at one rank exported (its per-level transfer
    permutations included), rewritten as the single-permutation structures of GemslrClass.

    ParallelGemslrClass::SolveLevelGemslr (parallel_gemslr.cpp:5563-5810) permutes level l's vector by that
    level's transfer before solving it and back after.  Level l + 1 receives the trailing part of level l's
    frame, so the frames nest: composing the transfers gives one global order (pperm) in which every level's
    B block keeps its own frame, and each level's E and W (rows) and F (columns), which the reference
    applies in level l's trailing frame, are re-indexed into the composed order of the levels below.  The
    entries of a row keep their order, so every SpMV sums as the reference's does.
    """
    n = int(d["n"][0])
    nlev = int(d["nlev"][0])
    if int(d.get("lrcA", np.zeros(1))[0]) > 0:
        raise ValueError("a global low-rank correction on A is not supported")
    if int(d["global_precond"][0]) not in (0, 2):
        raise ValueError("only the block-Jacobi and GeMSLR global preconditioners are supported")
    lev_ptr = d["lev_ptr"].astype(np.int64)
    perms = [d["L%d.perm" % l].astype(np.int64) for l in range(nlev)]

    def composed(start: int, l0: int) -> np.ndarray:
        # final position (relative to `start`) -> index of the frame whose trailing part begins at `start`,
        # through the transfers of levels l0 .. nlev-1
        comp = np.arange(n - start, dtype=np.int64)
        for j in range(l0, nlev):
            o = int(lev_ptr[j]) - start
            comp[o:] = comp[o:][perms[j]]
        return comp

    out: Dict[str, np.ndarray] = {}
    for k in ("n", "nlev", "lev_ptr", "solve_option", "inner.enable", "inner.maxits", "inner.tol"):
        out[k] = d[k]
    for k in ("A.i", "A.j", "A.a", "A.shape"):
        out[k] = d[k]
    out["solve_class"] = np.array([1], np.int32)  # ParallelGemslrClass: option 2 is its multiplicative solve
    out["pperm"] = composed(0, 0).astype(np.int32)
    out["qperm"] = np.zeros(0, np.int32)
    for l in range(nlev):
        pre = "L%d." % l
        ncomp = int(d[pre + "ncomp"][0])
        out[pre + "ncomp"] = d[pre + "ncomp"]
        out[pre + "dom_ptr"] = d[pre + "dom_ptr"]
        for c in range(ncomp):
            pc = "%sB%d." % (pre, c)
            if int(d[pc + "perms"][0]) != 0:
                raise ValueError("ILU factors with an internal permutation are not supported")
            for m in ("A", "L", "U"):
                for suf in (".i", ".j", ".a", ".shape"):
                    out[pc + m + suf] = d[pc + m + suf]
            out[pc + "D"] = d[pc + "D"]
            out[pc + "rperm"] = np.zeros(0, np.int32)
            out[pc + "cperm"] = np.zeros(0, np.int32)
        if l < nlev - 1:
            comp = composed(int(lev_ptr[l + 1]), l + 1)
            inv = np.empty_like(comp)
            inv[comp] = np.arange(comp.size)
            tmp = {}
            for m in ("E", "F"):
                for suf in (".i", ".j", ".a", ".shape"):
                    tmp[pre + m + suf] = d[pre + m + suf].copy()
            _permute_rows(tmp, pre + "E", comp)
            tmp[pre + "F.j"] = inv[tmp[pre + "F.j"].astype(np.int64)].astype(np.int32)
            out.update(tmp)
            rank = int(d[pre + "lrc"][0])
            out[pre + "lrc"] = d[pre + "lrc"]
            if rank > 0:
                m_l = comp.size
                for w in ("W", "WH"):
                    W = d[pre + w].reshape(rank, m_l)  # column-major m_l x rank: one row of this array per column
                    out[pre + w] = np.ascontiguousarray(W[:, comp]).ravel()
                    out[pre + w + ".shape"] = d[pre + w + ".shape"]
    return out


def from_parallel_dump(path: str) -> GemslrStructures:
    """Load the structures a reference ParallelGemslrClass at one rank exported, in GemslrClass form."""
    seq = parallel_to_sequential_dump(pgxd.read(path))
    tmp = path + ".seq"
    pgxd.write(tmp, seq)
    try:
        return from_dump(tmp)
    finally:
        os.unlink(tmp)
