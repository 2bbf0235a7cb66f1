"""Runs of the reference solver (the oracle) for the parity tests.

The reference ParGeMSLR CPU solver is built by oracle/Makefile into
oracle/_ref/ (pgx_ref_driver + libpargemslr_ref.so).  This helper runs it on
a problem and returns its setup dump, its preconditioner applications and its
FGMRES solution, cached per (problem, parameters) in a temporary directory.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import tempfile
from typing import Dict, Optional

import numpy as np

from pargemslr_b200 import pgxd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "pgx_ref_driver")
CACHE = os.path.join(tempfile.gettempdir(), "pgx_oracle_cache")


def available() -> bool:
    return os.path.exists(DRIVER)


def param_args(p: np.ndarray):
    out = []
    for i, v in enumerate(p):
        out += ["--param", f"{i}={float(v)!r}"]
    return out


def _file_digest(path: Optional[str]) -> Optional[str]:
    if path is None:
        return None
    with open(path, "rb") as f:
        return hashlib.sha1(f.read()).hexdigest()


def run(lap=None, csr_file: Optional[str] = None, params: Optional[np.ndarray] = None, xtrue: Optional[np.ndarray] = None,
        apply_k: int = 0, solve: bool = True, dump: bool = True, threads: int = 1, tag: str = "",
        rhs_file: Optional[str] = None) -> Dict[str, object]:
    """Run the reference once; returns paths and parsed results."""
    key = hashlib.sha1(repr((lap, _file_digest(csr_file), None if params is None else params.tobytes(),
                             None if xtrue is None else xtrue.tobytes(), apply_k, solve, dump, threads, tag,
                             _file_digest(rhs_file), _file_digest(DRIVER)))
                       .encode()).hexdigest()[:16]
    out = os.path.join(CACHE, key)
    done = os.path.join(out, "result.txt")
    if not os.path.exists(done):
        os.makedirs(out, exist_ok=True)
        cmd = [DRIVER, "--out", out, "--threads", str(threads)]
        if lap is not None:
            cmd += ["--lap", *[str(v) for v in lap]]
        else:
            cmd += ["--csr", csr_file]
        if rhs_file is not None:
            cmd += ["--rhs", rhs_file]
        elif xtrue is not None:
            xf = os.path.join(out, "xtrue.bin")
            pgxd.write(xf, {"x_true": np.ascontiguousarray(xtrue, np.float64)})
            cmd += ["--xtrue", xf]
        if params is not None:
            cmd += param_args(params)
        if dump:
            cmd.append("--dump")
        if solve:
            cmd.append("--solve")
        if apply_k:
            cmd += ["--apply", str(apply_k)]
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
        subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL)
    res: Dict[str, object] = {"dir": out}
    with open(done) as f:
        for line in f:
            k, v = line.strip().split("=", 1)
            if "," in v:
                res[k] = [float(t) for t in v.split(",")]
            else:
                res[k] = float(v) if any(c in v for c in ".e") else int(v)
    res["setup"] = os.path.join(out, "setup.bin") if dump else None
    res["problem"] = os.path.join(out, "problem.bin")
    if solve:
        res["solution"] = pgxd.read(os.path.join(out, "solution.bin"))
    if apply_k:
        res["apply"] = pgxd.read(os.path.join(out, "apply.bin"))
    return res


def x_true(n: int, seed: int) -> np.ndarray:
    """x_true = 2u - 1, u ~ U[0,1) from a seeded generator (the workloads' solution)."""
    rng = np.random.default_rng(seed)
    return 2.0 * rng.random(n) - 1.0


DRIVER_Z = os.path.join(ROOT, "oracle", "_ref", "pgx_ref_driver_z")


def available_complex() -> bool:
    return os.path.exists(DRIVER_Z)


def complex_rhs(n: int, nrhs: int, seed: int) -> np.ndarray:
    """nrhs seeded complex-Gaussian right-hand sides (real and imaginary parts ~ N(0,1)), one per row."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nrhs, n)) + 1j * rng.standard_normal((nrhs, n))


def run_complex(lap, params: np.ndarray, B: np.ndarray, apply_k: int = 0, threads: int = 1,
                tag: str = "") -> Dict[str, object]:
    """Run the reference over complexd (pgx_ref_driver_z) on the complex shifted Laplacian
    lap = (nx, ny, nz, shift_re, shift_im, ax, ay, az): setup dump, one FGMRES solve per row of B
    from x0 = 0, and apply_k preconditioner applications.  Cached like run()."""
    B = np.ascontiguousarray(B, np.complex128)
    key = hashlib.sha1(repr((lap, params.tobytes(), B.tobytes(), apply_k, threads, tag, _file_digest(DRIVER_Z)))
                       .encode()).hexdigest()[:16]
    out = os.path.join(CACHE, "z" + key)
    done = os.path.join(out, "result.txt")
    if not os.path.exists(done):
        os.makedirs(out, exist_ok=True)
        rf = os.path.join(out, "rhs.bin")
        pgxd.write(rf, {"B": B.view(np.float64).ravel(), "nrhs": np.array([B.shape[0]], np.int32)})
        cmd = [DRIVER_Z, "--out", out, "--threads", str(threads), "--lap", *[str(v) for v in lap], "--rhs", rf,
               "--dump", "--solve"] + param_args(params)
        if apply_k:
            cmd += ["--apply", str(apply_k)]
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
        subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL)
    res: Dict[str, object] = {"dir": out, "setup": os.path.join(out, "setup.bin")}
    with open(done) as f:
        for line in f:
            k, v = line.strip().split("=", 1)
            res[k] = v
    res["iters"] = [int(t) for t in str(res["iters"]).split(",")]
    res["true_rel_res"] = [float(t) for t in str(res["true_rel_res"]).split(",")]
    sol = pgxd.read(os.path.join(out, "solution.bin"))
    res["x"] = [sol["x%d" % r].view(np.complex128) for r in range(B.shape[0])]
    if apply_k:
        ap = pgxd.read(os.path.join(out, "apply.bin"))
        res["apply_in"] = ap["in"].view(np.complex128).reshape(apply_k, -1)
        res["apply_out"] = ap["out"].view(np.complex128).reshape(apply_k, -1)
    return res


DRIVER_PAR = os.path.join(ROOT, "oracle", "_ref", "pgx_ref_driver_par")


def available_parallel() -> bool:
    return os.path.exists(DRIVER_PAR)


def run_parallel(lap, params: np.ndarray, xtrue: np.ndarray, apply_k: int = 0, threads: int = 1,
                 tag: str = "") -> Dict[str, object]:
    """Run the reference's ParallelGemslrClass at one rank (pgx_ref_driver_par) on the Laplacian
    lap = (nx, ny, nz, shift, ax, ay, az) with b = A xtrue: its setup dump (setup_par.bin, with the
    per-level transfer permutations), one FGMRES solve from x0 = 0 and apply_k preconditioner
    applications.  Cached like run()."""
    key = hashlib.sha1(repr((lap, params.tobytes(), np.ascontiguousarray(xtrue, np.float64).tobytes(), apply_k,
                             threads, tag, _file_digest(DRIVER_PAR))).encode()).hexdigest()[:16]
    out = os.path.join(CACHE, "p" + key)
    done = os.path.join(out, "result.txt")
    if not os.path.exists(done):
        os.makedirs(out, exist_ok=True)
        xf = os.path.join(out, "xtrue.bin")
        pgxd.write(xf, {"x_true": np.ascontiguousarray(xtrue, np.float64)})
        cmd = [DRIVER_PAR, "--out", out, "--threads", str(threads), "--lap", *[str(v) for v in lap], "--xtrue", xf,
               "--dump", "--solve"] + param_args(params)
        if apply_k:
            cmd += ["--apply", str(apply_k)]
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
        subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL)
    res: Dict[str, object] = {"dir": out, "setup_par": os.path.join(out, "setup_par.bin")}
    with open(done) as f:
        for line in f:
            k, v = line.strip().split("=", 1)
            res[k] = float(v) if any(c in v for c in ".e") else int(v)
    res["problem"] = pgxd.read(os.path.join(out, "problem.bin"))
    res["x"] = pgxd.read(os.path.join(out, "solution.bin"))["x"]
    if apply_k:
        ap = pgxd.read(os.path.join(out, "apply.bin"))
        n = res["x"].size
        res["apply_in"] = ap["in"].reshape(apply_k, n)
        res["apply_out"] = ap["out"].reshape(apply_k, n)
    return res
