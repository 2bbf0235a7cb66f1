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
