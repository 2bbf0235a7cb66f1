"""Regenerate the golden fixtures from the reference solver itself.

    make -C oracle REF=/root/reference/ParGeMSLR && python tests/golden/make_golden.py

Each case runs the reference ParGeMSLR CPU solver (oracle/_ref/pgx_ref_driver,
one thread; oracle/_ref/pgx_ref_driver_z for the complex cases, seeded
complex-Gaussian right-hand sides) on a small problem and keeps its outputs:
  setup.bin     post-setup GeMSLR structures (permutation, levels, ILU factors,
                BuildLevels schedules, E, F, W, WH, inner-solve settings)
  problem.bin   the matrix A and right-hand side b = A x_true
  apply.bin     two preconditioner applications z = M^-1 v on seeded v
  solution.bin  the FGMRES solution and the Givens residual history
  result.txt    iteration count and residuals
These pin the CPU restatement in oracle/ (tests/test_oracle.py) and feed the
GPU parity checks that must run without the reference binary.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from pargemslr_b200 import params as P  # noqa: E402
from tests import oracle_runs  # noqa: E402

CASES = {
    # name: (nx ny nz shift alphax alphay alphaz, workload parameters, x_true seed)
    "lap2d_32": ((32, 32, 1, 0.0, 0.0, 0.0, 0.0), "lap2d_256", 3),
    "lap3d_10": ((10, 10, 10, 0.0, 0.0, 0.0, 0.0), "lap3d_128", 5),
    "convdiff2d_24": ((24, 24, 1, 0.0, 0.3, -0.2, 0.0), "lap2d_256", 9),
}


# complex cases: (nx ny nz shift_re shift_im alphax alphay alphaz, workload parameters, seed, right-hand sides)
ZCASES = {
    "zlap3d_12": ((12, 12, 12, 0.3, 0.05, 0.0, 0.0, 0.0), "zsmall", 11, 2),
}


def main():
    for name, (lap, wl, seed, nrhs) in ZCASES.items():
        p = P.workload_params(wl)
        n = lap[0] * lap[1] * lap[2]
        B = oracle_runs.complex_rhs(n, nrhs, seed)
        r = oracle_runs.run_complex(lap, p, B, apply_k=2, tag="golden")
        dst = os.path.join(HERE, name)
        os.makedirs(dst, exist_ok=True)
        for f in ("setup.bin", "problem.bin", "apply.bin", "solution.bin", "result.txt"):
            shutil.copy(os.path.join(r["dir"], f), os.path.join(dst, f))
        with open(os.path.join(dst, "params.txt"), "w") as f:
            f.write(f"workload={wl}\nlap={' '.join(str(v) for v in lap)}\nseed={seed}\nnrhs={nrhs}\n")
        print(name, "iters", r["iters"])
    for name, (lap, wl, seed) in CASES.items() if "--complex-only" not in sys.argv else ():
        p = P.workload_params(wl)
        n = lap[0] * lap[1] * lap[2]
        r = oracle_runs.run(lap=lap, params=p, xtrue=oracle_runs.x_true(n, seed), apply_k=2, tag="golden")
        dst = os.path.join(HERE, name)
        os.makedirs(dst, exist_ok=True)
        for f in ("setup.bin", "problem.bin", "apply.bin", "solution.bin", "result.txt"):
            shutil.copy(os.path.join(r["dir"], f), os.path.join(dst, f))
        with open(os.path.join(dst, "params.txt"), "w") as f:
            f.write(f"workload={wl}\nlap={' '.join(str(v) for v in lap)}\nseed={seed}\n")
        print(name, "iters", r["iters"])


if __name__ == "__main__":
    main()
