"""The multiplicative solve (solve option 2) of the reference's ParallelGemslrClass against the reference.

SolveLevelGemslrMul (parallel_gemslr.cpp:5816-6050) smooths with B^-1, restricts the residual, solves the Schur
system (at level 0 with the inner FGMRES on the RAP operator, RAPMatVec, :7194, when the inner iteration is on) and
corrects; the setup is the reference's own, run with the option and exported with its per-level permutations.  The
FP64 preconditioner application must match the reference's to 1e-9 and the solve its iterations within +-1 and its x
within 1e-6; the mixed precision solve stays within +15% iterations.
"""
import numpy as np
import pytest

from pargemslr_b200 import params as P
from pargemslr_b200.structures import from_parallel_dump
from tests import oracle_runs

pytestmark = pytest.mark.gpu

CASES = {
    # name: (nx ny nz shift ax ay az, workload, inner Schur iteration)
    "lap3d_16_inner": ((16, 16, 16, 0.0, 0.0, 0.0, 0.0), "lap3d_128", 1),
    "convdiff2d_48_noinner": ((48, 48, 1, 0.0, 0.3, -0.2, 0.0), "lap2d_256", 0),
}


def _run(name):
    if not oracle_runs.available_parallel():
        pytest.fail("oracle/_ref/pgx_ref_driver_par is missing (build it with make -C oracle)")
    lap, wl, schur = CASES[name]
    p = P.workload_params(wl)
    p[P.PRECOND_GLOBAL_PRECOND] = 2
    p[P.ADVANCED_GLOBAL_SOLVE] = 2
    p[P.SCHUR_ENABLE] = schur
    n = lap[0] * lap[1] * lap[2]
    return oracle_runs.run_parallel(lap, p, oracle_runs.x_true(n, 7), apply_k=2), p


@pytest.mark.parametrize("name", list(CASES))
def test_multiplicative_solve_fp64_matches_reference(name):
    from pargemslr_b200.handle import GemslrHandle
    ref, p = _run(name)
    st = from_parallel_dump(ref["setup_par"])
    assert st.solve_option == 2
    h = GemslrHandle(st, precision="fp64")
    for k in range(2):
        z = h.apply(ref["apply_in"][k])
        err = np.linalg.norm(z - ref["apply_out"][k]) / np.linalg.norm(ref["apply_out"][k])
        assert err <= 1e-9, f"apply {k}: relative difference {err:.3e}"
    x, r = h.solve(ref["problem"]["b"], params=p)
    assert r["status"] == 0 and r["true_rel_res"] <= 1e-8
    assert abs(r["iters"] - ref["iters"]) <= 1, (r["iters"], ref["iters"])
    assert np.linalg.norm(x - ref["x"]) / np.linalg.norm(ref["x"]) <= 1e-6
    h.close()


@pytest.mark.parametrize("name", list(CASES))
def test_multiplicative_solve_mixed_within_budget(name):
    from pargemslr_b200.handle import GemslrHandle
    ref, p = _run(name)
    h = GemslrHandle(from_parallel_dump(ref["setup_par"]), precision="mixed")
    x, r = h.solve(ref["problem"]["b"], params=p)
    assert r["status"] == 0 and r["true_rel_res"] <= 1e-8
    assert r["iters"] <= int(np.floor(1.15 * ref["iters"])) + 1, (r["iters"], ref["iters"])
    assert np.linalg.norm(x - ref["x"]) / np.linalg.norm(ref["x"]) <= 1e-6
    h.close()
