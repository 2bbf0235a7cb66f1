"""GPU parity of the solve on the reference's ParallelGemslrClass setup (one rank), the class the
reference's parallel drivers and config 2 use.

The reference (oracle/_ref/pgx_ref_driver_par) sets up ParallelGemslrClass, solves b = A x_true with
FlexGmresClass from x0 = 0 and exports its structures with each level's transfer permutation; they are
composed into one permutation (structures.from_parallel_dump) and imported through the C ABI.  Bars as
for GemslrClass: FP64 iterations within +-1, x within 1e-6 of the reference's, true relative residual
<= 1e-8; mixed at most 15% (plus one) more iterations.
"""
import numpy as np
import pytest

from pargemslr_b200 import params as P
from pargemslr_b200.structures import from_parallel_dump
from tests import oracle_runs

pytestmark = pytest.mark.gpu

CASES = {
    "lap3d_32_gemslr": ((32, 32, 32, 0.0, 0.0, 0.0, 0.0), "lap3d_128", 2),
    # the headline's parameters (4 levels, ILUT 1e-3/200, rank 16, inner Schur FGMRES) at 64^3
    "lap3d_64_gemslr": ((64, 64, 64, 0.0, 0.0, 0.0, 0.0), "lap3d_128", 2),
    "lap3d_32_bj": ((32, 32, 32, 0.0, 0.0, 0.0, 0.0), "lap3d_128", 0),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_on_parallel_setup_matches_reference(name, precision):
    import os
    from pargemslr_b200.handle import GemslrHandle
    if not oracle_runs.available_parallel():
        pytest.fail("oracle/_ref/pgx_ref_driver_par is missing (build it with make -C oracle)")
    lap, wl, glob = CASES[name]
    p = P.workload_params(wl)
    p[P.PRECOND_GLOBAL_PRECOND] = glob
    n = lap[0] * lap[1] * lap[2]
    ref = oracle_runs.run_parallel(lap, p, oracle_runs.x_true(n, 7), threads=os.cpu_count() or 1)
    h = GemslrHandle(from_parallel_dump(ref["setup_par"]), precision=precision)
    try:
        x, res = h.solve(ref["problem"]["b"], params=p)
        assert res["status"] == 0 and res["true_rel_res"] <= 1e-8, res
        if precision == "fp64":
            assert abs(res["iters"] - ref["iters"]) <= 1, (res["iters"], ref["iters"])
            dx = np.linalg.norm(x - ref["x"]) / np.linalg.norm(ref["x"])
            assert dx <= 1e-6, dx
        else:
            assert res["iters"] <= int(np.floor(1.15 * ref["iters"])) + 1, (res["iters"], ref["iters"])
    finally:
        h.close()
