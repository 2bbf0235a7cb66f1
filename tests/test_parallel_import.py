"""The reference's ParallelGemslrClass (the class its parallel drivers use) at one rank, imported.

ParallelGemslrClass permutes each level's vector through the level's communication helper before solving
the level and back after it (parallel_gemslr.cpp:5563-5810); GemslrClass permutes once at the top.  The
reference-side exporter (oracle/ref_driver_par.cpp) records every level's permutation, and
structures.parallel_to_sequential_dump composes them into one, re-indexing E, F, W and WH.  Here the CPU
oracle applies the composed preconditioner and must reproduce the reference's own
ParallelGemslrClass::Solve on seeded vectors: bit for bit for block Jacobi (one level), to rounding for the
multilevel GeMSLR (the low-rank dots sum over rows in the composed order).
"""
import numpy as np
import pytest

from oracle import oracle as O
from pargemslr_b200 import params as P
from pargemslr_b200 import pgxd
from pargemslr_b200.structures import from_parallel_dump, parallel_to_sequential_dump
from tests import oracle_runs

CASES = {
    # name: (nx ny nz shift ax ay az, workload, global preconditioner: 2 GeMSLR, 0 block Jacobi)
    "lap3d_16_gemslr": ((16, 16, 16, 0.0, 0.0, 0.0, 0.0), "lap3d_128", 2),
    "lap3d_20_bj": ((20, 20, 20, 0.0, 0.0, 0.0, 0.0), "lap3d_128", 0),
    "convdiff2d_48_gemslr": ((48, 48, 1, 0.0, 0.3, -0.2, 0.0), "lap2d_256", 2),
}


def _run(name):
    if not oracle_runs.available_parallel():
        pytest.fail("oracle/_ref/pgx_ref_driver_par is missing (build it with make -C oracle)")
    lap, wl, glob = CASES[name]
    p = P.workload_params(wl)
    p[P.PRECOND_GLOBAL_PRECOND] = glob
    n = lap[0] * lap[1] * lap[2]
    return oracle_runs.run_parallel(lap, p, oracle_runs.x_true(n, 7), apply_k=2), p


@pytest.mark.parametrize("name", list(CASES))
def test_composed_parallel_preconditioner_matches_reference(name):
    ref, _ = _run(name)
    seq = parallel_to_sequential_dump(pgxd.read(ref["setup_par"]))
    g = O.GemslrOracle(seq)
    for k in range(2):
        z = g.solve(ref["apply_in"][k])
        err = np.linalg.norm(z - ref["apply_out"][k]) / np.linalg.norm(ref["apply_out"][k])
        assert err <= (0.0 if int(seq["nlev"][0]) == 1 else 1e-13), err


def test_composed_structures_load_and_keep_the_level_blocks():
    ref, _ = _run("lap3d_16_gemslr")
    d = pgxd.read(ref["setup_par"])
    st = from_parallel_dump(ref["setup_par"])
    assert st.nlev == int(d["nlev"][0]) >= 2
    n = st.n
    assert sorted(st.pperm.tolist()) == list(range(n))
    # the top level's frame is the reference's first transfer
    perm0 = d["L0.perm"]
    nl0 = int(st.lev_ptr[1])
    np.testing.assert_array_equal(st.pperm[:nl0], perm0[:nl0])
    # every block's factors come through unchanged
    for l, lv in enumerate(st.levels):
        assert lv.L[3] == int(st.lev_ptr[l + 1] - st.lev_ptr[l])


def test_parallel_dump_refusals():
    ref, _ = _run("lap3d_16_gemslr")
    d = pgxd.read(ref["setup_par"])
    bad = dict(d)
    bad["lrcA"] = np.array([4], np.int32)
    with pytest.raises(ValueError, match="low-rank correction on A"):
        parallel_to_sequential_dump(bad)
    bad = dict(d)
    bad["global_precond"] = np.array([1], np.int32)
    with pytest.raises(ValueError, match="global preconditioners"):
        parallel_to_sequential_dump(bad)


@pytest.mark.parametrize("lap,workload", [((16, 16, 16, 0.0, 0.0, 0.0, 0.0), "lap3d_128"),
                                          ((48, 48, 1, 0.0, 0.3, -0.2, 0.0), "lap2d_256")])
@pytest.mark.parametrize("option,schur", [(1, 1), (2, 0), (2, 1)])
def test_solve_options_match_reference(lap, workload, option, schur):
    """The U solve (option 1, parallel_gemslr.cpp:5682) and the multiplicative solve (option 2,
    SolveLevelGemslrMul, :5816-6050; with the inner iteration on the RAP operator, RAPMatVec, :7194) of the
    reference's ParallelGemslrClass, restated by the oracle on the composed structures: the preconditioner
    applications to 1e-15 and the FGMRES solve with the same iteration count."""
    if not oracle_runs.available_parallel():
        pytest.skip("oracle/_ref/pgx_ref_driver_par is not built here")
    p = P.workload_params(workload)
    p[P.PRECOND_GLOBAL_PRECOND] = 2
    p[P.ADVANCED_GLOBAL_SOLVE] = option
    p[P.SCHUR_ENABLE] = schur
    n = lap[0] * lap[1] * lap[2]
    ref = oracle_runs.run_parallel(lap, p, oracle_runs.x_true(n, 7), apply_k=2)
    seq = parallel_to_sequential_dump(pgxd.read(ref["setup_par"]))
    g = O.GemslrOracle(seq)
    assert g.usolve == (option == 1) and g.mul == (option == 2)
    for k in range(2):
        z = g.solve(ref["apply_in"][k])
        assert np.linalg.norm(z - ref["apply_out"][k]) <= 1e-15 * np.linalg.norm(ref["apply_out"][k]) * 10
    x, r = g.fgmres_solve(ref["problem"]["b"], int(p[P.SOLVER_KDIM]), int(p[P.SOLVER_MAXITS]),
                          float(p[P.SOLVER_TOL]))
    assert r["iters"] == int(ref["iters"])
    assert np.linalg.norm(x - ref["x"]) <= 1e-13 * np.linalg.norm(ref["x"])


def test_solve_option_mapping_at_import(tmp_path):
    """GemslrClass checks only the U option (gemslr.cpp:3527), so a sequential setup run with option 2 or 3 solves
    with the LU sequence and imports as option 0; ParallelGemslrClass's option 2 is its multiplicative solve and
    imports as 2; the modified-ILU multiplicative option 3 is refused."""
    from pargemslr_b200.structures import from_dump
    if not (oracle_runs.available() and oracle_runs.available_parallel()):
        pytest.skip("reference solvers not built here")
    lap = (16, 16, 16, 0.0, 0.0, 0.0, 0.0)
    p = P.workload_params("lap3d_128")
    p[P.ADVANCED_GLOBAL_SOLVE] = 2
    seq = oracle_runs.run(lap=lap, params=p, xtrue=oracle_runs.x_true(16 ** 3, 7), solve=False)
    assert int(pgxd.read(seq["setup"])["solve_option"][0]) == 2
    assert from_dump(seq["setup"]).solve_option == 0
    p[P.PRECOND_GLOBAL_PRECOND] = 2
    par = oracle_runs.run_parallel(lap, p, oracle_runs.x_true(16 ** 3, 7))
    assert from_parallel_dump(par["setup_par"]).solve_option == 2
    d = pgxd.read(par["setup_par"])
    d["solve_option"] = np.array([3], np.int32)
    f = str(tmp_path / "opt3.bin")
    pgxd.write(f, d)
    with pytest.raises(ValueError, match="solve option 3"):
        from_parallel_dump(f)
