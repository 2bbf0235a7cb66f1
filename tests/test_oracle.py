"""The CPU oracle pinned against the reference's own outputs (no GPU).

The golden fixtures in tests/golden/ were written by the reference
ParGeMSLR solver (tests/golden/make_golden.py).  The restatement in oracle/
reproduces them bit for bit on the 2D fixtures; on the 3D fixture the
level-0 Schur operator of the inner FGMRES differs from the reference in the
last bit of a few entries (8 of 221 on a probe vector), so there the bar is
a relative difference of 1e-15 and the same iteration count.  Level-set
schedules and the stencil generator must match exactly.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pargemslr_b200 import params as P
from pargemslr_b200 import pgxd, problems

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# the real cases; the complex fixtures (zlap3d_*) are the complex parity tests' (test_complex_host.py,
# test_gpu_complex.py)
CASES = sorted(d for d in os.listdir(GOLDEN) if os.path.isdir(os.path.join(GOLDEN, d)) and not d.startswith("z"))


BIT_EXACT = {"lap2d_32", "convdiff2d_24"}


def same(a, b, case, rtol=1e-15):
    if case in BIT_EXACT:
        return np.array_equal(a, b)
    return np.max(np.abs(a - b)) <= rtol * max(1.0, np.max(np.abs(b)))


def load(case):
    d = os.path.join(GOLDEN, case)
    res = {}
    with open(os.path.join(d, "result.txt")) as f:
        for line in f:
            k, v = line.strip().split("=", 1)
            res[k] = v
    meta = {}
    with open(os.path.join(d, "params.txt")) as f:
        for line in f:
            k, v = line.strip().split("=", 1)
            meta[k] = v
    return (pgxd.read(os.path.join(d, "setup.bin")), pgxd.read(os.path.join(d, "problem.bin")),
            pgxd.read(os.path.join(d, "apply.bin")), pgxd.read(os.path.join(d, "solution.bin")), res, meta)


@pytest.fixture(scope="module", autouse=True)
def built():
    O.build()


@pytest.mark.parametrize("case", CASES)
def test_oracle_preconditioner_apply_bit_exact(case):
    setup, _, ap, _, _, _ = load(case)
    g = O.GemslrOracle(setup)
    n = g.n
    for k in range(int(ap["k"][0])):
        z = g.solve(ap["in"][k * n:(k + 1) * n])
        assert same(z, ap["out"][k * n:(k + 1) * n], case)


@pytest.mark.parametrize("case", CASES)
def test_oracle_fgmres_bit_exact(case):
    setup, prob, _, sol, res, meta = load(case)
    g = O.GemslrOracle(setup)
    p = P.workload_params(meta["workload"])
    x, r = g.fgmres_solve(prob["b"], int(p[P.SOLVER_KDIM]), int(p[P.SOLVER_MAXITS]), float(p[P.SOLVER_TOL]))
    assert r["iters"] == int(res["iters"])
    assert same(np.array(r["hist"]), sol["rel_res_hist"], case, rtol=1e-12)
    assert same(x, sol["x"], case, rtol=1e-13)


@pytest.mark.parametrize("case", CASES)
def test_level_schedules_match_reference(case):
    from pargemslr_b200 import _abi
    setup = load(case)[0]
    for l in range(int(setup["nlev"][0])):
        for c in range(int(setup[f"L{l}.ncomp"][0])):
            pc = f"L{l}.B{c}."
            for uplo, key in (("L", "l"), ("U", "u")):
                if pc + "lvl_ptr_" + key not in setup:
                    continue
                ref = (setup[pc + "lvl_ptr_" + key], setup[pc + "lvl_" + key])
                mine = O.build_levels(uplo, setup[pc + uplo + ".i"], setup[pc + uplo + ".j"])
                lib = _abi.build_levels(uplo, setup[pc + uplo + ".i"], setup[pc + uplo + ".j"])
                for got in (mine, lib):
                    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


@pytest.mark.parametrize("case", CASES)
def test_stencil_generator_matches_reference(case):
    _, prob, _, _, _, meta = load(case)
    nx, ny, nz, shift, ax, ay, az = [float(v) for v in meta["lap"].split()]
    A = problems.laplacian(int(nx), int(ny), int(nz), ax, ay, az, shift)
    assert np.array_equal(A[0], prob["A.i"]) and np.array_equal(A[1], prob["A.j"])
    assert np.array_equal(A[2], prob["A.a"])


def test_oracle_planted_error_is_detected():
    """A perturbed factor must break bit-exactness (the check is not vacuous)."""
    setup, _, ap, _, _, _ = load(CASES[0])
    setup = dict(setup)
    setup["L0.B0.D"] = setup["L0.B0.D"].copy()
    setup["L0.B0.D"][0] *= 1.0 + 1e-12
    g = O.GemslrOracle(setup)
    n = g.n
    assert not np.array_equal(g.solve(ap["in"][:n]), ap["out"][:n])


@pytest.mark.parametrize("case", CASES)
def test_preconditioner_nonzeros_match_reference(case):
    """pgx_gemslr_nnz on the reference's exported setup, against the reference's own count.

    ILU part: every B block's ILU holds n_c + nnz(L_c) + nnz(U_c) (ilu.cpp:2149), summed over blocks and levels in
    both GemslrClass::GetNumNonzeros (gemslr.cpp:4127) and ParallelGemslrClass::GetNumNonzeros
    (parallel_gemslr.cpp:7609).  Low-rank part: the parallel class, which the library follows, counts W_l and WH_l
    (m_l x r_l each); the sequential class the oracle runs counts W_l and H_l (r_l x r_l)."""
    import ctypes as C

    from pargemslr_b200 import _abi
    from pargemslr_b200.handle import import_structures
    from pargemslr_b200.structures import from_dump
    setup, _, _, _, _, meta = load(case)
    n, nlev = int(setup["n"][0]), int(setup["nlev"][0])
    lev_ptr = setup["lev_ptr"]
    ilu = sum(setup[f"L{l}.B{c}.D"].size + setup[f"L{l}.B{c}.L.j"].size + setup[f"L{l}.B{c}.U.j"].size
              for l in range(nlev) for c in range(int(setup[f"L{l}.ncomp"][0])))
    ranks = [int(setup[f"L{l}.lrc"][0]) if f"L{l}.lrc" in setup else 0 for l in range(nlev)]
    m = [n - int(lev_ptr[l + 1]) for l in range(nlev)]
    h = import_structures(from_dump(os.path.join(GOLDEN, case, "setup.bin")))
    try:
        nb, nl = C.c_int64(), C.c_int64()
        _abi.check(_abi.lib().pgx_gemslr_nnz(h, C.byref(nb), C.byref(nl)))
    finally:
        _abi.lib().pgx_gemslr_destroy(h)
    assert nb.value == ilu
    assert nl.value == sum(2 * m[l] * ranks[l] for l in range(nlev))
    from tests import oracle_runs
    if oracle_runs.available():
        lap = tuple(float(v) for v in meta["lap"].split())
        lap = (int(lap[0]), int(lap[1]), int(lap[2])) + lap[3:]
        ref = oracle_runs.run(lap=lap, params=P.workload_params(meta["workload"]), solve=False, dump=False)
        assert ref["nnz_bsolver"] == nb.value
        assert ref["nnz_lr"] == sum(m[l] * ranks[l] + ranks[l] ** 2 for l in range(nlev))


@pytest.mark.parametrize("case", CASES)
def test_residual_history_is_a_running_product_of_givens_sines(case):
    """The Givens residual history FlexGmresClass records (GetRelativeResidual, fgmres.hpp:430-450) is, bit for
    bit, a running product: P_0 = ||r_0||, P_j = |s_j| * P_(j-1) over all iterations (a restart keeps the estimate),
    history_j = P_j / ||b||.  Checked on the reference binary's own recorded history, so a solver that keeps only
    its sines can give the history back."""
    setup, prob, _, sol, res, meta = load(case)
    g = O.GemslrOracle(setup)
    p = P.workload_params(meta["workload"])
    _, r = g.fgmres_solve(prob["b"], int(p[P.SOLVER_KDIM]), int(p[P.SOLVER_MAXITS]), float(p[P.SOLVER_TOL]))
    prod = r["r0"]
    hist = [prod / r["normb"]]
    for s in r["givens_s"]:
        prod = abs(s) * prod
        hist.append(prod / r["normb"])
    np.testing.assert_array_equal(np.array(hist), np.array(r["hist"]))
    assert same(np.array(hist), sol["rel_res_hist"], case, rtol=1e-12)


@pytest.mark.parametrize("lap,workload", [((64, 64, 1, 0.0, 0.0, 0.0, 0.0), "lap2d_256"),
                                          ((32, 32, 32, 0.0, 0.0, 0.0, 0.0), "lap3d_128")])
def test_oracle_usolve_matches_reference(lap, workload):
    """The U solve option (params[141] = 1, gemslr.cpp:3527-3532) against the reference run with it: the
    preconditioner applications bit for bit up to 1e-13 and the FGMRES solve with the same iteration count."""
    from tests import oracle_runs
    if not oracle_runs.available():
        pytest.skip("reference solver not built here")
    p = P.workload_params(workload)
    p[P.ADVANCED_GLOBAL_SOLVE] = 1
    n = lap[0] * lap[1] * lap[2]
    ref = oracle_runs.run(lap=lap, params=p, xtrue=oracle_runs.x_true(n, seed=7), apply_k=2)
    g = O.GemslrOracle(pgxd.read(ref["setup"]))
    assert g.usolve
    ap = ref["apply"]
    for k in range(int(ap["k"][0])):
        z = g.solve(ap["in"][k * n:(k + 1) * n])
        z_ref = ap["out"][k * n:(k + 1) * n]
        assert np.linalg.norm(z - z_ref) <= 1e-13 * np.linalg.norm(z_ref)
    b = pgxd.read(ref["problem"])["b"]
    x, r = g.fgmres_solve(b, int(p[P.SOLVER_KDIM]), int(p[P.SOLVER_MAXITS]), float(p[P.SOLVER_TOL]))
    assert r["iters"] == int(ref["iters"])
    x_ref = ref["solution"]["x"]
    assert np.linalg.norm(x - x_ref) <= 1e-10 * np.linalg.norm(x_ref)
