"""Many systems in one persistent launch (pgx_systems_*), checked system by system.

Each system's solution must match the same handle's own pgx_gemslr_solve (same preconditioner, same arithmetic,
sums in another order): both converge to FP64 relative residual 1e-8, iteration counts within +-1, and the
solutions agree to 1e-6 relative.  One system is also compared with the reference CPU solver on the same matrix
(its own setup), as the per-handle batched-uneven test does.  Shapes: upwind convection-diffusion systems of
uneven sizes, 2 levels, rank 8, FGMRES(30), the level-0 inner Schur FGMRES on (the reference default).
"""
import numpy as np
import pytest

from pargemslr_b200 import _abi, problems
from pargemslr_b200 import params as P
from tests import oracle_runs
from tests.test_gpu_configs import _convdiff_params, _reference_solution

pytestmark = pytest.mark.gpu

GRIDS = [(24, 24, 5.0, 40.0), (40, 32, 30.0, 2.0), (64, 48, 12.0, 12.0), (20, 90, 45.0, 20.0),
         (96, 80, 3.0, 33.0), (33, 33, 0.0, 0.0), (128, 64, 25.0, 8.0), (50, 50, 48.0, 48.0)]


def _systems(grids, p, precision):
    from pargemslr_b200.handle import GemslrHandle
    rng = np.random.default_rng(41)
    out = []
    for nx, ny, bx, by in grids:
        A = problems.upwind_convdiff_2d(nx, ny, bx, by)
        b = 2.0 * rng.random(nx * ny) - 1.0
        out.append((A, b, GemslrHandle.from_matrix(A, p, precision=precision)))
    return out


def _check_against_singles(systems, X, R, p, it_slack=1):
    for k, (A, b, h) in enumerate(systems):
        xs, rs = h.solve(b, params=p)
        r = R[k]
        assert r["status"] == 0 and r["true_rel_res"] <= 1e-8, (k, r)
        assert abs(r["iters"] - rs["iters"]) <= it_slack, (k, r["iters"], rs["iters"])
        assert np.linalg.norm(X[k] - xs) <= 1e-6 * np.linalg.norm(xs), k
        res = problems.spmv(A, X[k]) - b
        assert np.linalg.norm(res) <= 1.01e-8 * np.linalg.norm(b), k


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_uneven_systems_in_one_launch_match_single_solves(precision):
    from pargemslr_b200.systems import SystemsBatch
    p = _convdiff_params()
    systems = _systems(GRIDS, p, precision)
    sb = SystemsBatch([h for _, _, h in systems])
    X, R = sb.solve([b for _, b, _ in systems], params=p)
    _check_against_singles(systems, X, R, p)
    s, e, _ = sb.timing()
    assert np.all(e >= s) and s.min() == 0.0
    assert all(r["launches"] == 1 for r in R)
    # a second solve reuses the packed structures and gives the same results (fixed reduction order)
    X2, R2 = sb.solve([b for _, b, _ in systems], params=p)
    for k in range(len(systems)):
        np.testing.assert_array_equal(X[k], X2[k])
        assert R[k]["iters"] == R2[k]["iters"]
    if precision == "mixed" and oracle_runs.available():
        A, b, _ = systems[2]
        x_ref = _reference_solution(A, b, p)["solution"]["x"]
        assert np.linalg.norm(X[2] - x_ref) <= 1e-6 * np.linalg.norm(x_ref)
    sb.close()
    for _, _, h in systems:
        h.close()


def test_schedules_and_autotuner_agree():
    from pargemslr_b200.systems import SystemsBatch
    p = _convdiff_params()
    systems = _systems(GRIDS[:5], p, "mixed")
    sb = SystemsBatch([h for _, _, h in systems])
    B = [b for _, b, _ in systems]
    base, _ = sb.solve(B, params=p)
    for sched in [(256, 4, 2, 2), (1024, 1, 8, 3), (512, 2, 1, 2), (256, 2, 4, 3)]:
        sb.set_schedule(*sched)
        assert sb.schedule == sched
        X, R = sb.solve(B, params=p)
        _check_against_singles(systems, X, R, p)
        for k in range(len(systems)):
            assert np.linalg.norm(X[k] - base[k]) <= 1e-6 * np.linalg.norm(base[k])
    best = sb.tune(B, params=p)
    table = sb.tune_table()
    assert len(table) == 7 and best > 0
    assert min(t[4] for t in table) == pytest.approx(best)
    chosen = sb.schedule
    assert any(t[:4] == chosen and t[4] == pytest.approx(best) for t in table)
    X, R = sb.solve(B, params=p)
    _check_against_singles(systems, X, R, p)
    sb.close()
    for _, _, h in systems:
        h.close()


def test_three_levels_without_inner_iteration_and_zero_rhs():
    """Level recursion below level 1 (3 levels) with low-rank corrections at two levels, no inner FGMRES; a
    zero right-hand side returns x = 0 after no iteration."""
    from pargemslr_b200.systems import SystemsBatch
    p = P.workload_params("small")
    p[P.SCHUR_ENABLE] = 0
    p[P.SOLVER_KDIM] = 30
    systems = _systems([(48, 48, 10.0, 3.0), (70, 40, 0.0, 25.0), (36, 36, 40.0, 40.0)], p, "mixed")
    sb = SystemsBatch([h for _, _, h in systems])
    B = [b for _, b, _ in systems]
    X, R = sb.solve(B, params=p)
    _check_against_singles(systems, X, R, p)
    B[1] = np.zeros_like(B[1])
    X, R = sb.solve(B, X0=[np.ones(len(b)) for b in B], params=p)
    assert R[1]["status"] == 0 and R[1]["iters"] == 0 and not np.any(X[1])
    assert R[0]["true_rel_res"] <= 1e-8 and R[2]["true_rel_res"] <= 1e-8
    sb.close()
    for _, _, h in systems:
        h.close()


def test_device_pointers_match_host_arrays():
    import torch
    from pargemslr_b200.systems import SystemsBatch
    p = _convdiff_params()
    systems = _systems(GRIDS[:4], p, "mixed")
    sb = SystemsBatch([h for _, _, h in systems])
    B = [b for _, b, _ in systems]
    X, _ = sb.solve(B, params=p)
    bd = [torch.from_numpy(b).cuda() for b in B]
    xd = [torch.zeros(len(b), dtype=torch.float64, device="cuda") for b in B]
    R = sb.solve_ptrs([x.data_ptr() for x in xd], [b.data_ptr() for b in bd], _abi.LOCATION_DEVICE, params=p)
    for k in range(len(B)):
        assert R[k]["status"] == 0
        np.testing.assert_array_equal(xd[k].cpu().numpy(), X[k])
    sb.close()
    for _, _, h in systems:
        h.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_reference_setups_in_one_launch_match_the_reference(precision):
    """Parity on the reference's own setup: uneven convection-diffusion systems set up by the reference CPU solver
    (GemslrClass::Setup, exported after setup) are solved together in one launch, each against the reference's own
    FGMRES solve of the same b: iterations within +-1 (FP64 preconditioner) or at most +15% (mixed), x within 1e-6
    relative of the reference's solution."""
    import os
    import tempfile

    from pargemslr_b200 import pgxd
    from pargemslr_b200.handle import GemslrHandle
    from pargemslr_b200.structures import from_dump
    from pargemslr_b200.systems import SystemsBatch
    if not oracle_runs.available():
        pytest.skip("reference solver not built")
    p = _convdiff_params()
    rng = np.random.default_rng(5)
    handles, refs, B = [], [], []
    for nx, ny, bx, by in GRIDS[:5]:
        A = problems.upwind_convdiff_2d(nx, ny, bx, by)
        b = 2.0 * rng.random(nx * ny) - 1.0
        d = tempfile.mkdtemp(prefix="pgx_sys_")
        f = os.path.join(d, "A.bin")
        pgxd.write(f, {"A.i": A[0].astype(np.int32), "A.j": A[1].astype(np.int32), "A.a": A[2].astype(np.float64)})
        rf = os.path.join(d, "rhs.bin")
        pgxd.write(rf, {"b": b})
        ref = oracle_runs.run(csr_file=f, params=p, rhs_file=rf, dump=True, solve=True)
        handles.append(GemslrHandle(from_dump(ref["setup"]), precision=precision))
        refs.append(ref)
        B.append(b)
    sb = SystemsBatch(handles)
    X, R = sb.solve(B, params=p)
    for k, ref in enumerate(refs):
        r = R[k]
        assert r["status"] == 0 and r["true_rel_res"] <= 1e-8, (k, r)
        if precision == "fp64":
            assert abs(r["iters"] - ref["iters"]) <= 1, (k, r["iters"], ref["iters"])
        else:
            assert r["iters"] <= int(np.floor(1.15 * ref["iters"])) + 1, (k, r["iters"], ref["iters"])
        x_ref = ref["solution"]["x"]
        assert np.linalg.norm(X[k] - x_ref) <= 1e-6 * np.linalg.norm(x_ref), k
    sb.close()
    for h in handles:
        h.close()
