"""Scaled-down parity cases of the batched-uneven and serving workloads.

Batched uneven systems: upwind convection-diffusion on grids of different
sizes with different convection, 2 levels, rank 8, FGMRES(30), each held
resident by its own handle and served concurrently (one server per matrix,
stepped round-robin).  Serving: a nonsymmetric random sparse matrix (7-27
nonzeros per row, diagonal 1.2 times the off-diagonal sum) with requests
arriving while others are on the GPU, over multi-lane slots.

Every result must equal, bit for bit, the same right-hand side solved alone;
convergence is checked in FP64, and the solution is compared with the
reference CPU solver's on the same matrix and right-hand side (different
setups, both to relative residual 1e-8, so the solutions agree to about the
condition number times 1e-8; bar 1e-6).
"""
import os
import tempfile

import numpy as np
import pytest

from pargemslr_b200 import params as P
from pargemslr_b200 import pgxd, problems
from tests import oracle_runs

pytestmark = pytest.mark.gpu

CONVDIFF = [(48, 48, 12.0, 30.0), (80, 64, 45.0, 5.0), (120, 96, 3.0, 40.0), (160, 160, 25.0, 25.0)]


def _convdiff_params():
    p = P.workload_params("lap2d_256")
    p[P.PREPOSS_NLEV_GLOBAL] = 2
    p[P.LR_RANK1_GLOBAL] = p[P.LR_RANK1_LOCAL] = 8
    p[P.LR_RANK2_GLOBAL] = p[P.LR_RANK2_LOCAL] = 8
    p[P.SOLVER_KDIM] = 30
    return p


def _reference_solution(A, b, p):
    """The reference CPU solver on a matrix given as CSR (its own setup)."""
    d = tempfile.mkdtemp(prefix="pgx_csr_")
    f = os.path.join(d, "A.bin")
    pgxd.write(f, {"A.i": A[0].astype(np.int32), "A.j": A[1].astype(np.int32), "A.a": A[2].astype(np.float64)})
    rf = os.path.join(d, "rhs.bin")
    pgxd.write(rf, {"b": np.ascontiguousarray(b, np.float64)})
    return oracle_runs.run(csr_file=f, params=p, rhs_file=rf, dump=False)


def test_uneven_convdiff_systems_served_together():
    from pargemslr_b200.handle import GemslrHandle
    p = _convdiff_params()
    rng = np.random.default_rng(21)
    systems = []
    for nx, ny, bx, by in CONVDIFF:
        A = problems.upwind_convdiff_2d(nx, ny, bx, by)
        n = nx * ny
        B = 2.0 * rng.random((2, n)) - 1.0
        h = GemslrHandle.from_matrix(A, p, precision="mixed")
        singles = [h.solve(b, params=p) for b in B]
        systems.append((A, B, h, singles))
    servers, outs = [], []
    for k, (A, B, h, _) in enumerate(systems):
        srv = h.server(p)
        xs = [np.zeros(B.shape[1]) for _ in range(len(B))]
        for r, b in enumerate(B):
            srv.submit(xs[r], b, r)
        servers.append(srv)
        outs.append(xs)
    done = [dict() for _ in systems]
    while any(len(d) < 2 for d in done):
        for k, srv in enumerate(servers):
            srv.step()
            for rid, res in srv.collect():
                done[k][rid] = res
    for k, (A, B, h, singles) in enumerate(systems):
        for r in range(len(B)):
            res = done[k][r]
            assert res["status"] == 0 and res["true_rel_res"] <= 1e-8, (k, r, res)
            assert res["iters"] == singles[r][1]["iters"]
            np.testing.assert_array_equal(outs[k][r], singles[r][0])
        servers[k].close()
    if oracle_runs.available():
        A, B, h, singles = systems[0]
        ref = _reference_solution(A, B[0], p)
        x_ref = ref["solution"]["x"]
        assert np.linalg.norm(singles[0][0] - x_ref) / np.linalg.norm(x_ref) <= 1e-6
    for _, _, h, _ in systems:
        h.close()


def test_random_sparse_requests_arriving_while_others_run():
    from pargemslr_b200.handle import GemslrHandle
    n = 20000
    A = problems.random_diag_dominant(n, seed=5)
    p = P.workload_params("lap3d_128")
    p[P.PREPOSS_NLEV_GLOBAL] = 3
    p[P.SOLVER_KDIM] = 40
    rng = np.random.default_rng(8)
    B = 2.0 * rng.random((7, n)) - 1.0
    h = GemslrHandle.from_matrix(A, p, precision="mixed")
    singles = [h.solve(b, params=p) for b in B]
    for x1, r1 in singles:
        assert r1["status"] == 0 and r1["true_rel_res"] <= 1e-8
    h.set_lanes(2)
    h.set_slots(3)
    srv = h.server(p)
    xs = [np.zeros(n) for _ in range(len(B))]
    got = {}
    arrivals = [[0, 1], [2], [3, 4, 5], [6]]
    for wave in arrivals:
        for rid in wave:
            srv.submit(xs[rid], B[rid], rid)
        for _ in range(3):
            srv.step()
            got.update(dict(srv.collect()))
    got.update(dict(srv.run()))
    assert sorted(got) == list(range(len(B)))
    for rid, res in got.items():
        assert res["status"] == 0 and res["true_rel_res"] <= 1e-8
        np.testing.assert_array_equal(xs[rid], singles[rid][0])
    srv.close()
    if oracle_runs.available():
        ref = _reference_solution(A, B[0], p)
        x_ref = ref["solution"]["x"]
        assert np.linalg.norm(singles[0][0] - x_ref) / np.linalg.norm(x_ref) <= 1e-6
    h.close()


def test_matrix_market_file_to_solution(tmp_path):
    """A matrix read from a Matrix Market file (pgx_csr_read_mm) set up and solved on the GPU."""
    import scipy.io
    import scipy.sparse as sp
    from pargemslr_b200 import _abi
    from pargemslr_b200.handle import GemslrHandle
    rp, cj, va = problems.upwind_convdiff_2d(70, 50, 20.0, 8.0)
    n = rp.size - 1
    path = str(tmp_path / "convdiff.mtx")
    scipy.io.mmwrite(path, sp.csr_matrix((va, cj, rp), shape=(n, n)))
    rp2, cj2, va2, shape = _abi.read_mm(path)
    assert shape == (n, n)
    p = _convdiff_params()
    xt = problems.x_true(n, 3)
    b = problems.spmv((rp2, cj2, va2), xt)
    h = GemslrHandle.from_matrix((rp2, cj2, va2), p, precision="fp64")
    x, r = h.solve(b, params=p)
    assert r["status"] == 0 and r["true_rel_res"] <= 1e-8
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) <= 1e-6
    h.close()
