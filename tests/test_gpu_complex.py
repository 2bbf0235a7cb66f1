"""GPU parity of the complex GeMSLR-FGMRES solve against the reference's own
complex solver (GemslrClass and FlexGmresClass over complexd).

The reference (tests/golden/zlap3d_12, and oracle/_ref/pgx_ref_driver_z run
here on larger grids) sets up the complex shifted Laplacian, solves each
complex-Gaussian right-hand side one at a time, and applies its
preconditioner to seeded vectors.  Its post-setup structures are imported
through the C ABI as interleaved {re, im} doubles.  Bars:
  complex128 path: preconditioner applications within 1e-9 relative of the
      reference's, iterations within +-1, FP64 true relative residual <= 1e-8,
      ||x - x_ref|| / ||x_ref|| <= 1e-6;
  complex64 preconditioner (mixed): iterations at most 15% above the
      reference (plus one), true relative residual <= 1e-8;
and a multi-lane slot gives every right-hand side the bits of its single solve.
"""
import os

import numpy as np
import pytest

from pargemslr_b200 import params as P
from pargemslr_b200 import pgxd
from pargemslr_b200.structures import from_dump
from tests import oracle_runs

pytestmark = pytest.mark.gpu

CASE = os.path.join(os.path.dirname(__file__), "golden", "zlap3d_12")


def _fixture():
    st = from_dump(os.path.join(CASE, "setup.bin"))
    prob = pgxd.read(os.path.join(CASE, "problem.bin"))
    B = prob["B"].view(np.complex128).reshape(int(prob["nrhs"][0]), -1)
    sol = pgxd.read(os.path.join(CASE, "solution.bin"))
    X = [sol["x%d" % r].view(np.complex128) for r in range(B.shape[0])]
    res = dict(line.strip().split("=", 1) for line in open(os.path.join(CASE, "result.txt")))
    iters = [int(t) for t in res["iters"].split(",")]
    ap = pgxd.read(os.path.join(CASE, "apply.bin"))
    return st, B, X, iters, ap["in"].view(np.complex128).reshape(2, -1), ap["out"].view(np.complex128).reshape(2, -1)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_complex_precond_apply_matches_reference():
    from pargemslr_b200.handle import GemslrHandle
    st, _, _, _, vin, vout = _fixture()
    h = GemslrHandle(st, precision="fp64")
    try:
        assert h.complex
        for k in range(2):
            z = h.apply(vin[k])
            assert z.dtype == np.complex128
            assert _rel(z, vout[k]) <= 1e-9, _rel(z, vout[k])
    finally:
        h.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_complex_fixture_solves_match_reference(precision):
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("zsmall")
    st, B, X, iters, _, _ = _fixture()
    h = GemslrHandle(st, precision=precision)
    try:
        for r in range(B.shape[0]):
            x, res = h.solve(B[r], params=p)
            assert res["status"] == 0 and res["true_rel_res"] <= 1e-8, res
            if precision == "fp64":
                assert abs(res["iters"] - iters[r]) <= 1, (res["iters"], iters[r])
                assert _rel(x, X[r]) <= 1e-6, _rel(x, X[r])
            else:
                assert res["iters"] <= int(np.floor(1.15 * iters[r])) + 1, (res["iters"], iters[r])
    finally:
        h.close()


@pytest.fixture(scope="module")
def zref32():
    """The reference on a 32^3 Laplacian shifted by 0.2 + 0.02i (indefinite), config-3 settings (5 levels,
    rank 32, FGMRES(100)), three complex-Gaussian right-hand sides."""
    if not oracle_runs.available_complex():
        pytest.fail("oracle/_ref/pgx_ref_driver_z is missing (build it with make -C oracle)")
    p = P.workload_params("zlap3d_96")
    n = 32 ** 3
    B = oracle_runs.complex_rhs(n, 3, 17)
    ref = oracle_runs.run_complex((32, 32, 32, 0.2, 0.02, 0.0, 0.0, 0.0), p, B, threads=os.cpu_count() or 1)
    return ref, p, B


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_complex_indefinite_solves_match_reference(zref32, precision):
    from pargemslr_b200.handle import GemslrHandle
    ref, p, B = zref32
    h = GemslrHandle(from_dump(ref["setup"]), precision=precision)
    try:
        for r in range(B.shape[0]):
            x, res = h.solve(B[r], params=p)
            it_ref = ref["iters"][r]
            assert res["status"] == 0 and res["true_rel_res"] <= 1e-8, res
            if precision == "fp64":
                assert abs(res["iters"] - it_ref) <= 1, (res["iters"], it_ref)
                assert _rel(x, ref["x"][r]) <= 1e-6, _rel(x, ref["x"][r])
            else:
                assert res["iters"] <= int(np.floor(1.15 * it_ref)) + 1, (res["iters"], it_ref)
    finally:
        h.close()


@pytest.mark.parametrize("lanes", [2, 4])
def test_complex_multilane_slot_equals_single_solves(zref32, lanes):
    from pargemslr_b200.handle import GemslrHandle
    ref, p, B = zref32
    st = from_dump(ref["setup"])
    h = GemslrHandle(st, precision="mixed")
    try:
        rng = np.random.default_rng(5)
        Bs = rng.standard_normal((lanes + 1, st.n)) + 1j * rng.standard_normal((lanes + 1, st.n))
        singles = [h.solve(b, params=p) for b in Bs]
        h.set_lanes(lanes)
        h.set_slots(2)
        X, res = h.solve_batch(Bs, params=p)
        for r, (x1, r1) in enumerate(singles):
            assert res[r]["status"] == 0 and res[r]["iters"] == r1["iters"], (r, res[r], r1)
            np.testing.assert_array_equal(X[r], x1)
        h.set_lanes(1)
    finally:
        h.close()


@pytest.mark.parametrize("nrhs,m,r", [(8, 1000, 32), (16, 4133, 32), (16, 200, 7)])
def test_tensor_core_block_lowrank_matches_numpy(nrhs, m, r):
    """x_q + WH (W^H x_q) for a block of complex64 vectors on tcgen05 (3xTF32), against FP64 numpy."""
    import torch
    from pargemslr_b200 import _abi
    from pargemslr_b200.handle import init
    init(0)
    rng = np.random.default_rng(m + r)
    W = (rng.standard_normal((r, m)) + 1j * rng.standard_normal((r, m))).astype(np.complex64)  # column c = W[c]
    WH = (rng.standard_normal((r, m)) + 1j * rng.standard_normal((r, m))).astype(np.complex64) / m
    X = (rng.standard_normal((nrhs, m)) + 1j * rng.standard_normal((nrhs, m))).astype(np.complex64)
    ref = X.astype(np.complex128) + (WH.T.astype(np.complex128) @ (np.conj(W.astype(np.complex128)) @ X.T.astype(np.complex128))).T
    dW = torch.from_numpy(W.view(np.float32).copy()).cuda()
    dWH = torch.from_numpy(WH.view(np.float32).copy()).cuda()
    dX = torch.from_numpy(X.view(np.float32).copy()).cuda()
    for _ in range(2):  # twice: the second call finds the first call's scratch released
        dX.copy_(torch.from_numpy(X.view(np.float32).copy()))
        _abi.check(_abi.lib().pgx_lowrank_block_apply_c64(m, r, nrhs, dW.data_ptr(), dWH.data_ptr(), dX.data_ptr(),
                                                          m))
        got = dX.cpu().numpy().view(np.complex64).astype(np.complex128)
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref - X)
        assert err <= 1e-5, err


def test_complex_block_of_16_solves_matches_single_solves(zref32):
    """Sixteen right-hand sides in one 16-lane slot: the triangular passes merged four lanes at a time and the
    low-rank corrections on the tensor cores.  Every solve converges to 1e-8 with the iterations of its single
    solve (+-1) and a solution within 1e-6 of it."""
    from pargemslr_b200.handle import GemslrHandle
    ref, p, _ = zref32
    st = from_dump(ref["setup"])
    h = GemslrHandle(st, precision="mixed")
    try:
        rng = np.random.default_rng(23)
        Bs = rng.standard_normal((16, st.n)) + 1j * rng.standard_normal((16, st.n))
        singles = [h.solve(b, params=p) for b in Bs]
        h.set_lanes(16)
        h.set_slots(2)
        assert "16 lanes" in h.describe(1)
        X, res = h.solve_batch(Bs, params=p)
        for r, (x1, r1) in enumerate(singles):
            assert res[r]["status"] == 0 and res[r]["true_rel_res"] <= 1e-8, (r, res[r])
            assert abs(res[r]["iters"] - r1["iters"]) <= 1, (r, res[r]["iters"], r1["iters"])
            assert _rel(X[r], x1) <= 1e-6, (r, _rel(X[r], x1))
        h.set_lanes(1)
    finally:
        h.close()
