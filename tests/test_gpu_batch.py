"""Concurrent solve slots, batch solves and the serving loop.

Every reduction on the solve path has a fixed order, so a right-hand side
gives the same bits whether it is solved alone, in a batch spread over
several slots, or among other requests in the serving queue.
"""
import numpy as np
import pytest

from pargemslr_b200 import params as P
from pargemslr_b200 import problems
from pargemslr_b200._abi import PgxError

pytestmark = pytest.mark.gpu


def _system(grid=(24, 24, 24), nrhs=6, seed=5):
    A = problems.laplacian(*grid)
    n = A[0].size - 1
    rng = np.random.default_rng(seed)
    return A, n, rng.standard_normal((nrhs, n))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_solves(precision):
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap3d_128")
    A, n, B = _system()
    h = GemslrHandle.from_matrix(A, p, precision=precision)
    singles = [h.solve(b, params=p) for b in B]
    h.set_slots(4)
    assert h.slot_bytes(int(p[P.SOLVER_KDIM])) > 0
    X, res = h.solve_batch(B, params=p)
    for r, (x1, r1) in enumerate(singles):
        assert res[r]["status"] == 0
        assert res[r]["iters"] == r1["iters"]
        assert res[r]["true_rel_res"] <= 1e-8
        np.testing.assert_array_equal(X[r], x1)
    # shrinking and growing the slot count keeps the shared factors intact
    h.set_slots(2)
    X2, _ = h.solve_batch(B[:3], params=p)
    np.testing.assert_array_equal(X2, X[:3])
    h.set_slots(1)
    x0, _ = h.solve(B[0], params=p)
    np.testing.assert_array_equal(x0, X[0])
    h.close()


@pytest.mark.parametrize("precision,lanes", [("mixed", 2), ("mixed", 4), ("fp64", 4)])
def test_multilane_slots_equal_single_solves(precision, lanes):
    """Lanes share the triangular passes; every other step is per lane, so bits match."""
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap3d_128")
    A, n, B = _system(nrhs=7, seed=13)
    h = GemslrHandle.from_matrix(A, p, precision=precision)
    singles = [h.solve(b, params=p) for b in B]
    kd = int(p[P.SOLVER_KDIM])
    base = h.device_bytes(kd)
    h.set_lanes(lanes)
    h.set_slots(3)
    # two more slots of `lanes` right-hand sides each, plus their factor layout
    assert h.device_bytes(kd) >= base + 2 * h.slot_bytes(kd)
    X, res = h.solve_batch(B, params=p)
    for r, (x1, r1) in enumerate(singles):
        assert res[r]["status"] == 0
        assert res[r]["iters"] == r1["iters"], (r, res[r]["iters"], r1["iters"])
        np.testing.assert_array_equal(X[r], x1)
    srv = h.server(p)
    xs = {}
    for rid in (5, 1, 6, 0, 3, 2, 4):
        xs[rid] = np.zeros(n)
        srv.submit(xs[rid], B[rid], rid)
    done = srv.run()
    assert sorted(i for i, _ in done) == list(range(7))
    for rid, rr in done:
        assert rr["status"] == 0
        np.testing.assert_array_equal(xs[rid], singles[rid][0])
    srv.close()
    h.set_lanes(1)
    h.close()


def test_many_concurrent_multilane_slots_equal_single_solves():
    """Fifteen 4-lane slots at once over subdomains of many staged chunks: the
    per-subdomain passes of different slots share the SMs with every other
    kernel in flight, and each result still equals its single solve bit for bit
    (a chunk's staging buffer is reused only after every read of it)."""
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap3d_128")
    A, n, B = _system(grid=(48, 48, 48), nrhs=61, seed=31)
    h = GemslrHandle.from_matrix(A, p, precision="mixed")
    singles = [h.solve(b, params=p) for b in B]
    h.set_lanes(4)
    h.set_slots(16)
    for _ in range(2):
        X, res = h.solve_batch(B, params=p)
        for r, (x1, r1) in enumerate(singles):
            assert res[r]["status"] == 0, (r, res[r])
            assert res[r]["iters"] == r1["iters"], (r, res[r]["iters"], r1["iters"])
            np.testing.assert_array_equal(X[r], x1)
    h.set_lanes(1)
    h.close()


def test_server_matches_single_solves_in_any_order():
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap3d_128")
    A, n, B = _system(nrhs=7, seed=9)
    h = GemslrHandle.from_matrix(A, p, precision="mixed")
    singles = [h.solve(b, params=p)[0] for b in B]
    h.set_slots(3)
    srv = h.server(p)
    xs = {}
    for rid in (4, 0, 6, 2, 1, 5, 3):
        xs[rid] = np.zeros(n)
        srv.submit(xs[rid], B[rid], rid)
    done = srv.run()
    assert sorted(i for i, _ in done) == list(range(7))
    for rid, res in done:
        assert res["status"] == 0 and res["true_rel_res"] <= 1e-8
        np.testing.assert_array_equal(xs[rid], singles[rid])
    # a live server owns the slots
    with pytest.raises(PgxError):
        h.set_slots(5)
    with pytest.raises(PgxError):
        h.solve(B[0], params=p)
    srv.close()
    h.set_slots(5)
    h.close()


@pytest.mark.parametrize("lanes", [1, 2])
def test_batch_reports_a_bad_column(lanes):
    from pargemslr_b200 import _abi
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap3d_128")
    A, n, B = _system(grid=(12, 12, 12), nrhs=5)
    h = GemslrHandle.from_matrix(A, p, precision="fp64")
    h.set_lanes(lanes)
    h.set_slots(2)
    B[1, 7] = np.nan
    with pytest.raises(PgxError):
        h.solve_batch(B, params=p)
    # the other columns are still solved, lanes shared with the bad one included
    X = np.zeros_like(B)
    res = (_abi.Result * 5)()
    import ctypes as C
    rc = _abi.lib().pgx_gemslr_solve_batch(h._h, 5, _abi.ptr(X), n, _abi.ptr(B), n, _abi.LOCATION_HOST,
                                           _abi.ptr(p), C.cast(res, C.c_void_p))
    assert rc == _abi.ERROR_NOT_FINITE
    assert res[1].status == _abi.ERROR_NOT_FINITE
    for r in (0, 2, 3, 4):
        assert res[r].status == 0 and res[r].true_rel_res <= 1e-8
    B[1, 7] = 0.0
    X, out = h.solve_batch(B, params=p)
    assert all(r["status"] == 0 for r in out)
    h.close()


def test_server_on_its_own_thread():
    """Requests submitted while the library's serving thread runs; each result equals a single solve."""
    import time
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap3d_128")
    A, n, B = _system(nrhs=6, seed=17)
    h = GemslrHandle.from_matrix(A, p, precision="mixed")
    singles = [h.solve(b, params=p)[0] for b in B]
    h.set_lanes(2)
    h.set_slots(2)
    srv = h.server(p)
    srv.start()
    with pytest.raises(PgxError):
        srv.step()  # the thread owns the stepping
    xs = [np.zeros(n) for _ in range(len(B))]
    got = {}
    for rid in range(len(B)):
        srv.submit(xs[rid], B[rid], rid)
        time.sleep(0.01)
        got.update(dict(srv.collect()))
    t0 = time.time()
    while len(got) < len(B) and time.time() - t0 < 120:
        time.sleep(0.005)
        got.update(dict(srv.collect()))
    srv.stop()
    assert sorted(got) == list(range(len(B)))
    for rid, res in got.items():
        assert res["status"] == 0 and res["true_rel_res"] <= 1e-8
        np.testing.assert_array_equal(xs[rid], singles[rid])
    srv.close()
    h.close()


def test_nonfinite_device_column_retires_only_its_request():
    """A NaN in one device right-hand side ends that solve with PGX_ERROR_NOT_FINITE; its lane mates finish normally."""
    import ctypes as C
    import torch
    from pargemslr_b200 import _abi
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap3d_128")
    p[P.SOLVER_MAXITS] = 20
    A, n, B = _system(grid=(12, 12, 12), nrhs=4, seed=23)
    h = GemslrHandle.from_matrix(A, p, precision="mixed")
    singles = [h.solve(b, params=p)[0] for b in B]
    h.set_lanes(4)
    h.set_slots(2)
    Bd = torch.tensor(B, device="cuda")
    Bd[2, 5] = float("nan")
    Xd = torch.zeros_like(Bd)
    torch.cuda.synchronize()
    res = (_abi.Result * 4)()
    rc = _abi.lib().pgx_gemslr_solve_batch(h._h, 4, Xd.data_ptr(), n, Bd.data_ptr(), n, _abi.LOCATION_DEVICE,
                                           _abi.ptr(p), C.cast(res, C.c_void_p))
    assert rc == _abi.ERROR_NOT_FINITE
    assert res[2].status == _abi.ERROR_NOT_FINITE
    X = Xd.cpu().numpy()
    for r in (0, 1, 3):
        assert res[r].status == 0 and res[r].true_rel_res <= 1e-8
        np.testing.assert_array_equal(X[r], singles[r])
    h.close()
