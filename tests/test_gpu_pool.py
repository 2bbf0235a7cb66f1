"""Serving pool: requests for several resident matrices under one device-memory budget.

Each request's result equals, bit for bit, the ordinary solve of the same right-hand side on the same handle before it
joined the pool (the pool only decides where and when a solve runs).  The budget holds the members' factors and two
more slots: the pool never counts more than the budget, it releases idle slots of one member to admit another's
requests, and every request finishes.  A member whose factors do not fit is refused.
"""
import numpy as np
import pytest

from pargemslr_b200 import _abi
from pargemslr_b200 import params as P
from pargemslr_b200 import problems

pytestmark = pytest.mark.gpu


def _members():
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap2d_256")
    p[P.SOLVER_KDIM] = 30
    mats = [problems.random_diag_dominant(n, seed) for n, seed in ((6000, 1), (9000, 2), (12000, 3))]
    return p, mats, [GemslrHandle.from_matrix(A, p, precision="mixed") for A in mats]


def test_pool_results_equal_solo_solves_under_a_tight_budget():
    from pargemslr_b200.serving import Pool
    p, mats, hs = _members()
    rng = np.random.default_rng(9)
    reqs = []
    for rid in range(24):
        m = int(rng.integers(0, len(hs)))
        b = rng.uniform(-1, 1, hs[m].n)
        x_ref, r_ref = hs[m].solve(b, params=p)
        reqs.append((rid, m, b, x_ref, r_ref))
    base = sum(h.device_bytes(int(p[P.SOLVER_KDIM])) for h in hs)
    extra = max(h.slot_bytes(int(p[P.SOLVER_KDIM])) for h in hs)
    pool = Pool(base + 2 * extra, p)
    try:
        idx = [pool.add(h) for h in hs]
        assert idx == [0, 1, 2]
        xs = {}
        for rid, m, b, _, _ in reqs:
            xs[rid] = np.zeros(hs[m].n)
            pool.submit(m, xs[rid], b, rid)
        done = dict(pool.run())
        st = pool.stats()
        assert sorted(done) == list(range(24))
        assert st["peak_bytes"] <= base + 2 * extra
        assert st["slots"] <= len(hs) + 2
        for rid, m, b, x_ref, r_ref in reqs:
            assert done[rid]["status"] == 0
            assert done[rid]["iters"] == r_ref["iters"]
            assert np.array_equal(xs[rid], x_ref), rid
    finally:
        pool.close()
        for h in hs:
            h.close()


def test_pool_refuses_a_member_that_does_not_fit():
    from pargemslr_b200.serving import Pool
    p, mats, hs = _members()
    pool = Pool(hs[0].device_bytes(int(p[P.SOLVER_KDIM])) + 1, p)
    try:
        pool.add(hs[0])
        with pytest.raises(_abi.PgxError) as e:
            pool.add(hs[2])
        assert e.value.code == _abi.ERROR_OOM
    finally:
        pool.close()
        for h in hs:
            h.close()


def test_pool_serves_on_its_own_thread():
    import time
    from pargemslr_b200.serving import Pool
    p, mats, hs = _members()
    pool = Pool(1 << 40, p)
    try:
        for h in hs:
            pool.add(h)
        pool.start()
        rng = np.random.default_rng(4)
        xs = {}
        for rid in range(12):
            m = rid % 3
            xs[rid] = np.zeros(hs[m].n)
            pool.submit(m, xs[rid], rng.uniform(-1, 1, hs[m].n), rid)
            time.sleep(0.002)
        got = {}
        t0 = time.time()
        while len(got) < 12 and time.time() - t0 < 120:
            got.update(dict(pool.collect()))
            time.sleep(0.005)
        pool.stop()
        assert len(got) == 12 and all(r["status"] == 0 and r["true_rel_res"] <= 1e-8 for r in got.values())
    finally:
        pool.close()
        for h in hs:
            h.close()
