"""The U solve option (PARGEMSLR_IO_ADVANCED_GLOBAL_SOLVE = 1) against the reference.

GemslrClass::SolveLevel (gemslr.cpp:3527-3532) skips a level's block-L part in the solve phase when the option is 1:
z = rhs instead of z_u = B^-1 rhs_u, z_l = rhs_l - E z_u.  The setup is the reference's own, run with the option set
and exported after setup (the option travels in the dump).  The FP64 preconditioner application must match the
reference's to 1e-9 and the solve its iterations within +-1 and its x within 1e-6; the mixed precision solve stays
within +15% iterations.  The multi-lane slots and the one-launch systems solve must follow the option too.
"""
import numpy as np
import pytest

from pargemslr_b200 import params as P
from pargemslr_b200 import pgxd
from pargemslr_b200.structures import from_dump
from tests import oracle_runs

pytestmark = pytest.mark.gpu

CASES = {
    "lap2d_64": ((64, 64, 1, 0.0, 0.0, 0.0, 0.0), "lap2d_256"),
    "lap3d_32": ((32, 32, 32, 0.0, 0.0, 0.0, 0.0), "lap3d_128"),
}


def _run(name):
    if not oracle_runs.available():
        pytest.fail("oracle/_ref/pgx_ref_driver is missing (build it with make -C oracle)")
    lap, wl = CASES[name]
    p = P.workload_params(wl)
    p[P.ADVANCED_GLOBAL_SOLVE] = 1
    n = lap[0] * lap[1] * lap[2]
    ref = oracle_runs.run(lap=lap, params=p, xtrue=oracle_runs.x_true(n, seed=7), apply_k=2)
    return ref, p


@pytest.mark.parametrize("name", list(CASES))
def test_usolve_fp64_matches_reference(name):
    from pargemslr_b200.handle import GemslrHandle
    ref, p = _run(name)
    st = from_dump(ref["setup"])
    assert st.solve_option == 1
    h = GemslrHandle(st, precision="fp64")
    ap = ref["apply"]
    n = h.n
    for k in range(int(ap["k"][0])):
        v = ap["in"][k * n:(k + 1) * n]
        z_ref = ap["out"][k * n:(k + 1) * n]
        err = np.linalg.norm(h.apply(v) - z_ref) / np.linalg.norm(z_ref)
        assert err <= 1e-9, f"apply {k}: relative difference {err:.3e}"
    b = pgxd.read(ref["problem"])["b"]
    x_ref = ref["solution"]["x"]
    x, r = h.solve(b, params=p)
    assert r["status"] == 0 and r["true_rel_res"] <= 1e-8
    assert abs(r["iters"] - ref["iters"]) <= 1, (r["iters"], ref["iters"])
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) <= 1e-6
    h.close()


@pytest.mark.parametrize("name", list(CASES))
def test_usolve_mixed_and_lanes(name):
    from pargemslr_b200.handle import GemslrHandle
    ref, p = _run(name)
    h = GemslrHandle(from_dump(ref["setup"]), precision="mixed")
    b = pgxd.read(ref["problem"])["b"]
    x, r = h.solve(b, params=p)
    assert r["status"] == 0 and r["true_rel_res"] <= 1e-8
    assert r["iters"] <= int(np.floor(1.15 * ref["iters"])) + 1, (r["iters"], ref["iters"])
    x_ref = ref["solution"]["x"]
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) <= 1e-6
    # four lanes in lockstep follow the option: each lane as the single solve
    rng = np.random.default_rng(3)
    B = np.vstack([b] + [2.0 * rng.random(h.n) - 1.0 for _ in range(3)])
    singles = [h.solve(bb, params=p) for bb in B]
    h.set_lanes(4)
    h.set_slots(2)
    X, res = h.solve_batch(B, params=p)
    for k in range(len(B)):
        assert res[k]["status"] == 0 and res[k]["true_rel_res"] <= 1e-8
        assert abs(res[k]["iters"] - singles[k][1]["iters"]) <= 1
        assert np.linalg.norm(X[k] - singles[k][0]) <= 1e-6 * np.linalg.norm(singles[k][0])
    h.close()


def test_usolve_systems_in_one_launch():
    from pargemslr_b200.handle import GemslrHandle
    from pargemslr_b200.systems import SystemsBatch
    hs, refs, B, ps = [], [], [], []
    for name in CASES:
        ref, p = _run(name)
        hs.append(GemslrHandle(from_dump(ref["setup"]), precision="fp64"))
        refs.append(ref)
        B.append(pgxd.read(ref["problem"])["b"])
        ps.append(p)
    sb = SystemsBatch(hs)
    X, R = sb.solve(B, params=ps[0])
    for k, ref in enumerate(refs):
        assert R[k]["status"] == 0 and R[k]["true_rel_res"] <= 1e-8, R[k]
        assert abs(R[k]["iters"] - ref["iters"]) <= 1, (R[k]["iters"], ref["iters"])
        x_ref = ref["solution"]["x"]
        assert np.linalg.norm(X[k] - x_ref) / np.linalg.norm(x_ref) <= 1e-6
    sb.close()
    for h in hs:
        h.close()
