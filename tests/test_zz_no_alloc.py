"""pgx_gemslr_solve_static: the solve for callers that cannot allocate.

Some callers of this library must not allocate device memory at solve time
(their device memory belongs to their own pool, or they cannot afford the
device-wide synchronisation of cudaMalloc).  pgx_gemslr_solve_static solves
with the Krylov basis in a fixed static pool of the library instead of an
allocated one.  These tests call it through the C ABI and compare it with
pgx_gemslr_solve on the same handle: same iteration count, solutions within
1e-12 relative, on two calls in a row (the second call finds the pool holding
the first call's basis).  The file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from pargemslr_b200 import _abi
from pargemslr_b200 import params as P
from pargemslr_b200 import problems

pytestmark = pytest.mark.gpu

POOL_BYTES = 32 << 20


def _static_solve(h, x, b, location, params):
    res = _abi.Result()
    rc = _abi.lib().pgx_gemslr_solve_static(h._h, x, b, location, _abi.ptr(params), C.byref(res))
    return rc, res


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_static_solve_matches_solve_twice(precision):
    import torch
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap2d_256")
    A = problems.laplacian(96, 96, 1)
    n = A[0].size - 1
    h = GemslrHandle.from_matrix(A, p, precision=precision)
    rng = np.random.default_rng(3)
    for call in range(2):
        b = rng.standard_normal(n)
        x_ref, r_ref = h.solve(b, params=p)
        # host vectors
        x = np.zeros(n)
        rc, res = _static_solve(h, _abi.ptr(x), _abi.ptr(b), _abi.LOCATION_HOST, p)
        _abi.check(rc)
        assert res.status == 0 and res.iters == r_ref["iters"], (call, res.iters, r_ref["iters"])
        assert res.true_rel_res <= 1e-8
        assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) <= 1e-12
        # device vectors
        bd = torch.tensor(b, device="cuda")
        xd = torch.zeros(n, dtype=torch.float64, device="cuda")
        rc, res = _static_solve(h, xd.data_ptr(), bd.data_ptr(), _abi.LOCATION_DEVICE, p)
        _abi.check(rc)
        assert res.iters == r_ref["iters"]
        xs = xd.cpu().numpy()
        assert np.linalg.norm(xs - x_ref) / np.linalg.norm(x_ref) <= 1e-12
    h.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_first_solve_of_a_fresh_handle_allocates_nothing(precision):
    """The static solve as the very first solve of a committed handle (no
    Krylov basis allocated yet) takes no device memory: the device's free
    memory is the same before and after it, and it equals the ordinary solve
    of a second handle over the same matrix."""
    import torch
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap2d_256")
    A = problems.laplacian(80, 80, 1)
    n = A[0].size - 1
    b = np.random.default_rng(11).standard_normal(n)
    # a warm-up handle: every kernel the static path launches is loaded once
    # (module loading is lazy) before the measured call
    warm = GemslrHandle.from_matrix(A, p, precision=precision)
    xw = np.zeros(n)
    _abi.check(_static_solve(warm, _abi.ptr(xw), _abi.ptr(b), _abi.LOCATION_HOST, p)[0])
    x_ref, r_ref = warm.solve(b, params=p)
    warm.close()
    fresh = GemslrHandle.from_matrix(A, p, precision=precision)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    x = np.zeros(n)
    rc, res = _static_solve(fresh, _abi.ptr(x), _abi.ptr(b), _abi.LOCATION_HOST, p)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    _abi.check(rc)
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert res.status == 0 and res.iters == r_ref["iters"]
    assert res.true_rel_res <= 1e-8
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) <= 1e-12
    fresh.close()


def test_static_solve_refuses_a_basis_larger_than_the_pool():
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap2d_256")
    A = problems.laplacian(160, 160, 1)
    n = A[0].size - 1
    h = GemslrHandle.from_matrix(A, p, precision="fp64")
    q = p.copy()
    q[P.SOLVER_KDIM] = 128  # V and Z of 25,600 x 129 doubles: 52.8 MB > 32 MiB
    assert 16 * n * 129 > POOL_BYTES
    assert 16 * n * (int(p[P.SOLVER_KDIM]) + 1) < POOL_BYTES
    b = np.ones(n)
    x = np.zeros(n)
    rc, _ = _static_solve(h, _abi.ptr(x), _abi.ptr(b), _abi.LOCATION_HOST, q)
    assert rc == _abi.ERROR_INVALID_PARAM
    assert "static pool" in _abi.lib().pgx_last_error().decode()
    # the refusal leaves the handle usable
    rc, res = _static_solve(h, _abi.ptr(x), _abi.ptr(b), _abi.LOCATION_HOST, p)
    _abi.check(rc)
    assert res.true_rel_res <= 1e-8
    h.close()
