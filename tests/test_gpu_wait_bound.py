"""Bounded device-side waits: a wait that nothing satisfies ends with PGX_ERROR_TIMEOUT, and the GPU stays usable.

The triangular kernels that cross subdomains poll for values other CTAs publish; every poll loop has a bound.  The
self-check runs that kernel over two rows of which only the dependent one is scheduled, so the value it waits for is
never published: the wait can only end by its bound.  No fault, trap or endless loop is involved.  Afterwards an
ordinary solve on the same device must still succeed, and a handle whose bound is set small still solves (its
waits are satisfied long before the bound on this small problem) with identical results.
"""
import ctypes as C

import numpy as np
import pytest

from pargemslr_b200 import _abi
from pargemslr_b200 import params as P
from pargemslr_b200 import problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("polls", [1, 1000, 100000])
def test_unsatisfied_wait_times_out_and_the_gpu_stays_usable(polls):
    from pargemslr_b200.handle import GemslrHandle, init
    init(0)
    st = C.c_int32(-1)
    ms = C.c_double(0)
    _abi.check(_abi.lib().pgx_wait_selfcheck(polls, C.byref(st), C.byref(ms)))
    assert st.value == _abi.ERROR_TIMEOUT
    assert ms.value < 5000.0
    p = P.workload_params("lap2d_256")
    A = problems.laplacian(48, 48, 1)
    h = GemslrHandle.from_matrix(A, p, precision="fp64")
    x, r = h.solve(np.ones(h.n), params=p)
    assert r["status"] == 0 and r["true_rel_res"] <= 1e-8
    h.close()


def test_wait_limit_is_settable_and_checked():
    from pargemslr_b200.handle import GemslrHandle
    p = P.workload_params("lap2d_256")
    A = problems.laplacian(64, 64, 1)
    h = GemslrHandle.from_matrix(A, p, precision="fp64")
    b = np.random.default_rng(5).standard_normal(h.n)
    x0, r0 = h.solve(b, params=p)
    assert _abi.lib().pgx_gemslr_set_wait_limit(h._h, 0) == _abi.ERROR_INVALID_PARAM
    _abi.check(_abi.lib().pgx_gemslr_set_wait_limit(h._h, 1 << 20))
    x1, r1 = h.solve(b, params=p)
    assert r1["status"] == 0 and r1["iters"] == r0["iters"]
    assert np.array_equal(x0, x1)
    h.close()
