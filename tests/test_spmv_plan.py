"""The SpMV variant choice from the row-length histogram (host side, no GPU).

pgx_csr_spmv_plan picks S lanes per row so that the 90th-percentile row fits one batch of S * 4 unrolled loads, and
the merge-path SpMV when the rows are skewed.  The 3D Laplacian (7 per row) takes 2 lanes, the uniform random
matrix of the serving workload (7-27 per row) 8, and a matrix whose few long rows hold most of the nonzeros takes
the merge path.
"""
import ctypes as C

import numpy as np
import pytest

from pargemslr_b200 import _abi
from pargemslr_b200 import problems


def plan(A):
    rp, cj, va = A
    keep = []
    Ac = _abi.csr_struct(rp, cj, va, rp.size - 1, rp.size - 1, keep=keep)
    lanes, merge = C.c_int32(0), C.c_int32(0)
    _abi.check(_abi.lib().pgx_csr_spmv_plan(C.byref(Ac), C.byref(lanes), C.byref(merge)))
    return lanes.value, bool(merge.value)


def expected(rp):
    lens = np.diff(rp)
    p90 = np.sort(lens)[int(np.ceil(0.9 * lens.size)) - 1]
    S = 2
    while S < 32 and S * 4 < p90:
        S *= 2
    batch = S * 4
    merge = lens.max() > 16 * batch and lens[lens > 4 * batch].sum() * 10 > lens.sum()
    return S, bool(merge)


@pytest.mark.parametrize("make", [
    lambda: problems.laplacian(24, 24, 24),
    lambda: problems.laplacian(64, 64, 1),
    lambda: problems.random_diag_dominant(5000, 3),
    lambda: problems.random_skewed(5000, 4),
    lambda: problems.random_skewed(5000, 5, heavy_frac=0.001),
])
def test_plan_follows_the_histogram_rule(make):
    A = make()
    assert plan(A) == expected(A[0])


def test_plan_of_the_workloads():
    assert plan(problems.laplacian(24, 24, 24)) == (2, False)
    assert plan(problems.random_diag_dominant(5000, 3)) == (8, False)
    assert plan(problems.random_skewed(5000, 4))[1] is True


def test_plan_refuses_bad_input():
    assert _abi.lib().pgx_csr_spmv_plan(None, None, None) == _abi.ERROR_INVALID_PARAM
