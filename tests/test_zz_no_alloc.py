"""ss_solve_block_tridiagonal_noalloc against ss_solve_block_tridiagonal, through the C ABI.

The no-allocation variant serves callers that cannot allocate device memory while they run (a
streaming acquisition loop, where cudaMalloc would synchronize the device and stall frames in
flight). Its workspace is a fixed array inside the library that every call reuses, so two calls in a
row must each give the allocating entry point's result, and sizes beyond the array are refused.
This file sorts last so that a run stopping at the first failure has run every other test first.
"""
import numpy as np
import pytest

from steadyscan_b200 import api
from tests.test_solve_gpu import random_spd_chain

pytestmark = pytest.mark.gpu

MAX_BLOCKS = 32768


def _check(n, seed):
    rng = np.random.default_rng(seed)
    d, c, b = random_spd_chain(n, rng)
    ref = api.solve_block_tridiagonal(d, c, b).cpu().numpy()
    got = api.solve_block_tridiagonal_noalloc(d, c, b).cpu().numpy()
    scale = np.abs(ref).max()
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-9 * scale)


def test_two_calls_in_a_row_match_allocating_entry():
    _check(16385, 1)   # a 64-frame chain of the 512x512, 2-line-knot workload
    _check(777, 2)     # a smaller chain right after: the workspace keeps the previous contents


def test_largest_size_and_refusal():
    _check(MAX_BLOCKS, 3)
    rng = np.random.default_rng(4)
    d, c, b = random_spd_chain(MAX_BLOCKS + 1, rng)
    with pytest.raises(api.SteadyScanError) as e:
        api.solve_block_tridiagonal_noalloc(d, c, b)
    assert e.value.code == -1 and "exceeds" in str(e.value)
