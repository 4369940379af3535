"""The FP64 block-tridiagonal solve (ss_solve_block_tridiagonal) against the oracle's sequential
block LDL^T on random symmetric positive definite systems, including chain lengths of the
512x512, 2-line-knot workload (64 frames: 16385 knots)."""
import numpy as np
import pytest

from oracle import oracle
from steadyscan_b200 import api

pytestmark = pytest.mark.gpu


def random_spd_chain(n, rng, cond=1e3):
    """Block-tridiagonal SPD system with 2x2 blocks from a random banded factor."""
    d = np.zeros((n, 3))
    c = np.zeros((max(n - 1, 0), 4))
    # A = B^T B + eps I with B block-bidiagonal
    Bd = rng.normal(size=(n, 2, 2))
    Bo = rng.normal(size=(max(n - 1, 0), 2, 2)) * 0.4
    for i in range(n):
        m = Bd[i].T @ Bd[i] + np.eye(2) / cond
        if i > 0:
            m += Bo[i - 1].T @ Bo[i - 1]
        d[i] = [m[0, 0], m[1, 1], 0.5 * (m[0, 1] + m[1, 0])]
    for i in range(n - 1):
        m = Bd[i].T @ Bo[i]  # coupling block between i (rows) and i+1 (cols)
        c[i] = [m[0, 0], m[1, 1], m[0, 1], m[1, 0]]
    b = rng.normal(size=(n, 2))
    return d, c, b


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 1000, 16385])
def test_matches_oracle_ldlt(n):
    rng = np.random.default_rng(n)
    d, c, b = random_spd_chain(n, rng)
    x_ref = oracle.block_tridiag_solve(d, c, b)
    x = api.solve_block_tridiagonal(d, c, b).cpu().numpy()
    scale = np.abs(x_ref).max()
    np.testing.assert_allclose(x, x_ref, rtol=0, atol=1e-9 * scale)
