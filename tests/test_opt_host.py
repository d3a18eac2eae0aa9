"""Host-side optimizer pieces (no GPU): the fluence-smoothness operator D_b
against the oracle's restatement of fluenceGradInit, block assembly, and the
oracle's optimizer against its own known answers (the prox constants of
IMRTOptimize_var1.cu:3-6 and the closed form of the half-norm prox)."""
import numpy as np
import pytest

import oracle
from fastdose_b200 import optimize


@pytest.mark.parametrize("n,seed", [(4, 0), (10, 1), (16, 2), (1, 3)])
def test_fluence_grad_matches_oracle(n, seed):
    rng = np.random.default_rng(seed)
    act = (rng.random(n * n) < 0.7).astype(np.uint8)
    got = optimize.fluence_grad(n, act)
    ref = oracle.fluence_grad(n, act)
    for a, b in zip(got[:3], ref[:3]):
        np.testing.assert_array_equal(a, b)
    assert got[3] == ref[3]


def test_fluence_grad_full_map_rows():
    n = 5
    off, col, val, na = optimize.fluence_grad(n, np.ones(n * n, np.uint8))
    assert na == n * n
    assert len(off) - 1 == 2 * n * (n - 1)  # x pairs then y pairs
    np.testing.assert_array_equal(val[:2], [-1.0, 1.0])
    np.testing.assert_array_equal(col[:2], [0, 1])
    np.testing.assert_array_equal(col[2 * n * (n - 1): 2 * n * (n - 1) + 2], [0, n])


def test_block_diag_shapes():
    b1 = optimize.fluence_grad(3, np.ones(9, np.uint8))
    b2 = optimize.fluence_grad(2, np.array([1, 1, 0, 1], np.uint8))
    off, col, val, nc = optimize.block_diag([b1, b2])
    assert nc == 9 + 3
    assert len(off) - 1 == (len(b1[0]) - 1) + (len(b2[0]) - 1)
    assert col[len(b1[1]):].min() >= 9


def test_oracle_t_hat_known_answers():
    # alpha above 2 sqrt(6) / 9 -> 0; alpha -> 0 -> scale 1
    assert oracle.that(1.0, 0.6) == 0.0
    assert abs(oracle.that(1e6, 1e-9) - 1.0) < 1e-6
    # the scale s minimises tau * |s g|^(1/2) + (s - 1)^2 |g|^2 / 2 along g
    for nrm2, tau in [(4.0, 0.3), (1.0, 0.2), (9.0, 1.0)]:
        s = oracle.that(nrm2, tau)
        g = np.sqrt(nrm2)
        f = lambda q: tau * np.sqrt(q * g) + 0.5 * (q - 1) ** 2 * nrm2  # noqa: E731
        grid = np.linspace(1e-3, 1.0, 20001)
        assert f(s) <= f(grid).min() + 1e-6


def test_reference_x0_is_glibc_rand():
    """The beam-orientation loop's initial fluence: srand(10086), then
    (float)rand() / RAND_MAX, checked against this host's C library."""
    import ctypes

    import numpy as np

    from fastdose_b200 import optimize

    libc = ctypes.CDLL("libc.so.6")
    libc.srand(10086)
    ref = np.array([np.float32(libc.rand()) / np.float32(2147483647) for _ in range(2000)], np.float32)
    np.testing.assert_array_equal(optimize.reference_x0(2000), ref)
    libc.srand(7)
    ref7 = np.array([np.float32(libc.rand()) / np.float32(2147483647) for _ in range(50)], np.float32)
    np.testing.assert_array_equal(optimize.reference_x0(50, seed=7), ref7)
