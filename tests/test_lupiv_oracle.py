"""The pivoted-LU oracle (oracle/lupiv.py) pinned against LAPACK dgetrf: the restated blocked
algorithm of the device task graph chooses the same interchanges and gives the same factors
(to rounding) on random, ragged, tied and singular inputs."""
import numpy as np
import pytest

from oracle import lupiv


@pytest.mark.parametrize("n,b", [(64, 64), (200, 64), (300, 128), (257, 64), (512, 256), (100, 128)])
def test_blocked_restatement_matches_lapack(n, b):
    a = lupiv.random_matrix(n, 10 + n)
    lu, ipiv, info = lupiv.blocked_getrf(a, b)
    ref, rpiv, rinfo = lupiv.lapack_getrf(a)
    assert info == rinfo == 0
    assert np.array_equal(ipiv, rpiv)
    assert np.abs(lu - ref).max() <= 1e-12 * np.abs(ref).max()
    assert lupiv.residual(a, lu, ipiv) < 1e-14


def test_ties_take_the_first_row():
    # integer matrix with repeated column maxima: dgetrf's idamax takes the first of them
    rng = np.random.default_rng(3)
    a = rng.integers(-3, 4, size=(96, 96)).astype(np.float64) + 8 * np.eye(96)
    a[:, 0] = 4.0  # every row ties in column 0
    lu, ipiv, info = lupiv.blocked_getrf(a, 32)
    ref, rpiv, rinfo = lupiv.lapack_getrf(a)
    assert ipiv[0] == 1 and np.array_equal(ipiv, rpiv) and info == rinfo


def test_singular_reports_the_first_zero_pivot():
    a = lupiv.random_matrix(128, 5)
    a[:, 70] = 0.0
    lu, ipiv, info = lupiv.blocked_getrf(a, 64)
    ref, rpiv, rinfo = lupiv.lapack_getrf(a)
    assert info == rinfo == 71
    assert np.array_equal(ipiv, rpiv)
    assert np.allclose(lu, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_apply_ipiv_is_dlaswp():
    a = np.arange(16.0).reshape(4, 4)
    out = lupiv.apply_ipiv(a, np.array([3, 3, 4, 4]))
    assert np.array_equal(out[:, 0], [8.0, 0.0, 12.0, 4.0])
