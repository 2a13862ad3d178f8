"""Input generators (oracle side).

``ref_spd``      -- the reference's generator, include/gen.h:23-38: glibc ``srand(420)``,
                    upper triangle of rand()/RAND_MAX, mirrored, +n on the diagonal.
                    Used for both LU and Cholesky by the reference drivers
                    (lu_mustard.cu:260, cholesky_mustard.cu:139).
``uniform_pm1``  -- counter-based uniform[-1, 1) stream: entry ``idx`` (column-major
                    linear index) of stream ``seed`` is a SplitMix64 finaliser of
                    ``seed * 0x9E3779B97F4A7C15 + (idx + 1) * 0xD1B54A32D192ED03``,
                    top 53 bits scaled to [0, 1), then ``2u - 1``.  The CUDA generator
                    in mustard_b200/csrc/gen.cu computes the same bits.
``lu_input``     -- U[-1, 1] + n I (column diagonally dominant: partial pivoting makes
                    no swaps, so no-pivot LU equals LAPACK's dgetrf here).
``spd_input``    -- B B^T / n + alpha I with B = uniform_pm1(n, n, seed).
All arrays are returned column-major (Fortran order).
"""
import numpy as np

from ._native import dptr, lib

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_GOLD = np.uint64(0x9E3779B97F4A7C15)
_STEP = np.uint64(0xD1B54A32D192ED03)


def _mix64(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def uniform_bits(count: int, seed: int, offset: int = 0) -> np.ndarray:
    idx = np.arange(offset, offset + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) * _GOLD + (idx + np.uint64(1)) * _STEP
        return _mix64(z)


def uniform_pm1(rows: int, cols: int, seed: int) -> np.ndarray:
    bits = uniform_bits(rows * cols, seed)
    u = (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    v = 2.0 * u - 1.0
    return v.reshape((cols, rows)).T  # column-major: idx = i + j * rows


def ref_spd(n: int) -> np.ndarray:
    a = np.empty((n, n), dtype=np.float64)  # row-major buffer as in the reference
    lib().oracle_ref_spd(dptr(a), n)
    return np.asfortranarray(a)  # symmetric: same matrix in column-major order


def lu_input(n: int, seed: int) -> np.ndarray:
    a = np.asfortranarray(uniform_pm1(n, n, seed))
    a[np.arange(n), np.arange(n)] += float(n)
    return a


def spd_input(n: int, seed: int, alpha: float = 1.0) -> np.ndarray:
    b = uniform_pm1(n, n, seed)
    a = (b @ b.T) / float(n)
    a[np.arange(n), np.arange(n)] += alpha
    return np.asfortranarray(a)
