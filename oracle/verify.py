"""The reference's ``--verify`` criterion and normwise residuals (oracle side).

include/verify.h:17-29 / :79-89 turn the in-place column-major factor into dense
L and U (unit diagonal on L for LU; the other triangle zeroed); :31-70 / :91-128 form
L*U (or L*L^T) and sum |A - L*U| over all entries; the run passes when that absolute
sum is <= 1e-6.  ``ref_error_*`` use the plain triple loop of oracle/gen_ref.c (same
loop order as the reference); ``*_fast`` use numpy's matmul for larger n.
"""
import numpy as np

from ._native import dptr, lib

REF_TOLERANCE = 1e-6  # include/verify.h:69 and :127


def split_lu(f: np.ndarray):
    l = np.tril(f, -1) + np.eye(f.shape[0])
    u = np.triu(f)
    return l, u


def split_chol(f: np.ndarray):
    return np.tril(f)


def ref_error_lu(a: np.ndarray, f: np.ndarray) -> float:
    a = np.ascontiguousarray(a)  # the reference indexes A row-major; A is symmetric there
    f = np.asfortranarray(f)
    return lib().oracle_ref_verify_lu(dptr(a), dptr(f), a.shape[0])


def ref_error_chol(a: np.ndarray, f: np.ndarray) -> float:
    a = np.ascontiguousarray(a)
    f = np.asfortranarray(f)
    return lib().oracle_ref_verify_chol(dptr(a), dptr(f), a.shape[0])


def error_lu_fast(a, f) -> float:
    l, u = split_lu(f)
    return float(np.abs(a - l @ u).sum())


def error_chol_fast(a, f) -> float:
    l = split_chol(f)
    return float(np.abs(a - l @ l.T).sum())


def normwise_residual_lu(a, f) -> float:
    l, u = split_lu(f)
    return float(np.linalg.norm(a - l @ u) / np.linalg.norm(a))


def normwise_residual_chol(a, f) -> float:
    l = split_chol(f)
    return float(np.linalg.norm(a - l @ l.T) / np.linalg.norm(a))


def probe_residual(a, f, kind: str, probes: int = 8, seed: int = 7) -> float:
    """||(A - L U) X||_F / ||A X||_F for a few random columns X: an O(n^2) estimate
    of the normwise residual that stays affordable at n = 24000."""
    n = a.shape[0]
    x = np.random.default_rng(seed).standard_normal((n, probes))
    if kind == "chol":
        l = np.tril(f)
        r = a @ x - l @ (l.T @ x)
    else:
        l = np.tril(f, -1)
        u = np.triu(f)
        ux = u @ x
        r = a @ x - (l @ ux + ux)
    return float(np.linalg.norm(r) / np.linalg.norm(a @ x))
