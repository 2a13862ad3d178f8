"""Oracle for the pivoted LU (test infrastructure only).  The reference has no pivoted LU
(mustard/lu_mustard.cu:361-369 factors with ipiv = NULL); the operation is LAPACK's dgetrf,
so LAPACK (scipy.linalg.lapack.dgetrf) is the oracle, and ``blocked_getrf`` restates the
blocked algorithm the device task graph runs, step for step, so the two can be compared on
the CPU:

  for each block column k of width w (rows r0 = k*b ..):
    panel: for each column c of the panel, the pivot is the first row (at or below c) of
           largest |a|; the two panel rows are interchanged in full, the column below the
           pivot is scaled by 1/pivot (left as it is when the pivot is zero: LAPACK's info),
           and the rest of the panel gets the rank-1 update;
    the panel's interchanges are applied to the block columns right of it, U(k, j) =
    L_kk^-1 A(k, j), A(k+1:, j) -= L(k+1:, k) U(k, j);
  finally each block column gets the interchanges of the panels right of it.

ipiv is LAPACK's: 1-based, row i was interchanged with row ipiv[i]."""
import numpy as np
from scipy.linalg import lapack


def lapack_getrf(a):
    """(lu, ipiv 1-based, info) from LAPACK dgetrf."""
    lu, piv, info = lapack.dgetrf(np.asfortranarray(a, dtype=np.float64))
    return lu, piv.astype(np.int64) + 1, int(info)


def apply_ipiv(x, ipiv, start=0):
    """Rows of x interchanged as ipiv[start:] says, in order (LAPACK's dlaswp)."""
    x = np.array(x, copy=True)
    for r in range(start, len(ipiv)):
        p = int(ipiv[r]) - 1
        if p != r:
            x[[r, p]] = x[[p, r]]
    return x


def blocked_getrf(a, b):
    """The device graph's algorithm on the host: (lu, ipiv 1-based, info)."""
    a = np.array(a, dtype=np.float64, order="F", copy=True)
    n = a.shape[0]
    ipiv = np.zeros(n, dtype=np.int64)
    info = 0
    for r0 in range(0, n, b):
        w = min(b, n - r0)
        for c in range(w):
            col = r0 + c
            p = col + int(np.argmax(np.abs(a[col:, col])))  # argmax returns the first maximum
            ipiv[col] = p + 1
            if p != col:
                a[[col, p], r0:r0 + w] = a[[p, col], r0:r0 + w]
            piv = a[col, col]
            if piv != 0.0:
                a[col + 1:, col] *= 1.0 / piv
            elif info == 0:
                info = col + 1
            a[col + 1:, col + 1:r0 + w] -= np.outer(a[col + 1:, col], a[col, col + 1:r0 + w])
        if r0 + w < n:
            right = slice(r0 + w, n)
            for c in range(w):  # the panel's interchanges on the columns to its right
                col = r0 + c
                p = int(ipiv[col]) - 1
                if p != col:
                    a[[col, p], right] = a[[p, col], right]
            lkk = np.tril(a[r0:r0 + w, r0:r0 + w], -1) + np.eye(w)
            a[r0:r0 + w, right] = np.linalg.solve(lkk, a[r0:r0 + w, right])
            a[r0 + w:, right] -= a[r0 + w:, r0:r0 + w] @ a[r0:r0 + w, right]
    for r0 in range(0, n, b):  # the later panels' interchanges on each block column
        w = min(b, n - r0)
        for col in range(r0 + w, n):
            p = int(ipiv[col]) - 1
            if p != col:
                a[[col, p], r0:r0 + w] = a[[p, col], r0:r0 + w]
    return a, ipiv, info


def unpack(lu):
    """(L unit lower, U upper) of a packed factor."""
    n = lu.shape[0]
    return np.tril(lu, -1) + np.eye(n), np.triu(lu)


def residual(a, lu, ipiv):
    """||P A - L U||_F / ||A||_F."""
    l, u = unpack(lu)
    return np.linalg.norm(apply_ipiv(a, ipiv) - l @ u) / np.linalg.norm(a)


def random_matrix(n, seed):
    """Uniform [-1, 1) entries: partial pivoting interchanges most rows."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=(n, n))
