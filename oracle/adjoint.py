"""Cholesky adjoint oracle (test infrastructure: only tests and benchmark checks use it).

No counterpart in the reference.  Reverse-mode derivative of A = L L^T, lower triangles:
given L and Lbar = dLoss/dL, Abar = dLoss/dA with respect to the lower triangle of A.

- ``unblocked``: the closed form M = L^-T Phi(L^T Lbar) L^-1, Phi = lower triangle with the
  diagonal halved; Abar = tril(M + M^T) - diag(M) (I. Murray, "Differentiation of the
  Cholesky decomposition", arXiv:1602.07527, 2016, eq. for the symbolic adjoint).
- ``blocked``: the reverse sweep over block columns that the GPU task graph runs
  (mustard_b200/csrc/adjoint_ops.cuh), in the same order and with the same 64-block
  diagonal adjoints, so the two agree to rounding.
- ``symmetric``: the symmetric gradient (Abar + Abar^T) / 2 with the diagonal kept, the
  convention of torch.linalg.cholesky's gradient.
Pinned in tests/test_adjoint_oracle.py against central finite differences and against
torch.linalg.cholesky's autograd (CPU, float64).
"""
import numpy as np
from scipy.linalg import solve_triangular


def phi(x):
    y = np.tril(x)
    y[np.diag_indices_from(y)] *= 0.5
    return y


def _m_of(L, Lbar):
    p = phi(L.T @ np.tril(Lbar))
    t = solve_triangular(L, p.T, lower=True, trans="T").T  # p L^-1 = (L^-T p^T)^T
    return solve_triangular(L, t, lower=True, trans="T")  # L^-T (p L^-1)


def unblocked(L, Lbar):
    m = _m_of(np.asarray(L, dtype=np.float64), np.asarray(Lbar, dtype=np.float64))
    return np.tril(m + m.T) - np.diag(np.diag(m))


def symmetric(abar):
    low = np.tril(abar)
    return 0.5 * (low + low.T)


def _diag_block(D, Dbar):
    """64-block diagonal adjoint: (Sbar lower, Y = M + M^T)."""
    w = solve_triangular(D, np.eye(D.shape[0]), lower=True)
    m = w.T @ phi(D.T @ np.tril(Dbar)) @ w
    return np.tril(m + m.T) - np.diag(np.diag(m)), m + m.T


def _diag_tile(D, G, nb=64):
    """Adjoint of one diagonal tile by the in-tile sweep over 64-blocks; returns (G, Y)."""
    G = np.tril(G.copy())
    tn = D.shape[0]
    Y = np.zeros((tn, tn))
    s = (tn + nb - 1) // nb
    for b in range(s - 1, -1, -1):
        bo, bn = b * nb, min(nb, tn - b * nb)
        lo = bo + bn
        W = solve_triangular(D[bo:lo, bo:lo], np.eye(bn), lower=True)
        if lo < tn:
            G[lo:, bo:lo] = G[lo:, bo:lo] @ W
            G[bo:lo, bo:lo] -= np.tril(G[lo:, bo:lo].T @ D[lo:, bo:lo])
        sb, yb = _diag_block(D[bo:lo, bo:lo], G[bo:lo, bo:lo])
        G[bo:lo, bo:lo] = sb
        Y[bo:lo, bo:lo] = yb
        for kb in range(0, bo, nb):
            ke = min(kb + nb, bo)
            if lo < tn:
                G[lo:, kb:ke] -= G[lo:, bo:lo] @ D[bo:lo, kb:ke]
                G[bo:lo, kb:ke] -= G[lo:, bo:lo].T @ D[lo:, kb:ke]
            G[bo:lo, kb:ke] -= yb @ D[bo:lo, kb:ke]
    low = np.tril(G, -1)
    for b in range(s):
        bo, lo = b * nb, min((b + 1) * nb, tn)
        low[bo:lo, bo:lo] = 0.0
    Y += low + low.T
    return G, Y


def blocked(L, Lbar, tile):
    """The GPU's reverse sweep with block columns of width ``tile`` (64 or 128)."""
    L = np.asarray(L, dtype=np.float64)
    n = L.shape[0]
    G = np.tril(np.asarray(Lbar, dtype=np.float64)).copy()
    nb = (n + tile - 1) // tile
    for j in range(nb - 1, -1, -1):
        jt, lo = j * tile, min((j + 1) * tile, n)
        if lo < n:
            D = L[jt:lo, jt:lo]
            G[lo:, jt:lo] = solve_triangular(D, G[lo:, jt:lo].T, lower=True, trans="T").T  # Cbar D^-1
            G[jt:lo, jt:lo] -= np.tril(G[lo:, jt:lo].T @ L[lo:, jt:lo])
        g, y = _diag_tile(L[jt:lo, jt:lo], G[jt:lo, jt:lo])
        G[jt:lo, jt:lo] = g
        for k in range(j):
            kt, ke = k * tile, (k + 1) * tile
            if lo < n:
                G[lo:, kt:ke] -= G[lo:, jt:lo] @ L[jt:lo, kt:ke]
                G[jt:lo, kt:ke] -= G[lo:, jt:lo].T @ L[lo:, kt:ke]
            G[jt:lo, kt:ke] -= y @ L[jt:lo, kt:ke]
    return np.tril(G)


def rbf_spd(n, d, seed, lengthscale=1.0, jitter=0.1):
    """A = K + jitter I, K the RBF kernel over n points in R^d drawn i.i.d. N(0, 1), and a
    right-hand side y ~ N(0, 1) (seeded)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, d))
    sq = np.sum(x * x, axis=1)
    d2 = np.maximum(sq[:, None] + sq[None, :] - 2.0 * x @ x.T, 0.0)
    a = np.exp(-0.5 * d2 / lengthscale ** 2) + jitter * np.eye(n)
    return a, rng.standard_normal(n)


def gp_loss(a, y):
    """0.5 y^T A^-1 y + sum(log diag L), L = chol(A)."""
    L = np.linalg.cholesky(a)
    z = solve_triangular(L, y, lower=True)
    return 0.5 * float(z @ z) + float(np.sum(np.log(np.diag(L))))


def gp_lbar(L, y):
    """dLoss/dL of gp_loss (lower triangle): with z = L^-1 y and u = L^-T z,
    d(0.5 z^T z) = -u^T dL z, so Lbar = tril(-u z^T) + diag(1 / L_ii)."""
    z = solve_triangular(L, y, lower=True)
    u = solve_triangular(L, z, lower=True, trans="T")
    lbar = np.tril(-np.outer(u, z))
    lbar[np.diag_indices_from(lbar)] += 1.0 / np.diag(L)
    return lbar
