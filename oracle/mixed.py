"""Oracle side of the mixed-precision solver checks (test infrastructure only).

``spd_kappa(n, kappa, seed)``  -- B B^T / n + alpha I with alpha = (4/3) / (kappa - 1): the
                                 spectrum of B B^T / n (B = U[-1, 1), variance 1/3) fills
                                 [~0, 4/3], so cond_2(A) ~= kappa (the configs' inputs) while
                                 alpha is far above the smallest eigenvalue of B B^T / n,
                                 about 1 / (3 n^2) (at n = 32768: kappa up to 1e8)
``rhs(n, k, seed)``            -- right-hand sides with i.i.d. N(0, 1) entries
``solve_fp64(a, b)``           -- LAPACK dpotrf/dpotrs reference solution in FP64
``backward_error(a, x, b)``    -- max over columns of ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)
``forward_error(x, x_ref)``    -- max over columns of ||x - x_ref||_inf / ||x_ref||_inf
``gmres_correction``, ``refine`` -- the refinement loop of the product's solver (IR, and
                                 GMRES-IR after Carson & Higham, SIAM J. Sci. Comput. 39 (2017),
                                 40 (2018)) restated for one right-hand side, with the
                                 preconditioner solve passed in
"""
import numpy as np
from scipy.linalg import cho_factor, cho_solve, solve_triangular

from . import gen


def alpha_for_kappa(kappa: float) -> float:
    return (4.0 / 3.0) / (kappa - 1.0)


def spd_kappa(n: int, kappa: float, seed: int) -> np.ndarray:
    return gen.spd_input(n, seed, alpha=alpha_for_kappa(kappa))


def rhs(n: int, k: int, seed: int) -> np.ndarray:
    return np.asfortranarray(np.random.default_rng(seed).standard_normal((n, k)))


def solve_fp64(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return cho_solve(cho_factor(a, lower=True), b)


def backward_error(a: np.ndarray, x: np.ndarray, b: np.ndarray) -> float:
    r = b - a @ x
    an = np.abs(a).sum(axis=1).max()
    num = np.abs(r).max(axis=0)
    den = an * np.abs(x).max(axis=0) + np.abs(b).max(axis=0)
    return float((num / den).max())


def forward_error(x: np.ndarray, x_ref: np.ndarray) -> float:
    return float((np.abs(x - x_ref).max(axis=0) / np.abs(x_ref).max(axis=0)).max())


def cond2(a: np.ndarray) -> float:
    w = np.linalg.eigvalsh(a)
    return float(w[-1] / w[0])


def gmres_correction(apply_a, apply_minv, r, rel_tol=1e-4, m=50):
    """One GMRES(m) cycle on M^-1 A d = M^-1 r, as the solver's correction step runs it: FP64
    Krylov basis, classical Gram-Schmidt applied twice, Givens rotations, stopping once the
    preconditioned residual is below rel_tol of its start.  Returns (d, inner iterations)."""
    v0 = apply_minv(r)
    beta = np.linalg.norm(v0)
    if beta == 0:
        return np.zeros_like(r), 0
    basis = [v0 / beta]
    h_all = np.zeros((m + 1, m))
    cs, sn, g = np.zeros(m), np.zeros(m), np.zeros(m + 1)
    g[0] = beta
    k = 0
    while k < m:
        w = apply_minv(apply_a(basis[k]))
        h = np.zeros(k + 2)
        for _ in range(2):
            c = np.array([v @ w for v in basis[:k + 1]])
            w = w - sum(ci * v for ci, v in zip(c, basis))
            h[:k + 1] += c
        hn = np.linalg.norm(w)
        h[k + 1] = hn
        if hn > 0:
            basis.append(w / hn)
        for i in range(k):
            t = cs[i] * h[i] + sn[i] * h[i + 1]
            h[i + 1] = -sn[i] * h[i] + cs[i] * h[i + 1]
            h[i] = t
        den = np.hypot(h[k], h[k + 1])
        cs[k], sn[k] = (h[k] / den, h[k + 1] / den) if den > 0 else (1.0, 0.0)
        h[k], h[k + 1] = den, 0.0
        g[k + 1] = -sn[k] * g[k]
        g[k] = cs[k] * g[k]
        h_all[:k + 1, k] = h[:k + 1]
        k += 1
        if abs(g[k]) <= rel_tol * beta or hn == 0:
            break
    y = solve_triangular(h_all[:k, :k], g[:k])
    return sum(yi * v for yi, v in zip(y, basis)), k


def refine(a, b, solve_m, method, tol=1e-13, max_iter=30):
    """x = 0, then x += correction until backward_error <= tol (IR: d = M^-1 r; GMRES-IR:
    d from gmres_correction), all in FP64.  Returns (x, iterations, inner, berr, converged)."""
    x = np.zeros_like(b)
    it = inner = 0
    while True:
        if it == 0:
            r, berr = b.copy(), 1.0
        else:
            r = b - a @ x
            berr = backward_error(a, x[:, None], b[:, None])
        if it > 0 and berr <= tol:
            return x, it, inner, berr, True
        if it >= max_iter:
            return x, it, inner, berr, False
        if method == "ir":
            d = solve_m(r)
        else:
            d, k = gmres_correction(lambda v: a @ v, solve_m, r)
            inner += k
        x = x + d
        it += 1
