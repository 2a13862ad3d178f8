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
"""
import numpy as np
from scipy.linalg import cho_factor, cho_solve

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
