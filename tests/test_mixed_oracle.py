"""The mixed-precision checker (oracle/mixed.py) pinned on CPU: the conditioned inputs have the
condition numbers they are built for, the error measures are the normwise infinity-norm ones
the solver reports, iterative refinement with a factor rounded to 11 significant bits (the
TF32 operand precision) reaches FP64 backward error at kappa = 1e2 under that measure, and the
restated refinement loop behaves as Carson & Higham's analysis says: with a preconditioner of
low-precision quality at kappa * u ~ 50, plain IR stalls and GMRES-IR converges."""
import numpy as np
import pytest
from scipy.linalg import cholesky, solve_triangular

from oracle import mixed


@pytest.mark.parametrize("n,kappa,tol", [(256, 1e2, 0.02), (400, 1e5, 0.10)])
def test_inputs_have_the_condition_number_asked_for(n, kappa, tol):
    # cond2(A) ~= kappa holds while alpha is far above the smallest eigenvalue of B B^T / n
    # (about 1 / (3 n^2)); at the configs' N = 32768 that covers kappa up to 1e8
    a = mixed.spd_kappa(n, kappa, 3)
    assert np.allclose(a, a.T) and np.linalg.eigvalsh(a)[0] > 0
    assert abs(mixed.cond2(a) / kappa - 1) < tol


def test_inputs_are_seeded():
    assert np.array_equal(mixed.spd_kappa(64, 1e2, 7), mixed.spd_kappa(64, 1e2, 7))
    assert not np.array_equal(mixed.spd_kappa(64, 1e2, 7), mixed.spd_kappa(64, 1e2, 8))
    b = mixed.rhs(64, 3, 9)
    assert b.shape == (64, 3) and b.flags.f_contiguous
    assert np.array_equal(b, mixed.rhs(64, 3, 9))


def test_error_measures_on_a_hand_example():
    a = np.array([[4.0, 1.0], [1.0, 3.0]])       # ||A||_inf = 5
    x = np.array([[1.0], [2.0]])                   # ||x||_inf = 2
    b = a @ x + np.array([[0.0], [0.5]])           # residual 0.5, ||b||_inf = 7.5
    assert mixed.backward_error(a, x, b) == pytest.approx(0.5 / (5 * 2 + 7.5))
    # two columns: the worse one counts
    x2 = np.hstack([x, x])
    b2 = np.hstack([a @ x, b])
    assert mixed.backward_error(a, x2, b2) == pytest.approx(0.5 / 17.5)
    assert mixed.forward_error(np.array([[1.0], [2.2]]), x) == pytest.approx(0.2 / 2)
    assert mixed.forward_error(x, x) == 0.0


def test_fp64_solve_has_roundoff_backward_error():
    a = mixed.spd_kappa(200, 1e5, 11)
    b = mixed.rhs(200, 4, 12)
    assert mixed.backward_error(a, mixed.solve_fp64(a, b), b) < 1e-15


def _round_bits(x, p):
    m, e = np.frexp(x)
    return np.ldexp(np.round(m * 2.0 ** p) / 2.0 ** p, e)


def test_refinement_with_an_11_bit_factor_reaches_fp64_accuracy():
    n = 256
    a = mixed.spd_kappa(n, 1e2, 5)
    b = mixed.rhs(n, 2, 6)
    low = _round_bits(cholesky(a, lower=True), 11)

    def solve_low(r):
        return solve_triangular(low.T, solve_triangular(low, r, lower=True), lower=False)

    x = solve_low(b)
    first = mixed.backward_error(a, x, b)
    assert 1e-7 < first < 1e-3  # about the factor's precision, far from FP64
    for _ in range(6):
        x = x + solve_low(b - a @ x)  # residual and update in FP64
    assert mixed.backward_error(a, x, b) < 1e-15
    assert mixed.forward_error(x, mixed.solve_fp64(a, b)) < 1e2 * 1e-13


def _shifted_low_precision_preconditioner(a, seed):
    """M = A + E, E = u ||A||_inf (G + 4 I), u = 2^-11 (TF32), G symmetric with ||G||_2 = 1: a
    perturbation of a low-precision factorisation's size, shifted like the solver tests shift
    the diagonal to keep the factor positive definite.  Returns a solve with M."""
    n = a.shape[0]
    g = np.random.default_rng(seed).standard_normal((n, n))
    g = (g + g.T) / 2
    g /= np.linalg.norm(g, 2)
    u = 2.0 ** -11
    low = cholesky(a + u * np.abs(a).sum(axis=1).max() * (g + 4 * np.eye(n)), lower=True)
    return lambda r: solve_triangular(low.T, solve_triangular(low, r, lower=True), lower=False)


def test_gmres_ir_converges_where_plain_ir_stalls():
    # kappa * u ~ 50: I - M^-1 A has spectral radius ~0.999 (plain IR crawls) while M^-1 A is
    # conditioned ~1e3 (GMRES resolves it) -- the regime of the solver's kappa = 1e5 runs
    a = mixed.spd_kappa(300, 1e5, 5)
    b = mixed.rhs(300, 1, 6)[:, 0]
    solve_m = _shifted_low_precision_preconditioner(a, 7)
    _, it, _, berr, ok = mixed.refine(a, b, solve_m, "ir", max_iter=30)
    assert not ok and it == 30 and berr > 1e-8
    x, it, inner, berr, ok = mixed.refine(a, b, solve_m, "gmres-ir", max_iter=30)
    assert ok and berr <= 1e-13 and it <= 6 and inner > it
    assert mixed.forward_error(x[:, None], mixed.solve_fp64(a, b[:, None])) <= 1e5 * 1e-12


def test_gmres_ir_needs_fewer_outer_iterations_at_kappa_1e2():
    a = mixed.spd_kappa(300, 1e2, 5)
    b = mixed.rhs(300, 1, 6)[:, 0]
    solve_m = _shifted_low_precision_preconditioner(a, 7)
    _, it_ir, _, berr_ir, ok_ir = mixed.refine(a, b, solve_m, "ir", max_iter=60)
    _, it_g, _, berr_g, ok_g = mixed.refine(a, b, solve_m, "gmres-ir", max_iter=60)
    assert ok_ir and ok_g and berr_ir <= 1e-13 and berr_g <= 1e-13
    assert it_g < it_ir
