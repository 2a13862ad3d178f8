"""The Cholesky adjoint oracle, pinned on the CPU: the closed form against central finite
differences and against torch.linalg.cholesky's autograd (float64), and the blocked
reverse sweep (the GPU's algorithm) against the closed form."""
import numpy as np
import pytest

from oracle import adjoint


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, (n, n))
    return b @ b.T / n + np.eye(n)


def _sym_perturb_grad(f, a, i, j, h):
    """d f / d a_ij for the symmetric variable a_ij = a_ji (central difference)."""
    e = np.zeros_like(a)
    e[i, j] = e[j, i] = 1.0
    return (f(a + h * e) - f(a - h * e)) / (2.0 * h)


@pytest.mark.parametrize("n", [5, 17])
def test_closed_form_matches_finite_differences(n):
    a = _spd(n, 1)
    rng = np.random.default_rng(2)
    w = np.tril(rng.standard_normal((n, n)))
    loss = lambda x: float(np.sum(w * np.linalg.cholesky(x)))  # Lbar = w
    L = np.linalg.cholesky(a)
    abar = adjoint.unblocked(L, w)
    for i, j in [(0, 0), (n - 1, 0), (n // 2, n // 3), (n - 1, n - 1), (3, 2)]:
        fd = _sym_perturb_grad(loss, a, i, j, 1e-6)
        assert abs(fd - abar[i, j]) <= 1e-7 * max(1.0, abs(fd)), (i, j, fd, abar[i, j])


def test_closed_form_matches_torch_autograd():
    torch = pytest.importorskip("torch")
    n = 40
    a = _spd(n, 3)
    w = np.tril(np.random.default_rng(4).standard_normal((n, n)))
    at = torch.tensor(a, requires_grad=True)
    (torch.linalg.cholesky(at) * torch.tensor(w)).sum().backward()
    g_torch = at.grad.numpy()
    L = np.linalg.cholesky(a)
    g = adjoint.symmetric(adjoint.unblocked(L, w))
    assert np.max(np.abs(g - g_torch)) <= 1e-12 * np.max(np.abs(g_torch))


def test_gp_loss_gradient_matches_finite_differences():
    a, y = adjoint.rbf_spd(30, 8, 5)
    L = np.linalg.cholesky(a)
    abar = adjoint.unblocked(L, adjoint.gp_lbar(L, y))
    for i, j in [(0, 0), (7, 3), (29, 0), (15, 15), (29, 28)]:
        fd = _sym_perturb_grad(lambda x: adjoint.gp_loss(x, y), a, i, j, 1e-6)
        assert abs(fd - abar[i, j]) <= 1e-6 * max(1.0, abs(fd)), (i, j, fd, abar[i, j])
    # the GP loss gradient in closed form: 0.5 (A^-1 - A^-1 y y^T A^-1), symmetric convention
    ai = np.linalg.inv(a)
    u = ai @ y
    g = 0.5 * (ai - np.outer(u, u))
    assert np.max(np.abs(adjoint.symmetric(abar) - g)) <= 1e-10 * np.max(np.abs(g))


@pytest.mark.parametrize("n,tile", [(64, 64), (128, 64), (200, 64), (256, 128), (300, 128), (77, 128), (600, 256)])
def test_blocked_sweep_matches_closed_form(n, tile):
    a = _spd(n, 6 + n)
    L = np.linalg.cholesky(a)
    w = np.tril(np.random.default_rng(n).standard_normal((n, n)))
    ref = adjoint.unblocked(L, w)
    got = adjoint.blocked(L, w, tile)
    assert np.max(np.abs(got - ref)) <= 1e-11 * np.max(np.abs(ref))
