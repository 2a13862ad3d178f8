"""Blocked Cholesky adjoint on the GPU (no reference counterpart): the reverse task graph
against the oracle's blocked sweep and closed form (FP64 within 1e-12 relative), batches of
mixed sizes in one launch, FP32 against FP64, and the torch.autograd.Function against
torch.linalg.cholesky's gradient and central finite differences on the GP loss
0.5 y^T A^-1 y + sum(log diag L) with A = K + 0.1 I, K an RBF kernel."""
import numpy as np
import pytest

from oracle import adjoint

pytestmark = pytest.mark.gpu


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, (n, n))
    return b @ b.T / n + np.eye(n)


def _col(x, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(x).T))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda().t()  # column-major (n, n) view


def _host(t):
    return np.asarray(t.t().contiguous().cpu().double().numpy().T)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("n,tile", [(64, 64), (100, 64), (128, 128), (300, 128), (513, 128), (1024, 128), (700, 256),
                                    (640, 64)])
def test_adjoint_matches_oracle(mtd, n, tile):
    a = _spd(n, n)
    L = np.linalg.cholesky(a)
    w = np.tril(np.random.default_rng(n + 1).standard_normal((n, n)))
    lc, gc = _col(L), _col(w)
    mtd.cholesky_adjoint(lc, gc, tile=tile)
    got = np.tril(_host(gc))
    assert _rel(got, adjoint.blocked(L, w, tile)) <= 1e-12
    assert _rel(got, adjoint.unblocked(L, w)) <= 1e-11
    # the strict upper triangle of Lbar's storage is untouched
    assert np.array_equal(np.triu(_host(gc), 1), np.triu(w, 1))


def test_batched_adjoint_mixed_sizes_one_launch(mtd):
    sizes = [64, 130, 256, 257, 511, 96]
    Ls, ws = [], []
    for i, n in enumerate(sizes):
        Ls.append(np.linalg.cholesky(_spd(n, 40 + i)))
        ws.append(np.tril(np.random.default_rng(50 + i).standard_normal((n, n))))
    adj = mtd.CholeskyAdjoint(sizes, tile=128, prec=mtd.PREC_FP64)
    assert adj.num_tasks() > len(sizes)
    lc = [_col(x) for x in Ls]
    gc = [_col(x) for x in ws]
    adj.run(lc, gc)
    ms = adj.status()
    assert ms > 0
    for L, w, g in zip(Ls, ws, gc):
        assert _rel(np.tril(_host(g)), adjoint.blocked(L, w, 128)) <= 1e-12
    adj.close()


def test_fp32_adjoint_close_to_fp64(mtd):
    import torch
    n = 384
    L = np.linalg.cholesky(_spd(n, 7))
    w = np.tril(np.random.default_rng(8).standard_normal((n, n)))
    lc, gc = _col(L, torch.float32), _col(w, torch.float32)
    mtd.cholesky_adjoint(lc, gc, tile=128)
    ref = adjoint.unblocked(L.astype(np.float32).astype(np.float64), w.astype(np.float32).astype(np.float64))
    assert _rel(np.tril(_host(gc)), ref) <= 1e-4


def _gp_loss_torch(L, y):
    import torch
    z = torch.linalg.solve_triangular(L, y.unsqueeze(-1), upper=False).squeeze(-1)
    return 0.5 * (z * z).sum() + torch.log(torch.diagonal(L, dim1=-2, dim2=-1)).sum()


@pytest.mark.parametrize("recompute", [False, True])
def test_autograd_gp_loss_matches_torch(mtd, recompute):
    import torch
    from mustard_b200 import autograd
    batch, n = 4, 256
    mats, ys = zip(*[adjoint.rbf_spd(n, 8, 100 + i) for i in range(batch)])
    a = torch.tensor(np.stack(mats), device="cuda", requires_grad=True)
    y = torch.tensor(np.stack(ys), device="cuda")
    _gp_loss_torch(autograd.cholesky(a, tile=128, recompute=recompute), y).backward()
    a_ref = a.detach().clone().requires_grad_(True)
    _gp_loss_torch(torch.linalg.cholesky(a_ref), y).backward()
    g, g_ref = a.grad.cpu().numpy(), a_ref.grad.cpu().numpy()
    assert _rel(g, g_ref) <= 1e-10
    # closed-form GP gradient 0.5 (A^-1 - A^-1 y y^T A^-1) for one matrix
    ai = np.linalg.inv(mats[0])
    u = ai @ ys[0]
    assert _rel(g[0], 0.5 * (ai - np.outer(u, u))) <= 1e-9


def test_autograd_central_finite_differences(mtd):
    import torch
    from mustard_b200 import autograd
    n = 200
    a_np, y_np = adjoint.rbf_spd(n, 8, 7)
    a = torch.tensor(a_np, device="cuda", requires_grad=True)
    y = torch.tensor(y_np, device="cuda")
    _gp_loss_torch(autograd.cholesky(a, tile=128), y).backward()
    g = a.grad.cpu().numpy()
    h = 1e-6
    for i, j in [(0, 0), (5, 3), (199, 0), (100, 100), (150, 77)]:
        e = np.zeros((n, n))
        e[i, j] = e[j, i] = 1.0
        fd = (adjoint.gp_loss(a_np + h * e, y_np) - adjoint.gp_loss(a_np - h * e, y_np)) / (2 * h)
        # a symmetric perturbation of the off-diagonal pair counts the gradient twice
        want = g[i, j] if i == j else 2.0 * g[i, j]
        assert abs(fd - want) <= 1e-6 * max(1.0, abs(fd)), (i, j, fd, want)


def test_autograd_fp32_close_to_fp64(mtd):
    import torch
    from mustard_b200 import autograd
    batch, n = 2, 320
    mats, ys = zip(*[adjoint.rbf_spd(n, 8, 300 + i) for i in range(batch)])
    grads = []
    for dt in (torch.float64, torch.float32):
        a = torch.tensor(np.stack(mats), device="cuda", dtype=dt, requires_grad=True)
        y = torch.tensor(np.stack(ys), device="cuda", dtype=dt)
        _gp_loss_torch(autograd.cholesky(a, tile=128), y).backward()
        grads.append(a.grad.double().cpu().numpy())
    assert _rel(grads[1], grads[0]) <= 5e-3
