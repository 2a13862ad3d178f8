"""The north-star extensions checked at their benchmark sizes (the other GPU tests use reduced
ones): config 3's full draw of 4096 batched SPD solves, config 4's 64 x 2048 Cholesky adjoint,
and config 2's hardest condition number (1e8) with the outcome the solver reports checked
against the host's own backward error.  All inputs are the benchmarks' seeded synthetic
ones (mustard_b200.batch_bench, mustard_b200.adjoint_bench, oracle.mixed)."""
import numpy as np
import pytest

from oracle import mixed

pytestmark = pytest.mark.gpu


def _host(t):
    return np.asfortranarray(t.t().contiguous().cpu().double().numpy().T)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_config3_full_draw_4096_batched_solves(mtd, prec):
    """4096 SPD matrices, N uniform in {32, 64, ..., 1024}, B B^T / N + I, 1-16 right-hand
    sides each: one merged factor launch, then the batched solves; FP64: every matrix's
    normwise backward error <= 1e-14 after one solve; FP32 (split-TF32 products) + FP64 IR:
    every matrix converged to <= 1e-13.  Eight matrices of different sizes are re-checked
    on the host against LAPACK."""
    import torch
    from mustard_b200 import batch_bench
    sizes, nrhs, groups, rhs = batch_bench.make_batch(4096, 7)
    count = len(sizes)
    a64 = batch_bench.views(groups, count)
    p, dt = batch_bench.PRECS[prec]
    work_groups = {n: (idx, a.to(dt).clone()) for n, (idx, a) in groups.items()}
    work = batch_bench.views(work_groups, count)
    b = mtd.Batch(sizes, prec=p)
    b.factor(work)
    rc, info, _ = b.status(latencies=True)
    assert rc == 0 and all(v == 0 for v in info)
    xs = [torch.zeros_like(r) for r in rhs]
    if prec == "fp64":
        st = b.solve(work, rhs, xs, a64=a64, method=mtd.REFINE_NONE)
        bound = 1e-14
    else:
        st = b.solve(work, rhs, xs, a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=20)
        bound = 1e-13
    torch.cuda.synchronize()
    assert st["converged_count"] == count and st["max_backward_error"] <= bound, st
    picked = {}
    for i, n in enumerate(sizes):
        if n not in picked and len(picked) < 8:
            picked[n] = i
    for n, i in picked.items():
        a = _host(a64[i])
        x = _host(xs[i])
        bb = _host(rhs[i])
        assert mixed.backward_error(a, x, bb) <= 2 * bound, (i, n)
        assert mixed.forward_error(x, mixed.solve_fp64(a, bb)) <= 1e-11, (i, n)
    b.close()


def test_config4_adjoint_64x2048_against_torch_and_finite_differences(mtd):
    """64 RBF-kernel matrices of N = 2048 (K + 0.1 I over X in R^{2048 x 8}), GP loss
    0.5 y^T A^-1 y + sum(log diag L): the blocked adjoint's gradient (store and recompute)
    within 1e-10 of torch.linalg.cholesky's, and central finite differences (step 1e-6) of
    the loss of one matrix at a few entries."""
    import torch
    from mustard_b200 import adjoint_bench, autograd
    a, y = adjoint_bench.rbf_batch(64, 2048, 8, 5, torch.float64)
    grads = {}
    for name, chol in (("store", lambda x: autograd.cholesky(x, tile=256)),
                       ("recompute", lambda x: autograd.cholesky(x, tile=256, recompute=True)),
                       ("torch", torch.linalg.cholesky)):
        x = a.detach().clone().requires_grad_(True)
        adjoint_bench.gp_loss(chol(x), y).backward()
        grads[name] = x.grad.detach()
        del x
    ref = grads["torch"]
    scale = ref.abs().max().item()
    for name in ("store", "recompute"):
        assert (grads[name] - ref).abs().max().item() <= 1e-10 * scale, name
    assert torch.equal(grads["store"], grads["recompute"])  # the same factor bits, the same sweep
    # finite differences on matrix 0 (host FP64)
    a0 = a[0].cpu().numpy()
    y0 = y[0].cpu().numpy()
    g0 = grads["store"][0].cpu().numpy()

    def loss(m):
        L = np.linalg.cholesky(m)
        z = np.linalg.solve(L, y0)
        return 0.5 * z @ z + np.log(np.diag(L)).sum()

    h = 1e-6
    for i, j in [(0, 0), (1000, 1000), (17, 3), (2047, 1024)]:
        e = np.zeros_like(a0)
        e[i, j] = e[j, i] = 1.0
        fd = (loss(a0 + h * e) - loss(a0 - h * e)) / (2 * h)
        want = g0[i, j] if i == j else 2.0 * g0[i, j]
        assert abs(fd - want) <= 1e-5 * max(1.0, abs(fd)), (i, j, fd, want)


def test_config2_kappa_1e8_outcome_reported_honestly(mtd):
    """Condition number 1e8 (kappa u_FP32 ~ 6): the FP32-accurate factor of A + shift I
    (shift of a few FP32 roundoffs times max |a_ii|) preconditions FP64 GMRES-IR.  Whatever
    the outcome, the backward error the solver reports is the one the host computes from
    the returned x, and a reported convergence means <= 1e-13."""
    from tests.gpu_util import to_dev
    import torch
    n, tile = 2048, 512
    a = mixed.spd_kappa(n, 1e8, 31)
    b = mixed.rhs(n, 1, 32)
    s = mtd.SpdSolver(n, tile, mtd.PREC_FP32)
    assert s.factor(to_dev(a), shift=4 * 2.0 ** -21 * np.abs(np.diag(a)).max()) == 0
    xd = torch.zeros((1, n), dtype=torch.float64, device="cuda").t()
    bd = torch.from_numpy(np.ascontiguousarray(b.T)).cuda().t()
    st = s.solve(bd, xd, method=mtd.REFINE_GMRES_IR, tol=1e-13, max_iter=20)
    x = _host(xd)
    host_berr = mixed.backward_error(a, x, b)
    assert host_berr <= 2 * st["backward_error"] + 1e-16 and st["backward_error"] <= 2 * host_berr + 1e-16, \
        (st, host_berr)
    if st["converged"]:
        assert st["backward_error"] <= 1e-13 and host_berr <= 2e-13
        assert mixed.forward_error(x, mixed.solve_fp64(a, b)) <= 1e8 * 1e-11
    s.close()
