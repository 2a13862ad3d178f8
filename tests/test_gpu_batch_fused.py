"""Batched factor AND solve in one persistent launch (mtd_batch_factor_solve): per matrix a
solve task after its factorisation (and, for low-precision batches, a conversion task
before it) in the merged task graph.  The solve tasks run the same per-matrix arithmetic as
the standalone solve launches (mtd_batch_solve), so the two paths must agree bit for bit;
every CTA-to-task schedule must give the same bits too.  Checked against LAPACK on the
host."""
import numpy as np
import pytest

from oracle import gen, mixed, tiled
from tests.gpu_util import from_dev, rel_diff, to_dev

pytestmark = pytest.mark.gpu


def _sizes(count, seed):
    return [int(32 * v) for v in np.random.default_rng(seed).integers(1, 33, size=count)]


def _dev_rect(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x).T)).cuda().t()


def _host(t):
    return np.asfortranarray(t.t().contiguous().cpu().double().numpy().T)


def _problem(sizes, seed):
    mats = [gen.spd_input(n, seed + i) for i, n in enumerate(sizes)]
    nrhs = [1 + (i % 16) for i in range(len(sizes))]
    bs = [mixed.rhs(n, k, seed + 1000 + i) for i, (n, k) in enumerate(zip(sizes, nrhs))]
    return mats, bs


def _fresh(mats, bs, dtype=None):
    import torch
    a64 = [to_dev(a) for a in mats]
    work = [to_dev(a) if dtype is None else torch.empty((a.shape[0],) * 2, dtype=dtype, device="cuda").t()
            for a in mats]
    bd = [_dev_rect(x) for x in bs]
    xd = [_dev_rect(np.zeros_like(x)) for x in bs]
    return a64, work, bd, xd


def test_fp64_factor_solve_matches_split_launches_bitwise(mtd):
    import torch
    sizes = _sizes(40, 11)
    mats, bs = _problem(sizes, 1100)
    b = mtd.Batch(sizes, prec=mtd.PREC_FP64)
    # split: factor launch, then the solve launches
    a64, work, bd, xd = _fresh(mats, bs)
    b.factor(work)
    rc, info = b.status()
    assert rc == 0 and not any(info)
    st = b.solve(work, bd, xd, a64=a64, method=mtd.REFINE_NONE)
    torch.cuda.synchronize()
    x_split = [_host(x) for x in xd]
    f_split = [from_dev(w) for w in work]
    # fused: one launch
    a64, work, bd, xd = _fresh(mats, bs)
    b.factor_solve(work, bd, xd, a64=a64, method=mtd.REFINE_NONE)
    rc, info, lat, berr, its, fst = b.solve_status()
    assert rc == 0 and not any(info)
    assert all(v > 0 for v in lat) and all(i == 1 for i in its)
    assert fst["converged_count"] == len(sizes) and fst["max_backward_error"] <= 1e-14, fst
    assert abs(fst["max_backward_error"] - st["max_backward_error"]) == 0.0
    for i, a in enumerate(mats):
        assert np.array_equal(np.tril(from_dev(work[i])), np.tril(f_split[i])), i
        assert np.array_equal(_host(xd[i]), x_split[i]), i
        assert mixed.forward_error(_host(xd[i]), mixed.solve_fp64(a, bs[i])) <= 1e-12
    b.close()


def test_fp64_factor_solve_without_matrix_and_with_refinement(mtd):
    sizes = [64, 320, 1024, 96, 700]
    mats, bs = _problem(sizes, 1300)
    b = mtd.Batch(sizes, prec=mtd.PREC_FP64)
    # no FP64 copy: one solve, no residual (backward error -1)
    a64, work, bd, xd = _fresh(mats, bs)
    b.factor_solve(work, bd, xd)
    rc, info, lat, berr, its, st = b.solve_status()
    assert rc == 0 and berr == [-1.0] * len(sizes) and its == [1] * len(sizes)
    for i, a in enumerate(mats):
        assert mixed.forward_error(_host(xd[i]), mixed.solve_fp64(a, bs[i])) <= 1e-12
    # FP64 refinement: converged after the first residual (<= tol) or one more step
    a64, work, bd, xd = _fresh(mats, bs)
    b.factor_solve(work, bd, xd, a64=a64, method=mtd.REFINE_IR, tol=1e-15, max_iter=3)
    rc, info, lat, berr, its, st = b.solve_status()
    assert rc == 0 and all(0 <= e <= 1e-15 for e in berr) and all(1 <= i <= 4 for i in its)
    for i, a in enumerate(mats):
        assert mixed.backward_error(a, _host(xd[i]), bs[i]) <= 2e-15
    b.close()


@pytest.mark.parametrize("prec", ["tf32", "fp32"])
def test_low_precision_factor_solve_matches_split_launches_bitwise(mtd, prec):
    import torch
    p = mtd.PREC_TF32 if prec == "tf32" else mtd.PREC_FP32
    sizes = _sizes(36, 12)
    mats, bs = _problem(sizes, 1200)
    b = mtd.Batch(sizes, prec=p)
    a64, f32, bd, xd = _fresh(mats, bs, torch.float32)
    b.convert(a64, f32, shift=0.0)
    b.factor(f32)
    rc, info = b.status()
    assert rc == 0 and not any(info)
    st = b.solve(f32, bd, xd, a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=20)
    torch.cuda.synchronize()
    x_split = [_host(x) for x in xd]
    f_split = [from_dev(f) for f in f32]
    a64, f32, bd, xd = _fresh(mats, bs, torch.float32)  # f32 uninitialised: the launch converts
    b.factor_solve(f32, bd, xd, a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=20)
    rc, info, lat, berr, its, fst = b.solve_status()
    assert rc == 0 and not any(info)
    assert fst["converged_count"] == len(sizes) and fst["max_backward_error"] <= 1e-13, fst
    assert fst["iterations"] == st["iterations"]
    for i, a in enumerate(mats):
        assert np.array_equal(np.tril(from_dev(f32[i])), np.tril(f_split[i])), i
        assert np.array_equal(_host(xd[i]), x_split[i]), i
        assert mixed.backward_error(a, _host(xd[i]), bs[i]) <= 2e-13
    b.close()


def test_every_schedule_gives_the_same_bits(mtd):
    import torch
    sizes = _sizes(30, 13)
    mats, bs = _problem(sizes, 1400)
    b = mtd.Batch(sizes, prec=mtd.PREC_FP32)
    outs = []
    for sched in range(16):
        if (sched & 3) == 3:
            continue
        b.schedule = sched
        assert b.schedule == sched
        a64, f32, bd, xd = _fresh(mats, bs, torch.float32)
        b.factor_solve(f32, bd, xd, a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=20)
        rc, info, lat, berr, its, st = b.solve_status()
        assert rc == 0 and st["converged_count"] == len(sizes), (sched, st)
        outs.append([_host(x) for x in xd])
    for o in outs[1:]:
        assert all(np.array_equal(x, y) for x, y in zip(o, outs[0]))
    with pytest.raises(mtd.MtdError):
        b.schedule = 3
    b.close()


def test_bad_pivot_skips_only_that_matrix(mtd):
    sizes = [96, 300, 160, 64]
    mats, bs = _problem(sizes, 1500)
    mats[1][200, 200] = -3.0  # the leading minor of order 201 is not positive definite
    b = mtd.Batch(sizes, prec=mtd.PREC_FP64)
    a64, work, bd, xd = _fresh(mats, bs)
    b.factor_solve(work, bd, xd, a64=a64, method=mtd.REFINE_NONE)
    rc, info, lat, berr, its, st = b.solve_status()
    assert rc == 0 and info == [0, 201, 0, 0]
    assert np.isnan(berr[1]) and its[1] == 0
    assert st["converged_count"] == 3
    for i in (0, 2, 3):
        assert berr[i] <= 1e-14
        assert rel_diff(np.tril(from_dev(work[i])), np.tril(tiled.cholesky_lapack(mats[i]))) <= 1e-12
        assert mixed.forward_error(_host(xd[i]), mixed.solve_fp64(mats[i], bs[i])) <= 1e-12
    b.close()


def test_factor_solve_captured_in_a_cuda_graph(mtd):
    import torch
    sizes = _sizes(20, 14)
    mats, bs = _problem(sizes, 1600)
    b = mtd.Batch(sizes, prec=mtd.PREC_FP32)
    a64, f32, bd, xd = _fresh(mats, bs, torch.float32)
    b.factor_solve(f32, bd, xd, a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=20)  # set-up outside
    rc, *_ = b.solve_status()
    assert rc == 0
    want = [_host(x) for x in xd]
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            b.factor_solve(f32, bd, xd, a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=20, stream=s)
    for _ in range(2):
        for x in xd:
            x.zero_()
        g.replay()
        torch.cuda.synchronize()
        rc, info, lat, berr, its, st = b.solve_status()
        assert rc == 0 and st["converged_count"] == len(sizes)
        assert all(np.array_equal(_host(x), w) for x, w in zip(xd, want))
    del g
    b.close()


def test_schedule_tuner_keeps_a_valid_fastest_schedule(mtd):
    sizes = _sizes(64, 15)
    mats, bs = _problem(sizes, 1700)
    b = mtd.Batch(sizes, prec=mtd.PREC_FP64)
    a64, work, bd, xd = _fresh(mats, bs)
    src = [to_dev(a) for a in mats]
    best, ms = b.tune_schedule(work, bd, xd, a64=a64, source=src, method=mtd.REFINE_NONE, reps=1)
    assert sorted(ms) == [0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14] and all(v > 0 for v in ms.values())
    assert best in ms and ms[best] == min(ms.values()) and b.schedule == best
    # the tuned batch still solves correctly from a restored input
    for w, s_ in zip(work, src):
        w.copy_(s_)
    b.factor_solve(work, bd, xd, a64=a64, method=mtd.REFINE_NONE)
    rc, info, lat, berr, its, st = b.solve_status()
    assert rc == 0 and st["converged_count"] == len(sizes)
    b.close()
