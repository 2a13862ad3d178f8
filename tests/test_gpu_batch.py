"""Batched Cholesky (no reference counterpart): many SPD matrices of sizes drawn from
{32, 64, ..., 1024}, built as in the reference's N=600 case (B B^T / n + I), factored as ONE
merged task graph in one persistent launch, then solved.  Checked per matrix against the
oracle (FP64 factors within 1e-12 relative; solves against LAPACK)."""
import numpy as np
import pytest

from oracle import gen, mixed, tiled
from tests.gpu_util import from_dev, rel_diff, to_dev

pytestmark = pytest.mark.gpu


def _sizes(count, seed):
    return [int(32 * v) for v in np.random.default_rng(seed).integers(1, 33, size=count)]


def _dev_rect(x, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(x).T))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda().t()


def _host(t):
    return np.asfortranarray(t.t().contiguous().cpu().double().numpy().T)


def test_batched_fp64_factor_and_solve(mtd):
    import torch
    sizes = _sizes(48, 1)
    mats = [gen.spd_input(n, 100 + i) for i, n in enumerate(sizes)]
    b = mtd.Batch(sizes, prec=mtd.PREC_FP64)
    dev = [to_dev(a) for a in mats]
    b.factor(dev)
    rc, info, lat = b.status(latencies=True)
    assert rc == 0 and all(v == 0 for v in info)
    assert all(x > 0 for x in lat)
    for i, (a, d) in enumerate(zip(mats, dev)):
        n = sizes[i]
        tile = n if n <= 512 else 512
        ref = a.copy(order="F")
        assert tiled.tiled_factor(ref, tile, "chol") == 0
        assert rel_diff(np.tril(from_dev(d)), np.tril(ref)) <= 1e-12, (i, n)
    nrhs = [1 + (i % 16) for i in range(len(sizes))]
    bs = [mixed.rhs(n, k, 7 + i) for i, (n, k) in enumerate(zip(sizes, nrhs))]
    bd = [_dev_rect(x) for x in bs]
    xd = [_dev_rect(np.zeros_like(x)) for x in bs]
    a64 = [to_dev(a) for a in mats]
    st = b.solve(dev, bd, xd, a64=a64, method=mtd.REFINE_NONE)
    torch.cuda.synchronize()
    assert st["max_backward_error"] <= 1e-14 and st["converged_count"] == len(sizes)
    for a, x, bb in zip(mats, xd, bs):
        assert mixed.forward_error(_host(x), mixed.solve_fp64(a, bb)) <= 1e-12
    b.close()


@pytest.mark.parametrize("prec", ["tf32", "fp32"])
def test_batched_low_precision_with_ir(mtd, prec):
    import torch
    p = mtd.PREC_TF32 if prec == "tf32" else mtd.PREC_FP32
    sizes = _sizes(40, 2)
    mats = [gen.spd_input(n, 300 + i) for i, n in enumerate(sizes)]
    b = mtd.Batch(sizes, prec=p)
    a64 = [to_dev(a) for a in mats]
    f32 = [torch.empty((n, n), dtype=torch.float32, device="cuda").t() for n in sizes]
    b.convert(a64, f32)
    b.factor(f32)
    rc, info = b.status()
    assert rc == 0 and all(v == 0 for v in info)
    bs = [mixed.rhs(n, 4, 11 + i) for i, n in enumerate(sizes)]
    bd = [_dev_rect(x) for x in bs]
    xd = [_dev_rect(np.zeros_like(x)) for x in bs]
    st = b.solve(f32, bd, xd, a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=20)
    torch.cuda.synchronize()
    assert st["converged_count"] == len(sizes) and st["max_backward_error"] <= 1e-13, st
    assert st["iterations"] >= 2
    for a, x, bb in zip(mats, xd, bs):
        assert mixed.backward_error(a, _host(x), bb) <= 2e-13
    b.close()


def test_batched_bad_pivot_is_per_matrix(mtd):
    sizes = [96, 300, 160, 64]
    mats = [gen.spd_input(n, 50 + i) for i, n in enumerate(sizes)]
    mats[1][200, 200] = -3.0  # matrix 1: leading minor of order 201 is not positive definite
    b = mtd.Batch(sizes, prec=mtd.PREC_FP64)
    dev = [to_dev(a) for a in mats]
    b.factor(dev)
    rc, info = b.status()
    assert rc == 0
    assert info[0] == 0 and info[2] == 0 and info[3] == 0
    assert info[1] == 201
    for i in (0, 2, 3):
        assert rel_diff(np.tril(from_dev(dev[i])), np.tril(tiled.cholesky_lapack(mats[i]))) <= 1e-12
    b.close()


def test_batched_factor_captured_in_a_cuda_graph(mtd):
    import torch
    sizes = _sizes(24, 3)
    mats = [gen.spd_input(n, 700 + i) for i, n in enumerate(sizes)]
    b = mtd.Batch(sizes, prec=mtd.PREC_FP64)
    src = [to_dev(a) for a in mats]
    work = [s.clone() for s in src]
    b.factor(work)  # warm-up outside the capture (per-device set-up)
    b.status()
    for w, s_ in zip(work, src):
        w.copy_(s_)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            b.factor(work, stream=s)
    for _ in range(2):
        for w, s_ in zip(work, src):
            w.copy_(s_)
        g.replay()
        torch.cuda.synchronize()
        rc, info = b.status()
        assert rc == 0 and all(v == 0 for v in info)
        for i, a in enumerate(mats):
            assert rel_diff(np.tril(from_dev(work[i])), np.tril(tiled.cholesky_lapack(a))) <= 1e-12
    del g
    b.close()


def test_autotune_choices_factor_correctly_and_persist(mtd, tmp_path):
    # the autotuner's per-size choices are valid tile / nested-tile edges for each size, a
    # batch built with them factors correctly, and a JSON table makes a second tune of the
    # same sizes free while a new size is tuned and added
    import json
    sizes = [96, 96, 300, 300, 520]
    table = str(tmp_path / "tune.json")
    tiles, nests, ms = mtd.batch_autotune(sizes, mtd.PREC_FP64, table=table)
    assert ms > 0
    for n, t, k in zip(sizes, tiles, nests):
        assert 1 <= t <= n and (k == 0 or (k % 64 == 0 and k < t))
    assert tiles[0] == tiles[1] and tiles[2] == tiles[3]  # one choice per size
    mats = [gen.spd_input(n, 900 + i) for i, n in enumerate(sizes)]
    b = mtd.Batch(sizes, tiles=tiles, nests=nests, prec=mtd.PREC_FP64)
    work = [to_dev(a) for a in mats]
    b.factor(work)
    rc, info = b.status()
    assert rc == 0 and all(v == 0 for v in info)
    for i, a in enumerate(mats):
        assert rel_diff(np.tril(from_dev(work[i])), np.tril(tiled.cholesky_lapack(a))) <= 1e-12
    b.close()
    t2, k2, ms2 = mtd.batch_autotune(sizes, mtd.PREC_FP64, table=table)
    assert (t2, k2, ms2) == (tiles, nests, 0.0)
    t3, k3, ms3 = mtd.batch_autotune(sizes + [160], mtd.PREC_FP64, table=table)
    assert ms3 > 0 and t3[:5] == tiles and k3[:5] == nests
    dev = json.load(open(table))["devices"]
    assert sorted(int(n) for n in next(iter(dev.values()))["fp64"]) == [96, 160, 300, 520]
