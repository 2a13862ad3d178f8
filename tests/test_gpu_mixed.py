"""Mixed-precision solver (no reference counterpart): TF32 tiled Cholesky on the task
scheduler plus FP64 iterative refinement / GMRES-IR, against an FP64 LAPACK oracle.
Bars: backward error <= 1e-13 (normwise, infinity norms, FP64) when converged; forward
error within cond(A) * 1e-13 of the FP64 oracle's solution."""
import numpy as np
import pytest

from oracle import gen, mixed, tiled
from tests.gpu_util import from_dev, rel_diff, to_dev

pytestmark = pytest.mark.gpu


def _dev_rect(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x).T)).cuda().t()


def _host_rect(t):
    return np.asfortranarray(t.t().contiguous().cpu().numpy().T)


def test_tf32_factor_close_to_fp64(mtd):
    import torch
    n, tile = 1536, 512
    a = gen.spd_input(n, 3)
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY, n, tile).build_tiled().set_precision(mtd.PREC_TF32).finalize()
    d = torch.from_numpy(np.ascontiguousarray(a.T).astype(np.float32)).cuda().t()
    assert g.run_f32(d) == 0
    l32 = np.tril(np.asfortranarray(d.t().contiguous().cpu().numpy().T).astype(np.float64))
    ref = np.tril(tiled.cholesky_lapack(a))
    err = rel_diff(l32, ref)
    assert 1e-7 < err < 5e-3  # TF32 products (unit roundoff 2^-11), FP32 accumulation
    # FP64 graphs refuse float runs and the other way round
    with pytest.raises(mtd.MtdError):
        g.run(to_dev(a))
    g.close()


@pytest.mark.parametrize("nrhs", [1, 16])
def test_ir_reaches_fp64_accuracy_kappa_1e2(mtd, nrhs):
    n, tile = 2048, 512
    a = mixed.spd_kappa(n, 1e2, 5)
    b = mixed.rhs(n, nrhs, 6)
    s = mtd.SpdSolver(n, tile, mtd.PREC_TF32)
    assert s.factor(to_dev(a)) == 0
    xd = _dev_rect(np.zeros((n, nrhs)))
    st = s.solve(_dev_rect(b), xd, method=mtd.REFINE_IR, tol=1e-13, max_iter=40)
    x = _host_rect(xd)
    assert st["converged"] and st["backward_error"] <= 1e-13
    assert 1 < st["iterations"] <= 40
    assert mixed.backward_error(a, x, b) <= 2e-13  # recomputed on the host in FP64
    assert mixed.forward_error(x, mixed.solve_fp64(a, b)) <= 1e2 * 1e-12
    s.close()


@pytest.mark.parametrize("prec,n,nrhs", [("fp64", 1000, 3), ("tf32", 1000, 1), ("fp32", 1217, 7)])
def test_ragged_sizes_and_rhs_groups(mtd, prec, n, nrhs):
    """n not a multiple of the 64-row solve blocks (partial last block in the triangular
    solves and the symmetric residual product) and right-hand-side counts in each group."""
    p = {"fp64": mtd.PREC_FP64, "tf32": mtd.PREC_TF32, "fp32": mtd.PREC_FP32}[prec]
    a = mixed.spd_kappa(n, 1e2, 21)
    b = mixed.rhs(n, nrhs, 22)
    s = mtd.SpdSolver(n, 256, p)
    assert s.factor(to_dev(a)) == 0
    xd = _dev_rect(np.zeros((n, nrhs)))
    method = mtd.REFINE_NONE if prec == "fp64" else mtd.REFINE_IR
    st = s.solve(_dev_rect(b), xd, method=method, tol=1e-13, max_iter=40)
    x = _host_rect(xd)
    bound = 1e-14 if prec == "fp64" else 1e-13
    assert st["backward_error"] <= bound, st
    assert mixed.backward_error(a, x, b) <= 2 * bound
    assert mixed.forward_error(x, mixed.solve_fp64(a, b)) <= 1e2 * 1e-12
    # factoring again reuses the buffers (whose upper triangle the solves use): same answer
    # (to rounding: the FP64 residual sums with atomics, so its last bits vary run to run)
    assert s.factor(to_dev(a)) == 0
    xd2 = _dev_rect(np.zeros((n, nrhs)))
    st2 = s.solve(_dev_rect(b), xd2, method=method, tol=1e-13, max_iter=40)
    assert abs(st2["iterations"] - st["iterations"]) <= 1 and st2["backward_error"] <= bound
    assert mixed.forward_error(_host_rect(xd2), x) <= 1e-12
    s.close()


def test_fp64_solver_one_solve(mtd):
    n, tile = 2048, 512
    a = mixed.spd_kappa(n, 1e2, 8)
    b = mixed.rhs(n, 4, 9)
    s = mtd.SpdSolver(n, tile, mtd.PREC_FP64)
    assert s.factor(to_dev(a)) == 0
    xd = _dev_rect(np.zeros((n, 4)))
    st = s.solve(_dev_rect(b), xd, method=mtd.REFINE_NONE, tol=1e-13)
    x = _host_rect(xd)
    assert st["backward_error"] <= 1e-14
    assert mixed.forward_error(x, mixed.solve_fp64(a, b)) <= 1e-12
    s.close()


def test_gmres_ir_kappa_1e5(mtd):
    n, tile = 2048, 512
    a = mixed.spd_kappa(n, 1e5, 10)
    b = mixed.rhs(n, 1, 11)
    s = mtd.SpdSolver(n, tile, mtd.PREC_TF32)
    # kappa * u_TF32 ~ 50: the unshifted TF32 factor may meet a non-positive pivot (which
    # rounding decides); it is then reported with its column, and a shift of a few TF32
    # roundoffs times ||A|| keeps the factor positive definite as a GMRES preconditioner
    try:
        s.factor(to_dev(a))
    except mtd.MtdError as e:
        assert e.status == 5 and 1 <= e.info <= n
        assert s.factor(to_dev(a), shift=4 * 2.0 ** -11 * np.abs(a).sum(axis=1).max()) == 0
    xd = _dev_rect(np.zeros((n, 1)))
    st = s.solve(_dev_rect(b), xd, method=mtd.REFINE_GMRES_IR, tol=1e-13, max_iter=20)
    x = _host_rect(xd)
    assert st["converged"] and st["backward_error"] <= 1e-13, st
    assert mixed.backward_error(a, x, b) <= 2e-13
    assert mixed.forward_error(x, mixed.solve_fp64(a, b)) <= 1e5 * 1e-12
    s.close()


def test_plain_ir_reports_non_convergence_honestly(mtd):
    # kappa 1e5 with a TF32 factor: kappa * u_TF32 >> 1, plain IR cannot converge; the
    # solver must say so rather than claim the tolerance.  The unshifted TF32
    # factorisation may break down (non-positive pivot, reported with its column); a
    # diagonal shift of a few TF32 roundoffs times ||A|| keeps it positive definite.
    n, tile = 1024, 512
    a = mixed.spd_kappa(n, 1e5, 12)
    b = mixed.rhs(n, 1, 13)
    s = mtd.SpdSolver(n, tile, mtd.PREC_TF32)
    try:
        s.factor(to_dev(a))
    except mtd.MtdError as e:
        assert e.status == 5 and 1 <= e.info <= n
    shift = 4 * 2.0 ** -11 * np.abs(a).sum(axis=1).max()
    assert s.factor(to_dev(a), shift=shift) == 0
    xd = _dev_rect(np.zeros((n, 1)))
    st = s.solve(_dev_rect(b), xd, method=mtd.REFINE_IR, tol=1e-13, max_iter=8)
    x = _host_rect(xd)
    assert st["converged"] == (st["backward_error"] <= 1e-13)
    assert abs(mixed.backward_error(a, x, b) - st["backward_error"]) <= 0.05 * st["backward_error"] + 1e-15
    s.close()


def test_solver_argument_checks(mtd):
    with pytest.raises(mtd.MtdError):
        mtd.SpdSolver(1000, 100, mtd.PREC_TF32)  # tile must be a multiple of 64
    s = mtd.SpdSolver(512, 128, mtd.PREC_TF32)
    xd = _dev_rect(np.zeros((512, 1)))
    with pytest.raises(mtd.MtdError) as e:
        s.solve(xd, xd)  # not factored yet
    assert e.value.status == 2
    s.close()


def _low_factor(mtd, a, tile, prec):
    import torch
    n = a.shape[0]
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY, n, tile).build_tiled().set_precision(prec).finalize()
    d = torch.from_numpy(np.ascontiguousarray(a.T).astype(np.float32)).cuda().t()
    assert g.run_f32(d) == 0
    g.close()
    return np.tril(np.asfortranarray(d.t().contiguous().cpu().numpy().T).astype(np.float64))


@pytest.mark.parametrize("n,tile,ratio", [(2048, 512, 2.0), (1024, 320, 1.0)])
def test_bf16_update_factor_accuracy(mtd, n, tile, ratio):
    # GEMM / SYRK updates with BF16 operands (tcgen05 kind::f16 from the BF16 copy of the
    # panels): at tile 512 every update is a BF16 one and the factor is accurate to about
    # BF16 roundoff, clearly coarser than the TF32 factor (7 against 10 mantissa bits); at
    # tile 320 the 320-deep outer updates (most of the work) take the TF32 path and only the
    # nested 128-deep ones the BF16 path.  Either way far from a wrong factor.
    a = mixed.spd_kappa(n, 1e2, 31)
    err = {}
    for prec in (mtd.PREC_TF32, mtd.PREC_BF16):
        l = _low_factor(mtd, a, tile, prec)
        err[prec] = np.linalg.norm(l @ l.T - a) / np.linalg.norm(a)
    assert err[mtd.PREC_TF32] < 2e-3
    assert ratio * err[mtd.PREC_TF32] < err[mtd.PREC_BF16] < 2e-2, err


@pytest.mark.parametrize("method", ["ir", "gmres-ir"])
def test_bf16_factor_refines_to_fp64_accuracy(mtd, method):
    n, tile = 2048, 512
    a = mixed.spd_kappa(n, 1e2, 32)
    k = 2 if method == "ir" else 1  # GMRES-IR solves one right-hand side at a time
    b = mixed.rhs(n, k, 33)
    m = mtd.REFINE_IR if method == "ir" else mtd.REFINE_GMRES_IR
    s = mtd.SpdSolver(n, tile, mtd.PREC_BF16)
    assert s.factor(to_dev(a)) == 0
    xd = _dev_rect(np.zeros((n, k)))
    st = s.solve(_dev_rect(b), xd, method=m, tol=1e-13, max_iter=60)
    x = _host_rect(xd)
    assert st["converged"] and st["backward_error"] <= 1e-13, st
    assert mixed.backward_error(a, x, b) <= 2e-13
    assert mixed.forward_error(x, mixed.solve_fp64(a, b)) <= 1e2 * 1e-12
    s.close()


@pytest.mark.parametrize("n,tile,nest", [(1536, 512, 128), (2048, 384, 64), (1024, 256, 128)])
def test_fp32_three_pass_factor_accuracy(mtd, n, tile, nest):
    """MTD_PREC_FP32 with n, the tile and the nested sub-tile multiples of 32: the GEMM / SYRK
    items run three TF32 passes on tcgen05 (panel x panel + panel x low part + low part x
    panel, the low parts written by the TRSM items); the factor is FP32-accurate, more than an
    order of magnitude closer to LAPACK's FP64 factor than the single-pass TF32 one (4.4e-7
    against 2.5e-5 at n = 1536 on a B200)."""
    import torch
    a = gen.spd_input(n, 3)
    ref = np.tril(tiled.cholesky_lapack(a))
    errs = {}
    for prec in (mtd.PREC_TF32, mtd.PREC_FP32):
        g = mtd.TaskGraph(mtd.KIND_CHOLESKY, n, tile).build_tiled().set_precision(prec)
        g.set_nest(nest).finalize()
        d = torch.from_numpy(np.ascontiguousarray(a.T).astype(np.float32)).cuda().t()
        assert g.run_f32(d) == 0
        l32 = np.tril(np.asfortranarray(d.t().contiguous().cpu().numpy().T).astype(np.float64))
        errs[prec] = rel_diff(l32, ref)
        # a second run on the same graph (barrier parities and the low copy reused)
        d = torch.from_numpy(np.ascontiguousarray(a.T).astype(np.float32)).cuda().t()
        assert g.run_f32(d) == 0
        assert rel_diff(np.tril(np.asfortranarray(d.t().contiguous().cpu().numpy().T).astype(np.float64)), ref) \
            == errs[prec]
        g.close()
    assert errs[mtd.PREC_FP32] < 3e-6, errs
    assert errs[mtd.PREC_FP32] * 20 < errs[mtd.PREC_TF32], errs


def test_fp32_three_pass_ir_kappa_1e5(mtd):
    """kappa = 1e5 (kappa u_TF32 ~ 50: a single-pass TF32 factor is at the edge of breaking
    down): the FP32-accurate factor refines by plain IR to FP64 backward error."""
    n, tile = 2048, 512
    a = mixed.spd_kappa(n, 1e5, 10)
    b = mixed.rhs(n, 1, 11)
    s = mtd.SpdSolver(n, tile, mtd.PREC_FP32)
    assert s.factor(to_dev(a)) == 0
    xd = _dev_rect(np.zeros((n, 1)))
    st = s.solve(_dev_rect(b), xd, method=mtd.REFINE_IR, tol=1e-13, max_iter=30)
    x = _host_rect(xd)
    assert st["converged"] and st["backward_error"] <= 1e-13, st
    assert st["iterations"] <= 20, st
    assert mixed.backward_error(a, x, b) <= 2e-13
    assert mixed.forward_error(x, mixed.solve_fp64(a, b)) <= 1e5 * 1e-12
    s.close()
