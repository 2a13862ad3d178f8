"""Whole tiled factorisations on the GPU against the oracle (the reference's task list
run sequentially with LAPACK/BLAS tiles), the reference's --verify criterion, and
LAPACK.  FP64 parity bar: max |diff| / max |oracle| <= 1e-12."""
import numpy as np
import pytest

from oracle import gen, tiled, verify
from tests.gpu_util import from_dev, rel_diff, to_dev

pytestmark = pytest.mark.gpu
TOL = 1e-12


def factor(mtd, a, tile, kind, trace=False):
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU, a.shape[0], tile).build_tiled()
    if trace:
        g.set_trace(True)
    g.finalize()
    d = to_dev(a)
    info = g.run(d)
    return from_dev(d), info, g


def oracle_factor(a, tile, kind):
    f = a.copy(order="F")
    assert tiled.tiled_factor(f, tile, kind) == 0
    return f


@pytest.mark.parametrize("kind", ["chol", "lu"])
def test_reference_config_n600_t2(mtd, kind):
    # cholesky_mustard / lu_mustard -n=600 -t=2 --subgraph --verify (README.md:168-169)
    a = gen.ref_spd(600)
    out, info, g = factor(mtd, a, 300, kind)
    assert info == 0
    ref = oracle_factor(a, 300, kind)
    if kind == "chol":
        assert rel_diff(np.tril(out), np.tril(ref)) <= TOL
        assert np.array_equal(np.triu(out, 1), np.triu(a, 1))
        err = verify.ref_error_chol(a, out)
    else:
        assert rel_diff(out, ref) <= TOL
        err = verify.ref_error_lu(a, out)
    assert err <= verify.REF_TOLERANCE  # include/verify.h:69,127
    g.close()


@pytest.mark.parametrize("kind", ["chol", "lu"])
@pytest.mark.parametrize("n,tile", [(1000, 384), (1030, 512), (2048, 512), (15, 3), (301, 100), (640, 128), (257, 64)])
def test_tiled_parity(mtd, kind, n, tile):
    a = gen.spd_input(n, 5) if kind == "chol" else gen.lu_input(n, 5)
    out, info, g = factor(mtd, a, tile, kind)
    assert info == 0
    ref = oracle_factor(a, tile, kind)
    if kind == "chol":
        assert rel_diff(np.tril(out), np.tril(ref)) <= TOL
        assert np.array_equal(np.triu(out, 1), np.triu(a, 1))
        assert verify.normwise_residual_chol(a, out) < 1e-14
    else:
        assert rel_diff(out, ref) <= TOL
        assert verify.normwise_residual_lu(a, out) < 1e-14
    g.close()


@pytest.mark.parametrize("kind", ["chol", "lu"])
def test_repeat_runs_bitwise_identical(mtd, kind):
    a = gen.spd_input(1200, 9) if kind == "chol" else gen.lu_input(1200, 9)
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU, 1200, 256).build_tiled().finalize()
    outs = []
    for _ in range(3):
        d = to_dev(a)
        g.run(d)
        outs.append(from_dev(d))
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[1], outs[2])
    g.close()


def test_not_positive_definite_reports_info(mtd):
    n, tile = 600, 200
    a = gen.spd_input(n, 4)
    a[450, 450] = -1.0  # leading minor of order 451 is not positive definite
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY, n, tile).build_tiled().finalize()
    d = to_dev(a)
    with pytest.raises(mtd.MtdError) as e:
        g.run(d)
    assert e.value.status == 5
    assert e.value.info == 451
    # the context stays usable: a good matrix factors afterwards
    d = to_dev(gen.spd_input(n, 4))
    assert g.run(d) == 0
    g.close()


def test_zero_pivot_reports_info(mtd):
    n, tile = 300, 100
    a = np.asfortranarray(np.eye(n) * 2.0)
    a[130, 130] = 0.0
    g = mtd.TaskGraph(mtd.KIND_LU, n, tile).build_tiled().finalize()
    with pytest.raises(mtd.MtdError) as e:
        g.run(to_dev(a))
    assert e.value.status == 6 and e.value.info == 131
    g.close()


def test_bounded_wait_times_out_cleanly(mtd):
    # A deadline far shorter than one tile operation: waiting CTAs give up, record
    # MTD_ERR_TIMEOUT and return; nothing hangs and the next run succeeds.
    n, tile = 2048, 1024
    a = gen.spd_input(n, 8)
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY, n, tile).build_tiled().set_timeout(1e-6).finalize()
    with pytest.raises(mtd.MtdError) as e:
        g.run(to_dev(a))
    assert e.value.status == 4
    g.set_timeout(10.0)
    d = to_dev(a)
    assert g.run(d) == 0
    assert verify.normwise_residual_chol(a, from_dev(d)) < 1e-14
    g.close()


def test_one_call_drivers(mtd):
    a = gen.spd_input(700, 12)
    d = to_dev(a)
    assert mtd.tiled_cholesky(d, 256) == 0
    assert rel_diff(np.tril(from_dev(d)), np.tril(oracle_factor(a, 256, "chol"))) <= TOL
    b = gen.lu_input(700, 12)
    d = to_dev(b)
    assert mtd.tiled_lu(d, 256) == 0
    assert rel_diff(from_dev(d), oracle_factor(b, 256, "lu")) <= TOL


def test_trace_and_stats(mtd):
    a = gen.spd_input(1024, 1)
    out, info, g = factor(mtd, a, 256, "chol", trace=True)
    st = g.stats()
    total_items = sum(g.items(t) for t in range(g.num_tasks))
    assert st["tasks"] == g.num_device_tasks and st["items"] == total_items
    assert g.num_device_tasks > g.num_tasks  # the 256-wide diagonal tiles are nested (128)
    assert 0.0 < st["busy_fraction"] <= 1.0 and st["span_ms"] > 0
    recs = g.trace()
    assert len(recs) == total_items
    assert all(e >= s for s, e, _, _, _ in recs)
    g.close()


def test_device_generators_match_oracle(mtd):
    import torch
    n = 512
    d = torch.empty((n, n), dtype=torch.float64, device="cuda").t()
    mtd.generate(d, mtd.GEN_UNIFORM_DIAG, seed=21)
    assert np.array_equal(from_dev(d), gen.lu_input(n, 21))
    mtd.generate(d, mtd.GEN_SPD, seed=21, alpha=1.0)
    assert rel_diff(from_dev(d), gen.spd_input(n, 21)) <= 1e-14


def test_large_cholesky_against_lapack(mtd):
    from scipy.linalg import lapack
    n, tile = 6000, 1024
    a = gen.spd_input(n, 2)
    out, info, g = factor(mtd, a, tile, "chol")
    ref, rinfo = lapack.dpotrf(a, lower=1, clean=1)
    assert rinfo == 0
    assert rel_diff(np.tril(out), ref) <= TOL
    # backward stable as LAPACK is: the probe residual within 25 % of dpotrf's on the same
    # input (dpotrf itself gives 9.5e-16 here; the summation order differs from ours)
    assert verify.probe_residual(a, out, "chol") <= 1.25 * verify.probe_residual(a, ref, "chol")
    g.close()


def test_large_lu_against_lapack(mtd):
    n, tile = 6000, 768
    a = gen.lu_input(n, 2)
    out, info, g = factor(mtd, a, tile, "lu")
    ref = tiled.lu_nopiv_lapack(a)
    assert rel_diff(out, ref) <= TOL
    assert verify.probe_residual(a, out, "lu") < 1e-15
    g.close()


@pytest.mark.parametrize("kind", ["chol", "lu"])
@pytest.mark.parametrize("n,tma", [(1100, "0"), (1024, "1")])
def test_cuda_graph_executor_matches_scheduler(mtd, kind, n, tma, monkeypatch):
    # --tiled mode: the same tile kernels as one host-launched CUDA graph (its GEMM items are
    # always on the cp.async engine; at n = 1024 with MTD_TMA64=1 the scheduler's are TMA-fed).
    monkeypatch.setenv("MTD_TMA64", tma)
    tile = 256
    a = gen.spd_input(n, 6) if kind == "chol" else gen.lu_input(n, 6)
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU, n, tile).build_tiled().finalize()
    d1, d2 = to_dev(a), to_dev(a)
    g.run(d1)
    g.run_graph(d2)
    x, y = from_dev(d1), from_dev(d2)
    assert np.array_equal(x, y)  # same arithmetic per tile, same order per tile: bitwise equal
    d3 = to_dev(a)
    g.run_graph(d3)  # cached CUDA graph, second launch
    assert np.array_equal(from_dev(d3), y)
    g.close()


@pytest.mark.parametrize("kind", ["chol", "lu"])
@pytest.mark.parametrize("nest", [0, 64, 128, 256])
def test_nested_diagonal_factorisation(mtd, kind, nest):
    # POTRF / GETRF of a 640-wide tile lowered to a tiled sub-factorisation (or not: 0)
    n, tile = 1400, 640
    a = gen.spd_input(n, 13) if kind == "chol" else gen.lu_input(n, 13)
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU, n, tile).build_tiled()
    g.set_nest(nest).finalize()
    if nest:
        assert g.num_device_tasks > g.num_tasks
    d = to_dev(a)
    assert g.run(d) == 0
    ref = oracle_factor(a, tile, kind)
    out = from_dev(d)
    if kind == "chol":
        out, ref = np.tril(out), np.tril(ref)
    assert rel_diff(out, ref) <= TOL
    g.close()


@pytest.mark.parametrize("kind", ["chol", "lu"])
def test_uneven_tile_edges(mtd, kind):
    # a narrower first and last tile (mtd_graph_set_tile_edges), nested diagonal
    # factorisations inside the wide ones: the factors match LAPACK's as with uniform tiles
    n = 3000
    edges = [0, 256, 1024, 1792, 2560, 2816, 3000]
    a = gen.spd_input(n, 21) if kind == "chol" else gen.lu_input(n, 21)
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU, n, 768)
    g.set_tile_edges(edges).build_tiled().finalize()
    d = to_dev(a)
    assert g.run(d) == 0
    out = from_dev(d)
    if kind == "chol":
        assert rel_diff(np.tril(out), np.tril(tiled.cholesky_lapack(a))) <= TOL
    else:
        assert rel_diff(out, tiled.lu_nopiv_lapack(a)) <= TOL
    g.close()


def test_nest_edge_must_be_multiple_of_64(mtd):
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY, 600, 300).build_tiled()
    with pytest.raises(mtd.MtdError):
        g.set_nest(100)


@pytest.mark.parametrize("kind", ["chol", "lu"])
@pytest.mark.parametrize("n,tile,nest", [(1024, 256, 128), (2048, 512, 128), (1040, 384, 128), (1536, 768, 64),
                                         (4096, 1024, 128)])
def test_tma_fed_updates_match_cp_async_engine(mtd, kind, n, tile, nest, monkeypatch):
    # With MTD_TMA64=1, FP64 GEMM / SYRK items read their operands by TMA when n, the tile and
    # the nested sub-tile are multiples of 16; by default they use the cp.async engine.  Both
    # sum every element in the same k order, so the factors agree bit for bit (and with the
    # oracle).
    a = gen.spd_input(n, 17) if kind == "chol" else gen.lu_input(n, 17)
    outs = []
    for flag in ("0", "1"):
        monkeypatch.setenv("MTD_TMA64", flag)
        g = mtd.TaskGraph(mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU, n, tile).build_tiled()
        g.set_nest(nest).finalize()
        d = to_dev(a)
        assert g.run(d) == 0
        outs.append(from_dev(d))
        d = to_dev(a)
        assert g.run(d) == 0  # a second run on the same graph: barrier parities carried over
        assert np.array_equal(from_dev(d), outs[-1])
        g.close()
    assert np.array_equal(outs[0], outs[1])
    ref = oracle_factor(a, tile, kind)
    out = outs[1]
    if kind == "chol":
        out, ref = np.tril(out), np.tril(ref)
    assert rel_diff(out, ref) <= TOL


def test_mixed_operation_families_in_one_custom_graph(mtd):
    """A custom graph with Cholesky and LU operations together runs the kernel instance that
    carries every operation (pure Cholesky or LU graphs run their family's instance): the
    tiled Cholesky of the leading 2 x 2 tile block beside a tiled LU of the trailing one, on
    a block-diagonal matrix, each against the oracle."""
    n, b = 1024, 256
    a = np.zeros((n, n), order="F")
    a[:512, :512] = gen.spd_input(512, 21)
    a[512:, 512:] = gen.lu_input(512, 22)
    g = mtd.TaskGraph(mtd.KIND_CUSTOM, n, b)
    ch = tiled.cholesky_tasks(2)
    lu = [(op, (wi + 2, wj + 2), [(ri + 2, rj + 2) for ri, rj in reads]) for op, (wi, wj), reads in tiled.lu_tasks(2)]
    for op, write, reads in ch + lu:
        g.add_task(getattr(mtd, "OP_" + {"SYRK": "SYRK_LN"}.get(op, op)), write, reads)
    g.finalize()
    d = to_dev(a)
    assert g.run(d) == 0
    got = from_dev(d)
    want = a.copy(order="F")
    for task in ch + lu:
        assert tiled.run_task(want, b, task) == 0
    assert rel_diff(np.tril(got[:512, :512]), np.tril(want[:512, :512])) <= TOL
    assert rel_diff(got[512:, 512:], want[512:, 512:]) <= TOL
    g.close()
