"""The oracle against the reference's own generator and verifier (golden fixtures made
by tests/golden/make_golden.py from oracle/_ref/ref_driver), and against LAPACK."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import gen, tiled, verify

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_reference_generator_n15_bit_exact():
    want = np.array([float.fromhex(v) for v in _load("ref_gen.json")["n15"]]).reshape(15, 15)
    got = gen.ref_spd(15)
    assert np.array_equal(np.ascontiguousarray(got), want)


@pytest.mark.parametrize("n", [64, 300, 600])
def test_reference_generator_hash(n):
    want = _load("ref_gen.json")["sha256"][str(n)]
    got = np.ascontiguousarray(gen.ref_spd(n))  # symmetric: row-major bytes as the reference writes
    assert hashlib.sha256(got.tobytes()).hexdigest() == want


def test_product_host_generator_matches_oracle(mtd):
    for n in (15, 64, 300):
        a = mtd.generate_reference_host(n)
        assert np.array_equal(a, np.ascontiguousarray(gen.ref_spd(n)))


@pytest.mark.parametrize("case", _load("ref_verify.json")["cases"], ids=lambda c: f"{c['kind']}-{c['case']}")
def test_verify_matches_reference(case):
    n, b, kind = case["n"], case["tile"], case["kind"]
    a = gen.ref_spd(n)
    f = a.copy(order="F")
    assert tiled.tiled_factor(f, b, kind) == 0
    if case["scale"]:
        rng = np.random.default_rng(case["perturb_seed"])
        for i, j in rng.integers(0, n, size=(case["perturb_count"], 2)):
            if kind == "chol" and i < j:
                i, j = j, i
            f[i, j] += case["scale"]
    err = verify.ref_error_chol(a, f) if kind == "chol" else verify.ref_error_lu(a, f)
    assert f"error = {err:.6f}" == case["error_line"]
    assert int(err <= verify.REF_TOLERANCE) == case["pass"]


def test_task_counts_match_reference_formulas():
    for t in (1, 2, 3, 6, 12):
        assert len(tiled.cholesky_tasks(t)) == tiled.cholesky_task_count(t)
        assert len(tiled.lu_tasks(t)) == tiled.lu_task_count(t)
    assert tiled.lu_task_count(12) == 650 and tiled.lu_task_count(48) == 38024
    assert tiled.cholesky_task_count(12) == 364 and tiled.cholesky_task_count(48) == 19600


def test_dependencies_known_answer_t2():
    # Cholesky, T=2: POTRF(0,0); TRSM(1,0); SYRK(1,1); POTRF(1,1)
    deps = tiled.subgraph_dependencies(tiled.cholesky_tasks(2))
    assert deps == [[], [0], [1], [2]]
    # LU, T=2: GETRF(0,0); TRSM-L(0,1); TRSM-R(1,0); GEMM(1,1); GETRF(1,1)
    deps = tiled.subgraph_dependencies(tiled.lu_tasks(2))
    assert deps == [[], [0], [0], [1, 2], [3]]


def test_dependencies_known_answer_chol_t3():
    tasks = tiled.cholesky_tasks(3)
    names = [(op, w) for op, w, _ in tasks]
    assert names == [("POTRF", (0, 0)), ("TRSM_RLT", (1, 0)), ("TRSM_RLT", (2, 0)),
                     ("SYRK", (1, 1)), ("GEMM_NT", (2, 1)), ("SYRK", (2, 2)),
                     ("POTRF", (1, 1)), ("TRSM_RLT", (2, 1)), ("SYRK", (2, 2)), ("POTRF", (2, 2))]
    assert tiled.subgraph_dependencies(tasks) == [[], [0], [0], [1], [1, 2], [2], [3], [4, 6], [5, 7], [8]]


@pytest.mark.parametrize("n,b", [(600, 300), (257, 64), (100, 32), (15, 3), (130, 128)])
@pytest.mark.parametrize("kind", ["chol", "lu"])
def test_tiled_oracle_matches_lapack(kind, n, b):
    a = gen.ref_spd(n) if n in (600, 15) else (gen.spd_input(n, 3) if kind == "chol" else gen.lu_input(n, 3))
    f = a.copy(order="F")
    assert tiled.tiled_factor(f, b, kind) == 0
    if kind == "chol":
        ref = tiled.cholesky_lapack(a)
        assert np.allclose(np.tril(f), np.tril(ref), rtol=0, atol=1e-13 * np.abs(ref).max())
        assert np.array_equal(np.triu(f, 1), np.triu(a, 1))  # upper triangle untouched
        assert verify.normwise_residual_chol(a, f) < 1e-15
    else:
        ref = tiled.lu_nopiv_lapack(a)
        assert np.allclose(f, ref, rtol=0, atol=1e-13 * np.abs(ref).max())
        assert verify.normwise_residual_lu(a, f) < 1e-15


def test_uniform_generator_stream_properties():
    x = gen.uniform_pm1(300, 200, seed=5)
    assert x.shape == (300, 200) and x.min() >= -1.0 and x.max() < 1.0
    assert abs(x.mean()) < 0.01 and abs(x.var() - 1.0 / 3.0) < 0.01
    # column-major index: entry (i, j) is stream element i + j * rows
    flat = gen.uniform_pm1(300 * 200, 1, seed=5)[:, 0]
    assert np.array_equal(x[:, 7], flat[7 * 300:8 * 300])
    assert not np.array_equal(x, gen.uniform_pm1(300, 200, seed=6))


def test_lu_input_is_column_diagonally_dominant():
    a = gen.lu_input(200, 1)
    off = np.abs(a).sum(axis=0) - np.abs(np.diag(a))
    assert np.all(np.abs(np.diag(a)) > off)


def test_getrf_nopiv_reports_zero_pivot():
    a = np.asfortranarray(np.array([[1.0, 2.0], [0.5, 1.0]]))
    assert tiled.getrf_nopiv(a) == 2


def test_probe_residual_tracks_exact_residual():
    a = gen.spd_input(300, 2)
    f = a.copy(order="F")
    tiled.tiled_factor(f, 128, "chol")
    assert verify.probe_residual(a, f, "chol") < 1e-15
    g = f.copy(order="F")
    g[5, 3] += 1e-6
    assert verify.probe_residual(a, g, "chol") > 1e-10
