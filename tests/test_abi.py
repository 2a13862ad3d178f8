"""C-ABI library: loads, exports every declared symbol, and builds the reference's DAGs
on the host exactly as the oracle's restatement of getSubgraphDependencies does."""
import ctypes
import os
import re

import pytest

from oracle import tiled

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    with open(os.path.join(ROOT, "include", "mustard_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mtd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(mtd):
    lib = ctypes.CDLL(mtd.lib_path())
    names = _declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    # and the Python binding declares a signature for each of them
    from mustard_b200 import _capi
    assert set(names) <= set(_capi.SIGNATURES)


def test_abi_version_and_strerror(mtd):
    lib = mtd.lib()
    assert lib.mtd_abi_version() == 1
    for code in range(11):
        assert lib.mtd_strerror(code)
    assert lib.mtd_strerror(0) == b"ok"


def _oracle_ops(kind):
    return {"POTRF": mtd_op("OP_POTRF"), "TRSM_RLT": mtd_op("OP_TRSM_RLT"), "SYRK": mtd_op("OP_SYRK_LN"),
            "GEMM_NT": mtd_op("OP_GEMM_NT"), "GETRF": mtd_op("OP_GETRF"), "TRSM_LLNU": mtd_op("OP_TRSM_LLNU"),
            "TRSM_RUN": mtd_op("OP_TRSM_RUN"), "GEMM_NN": mtd_op("OP_GEMM_NN")}


def mtd_op(name):
    import mustard_b200
    return getattr(mustard_b200, name)


@pytest.mark.parametrize("kind", ["chol", "lu"])
@pytest.mark.parametrize("n,b", [(600, 300), (600, 100), (1000, 128), (24000, 2048), (24000, 1000), (4000, 125)])
def test_build_tiled_matches_oracle_dependencies(mtd, kind, n, b):
    k = mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU
    g = mtd.TaskGraph(k, n, b).build_tiled()
    t = (n + b - 1) // b
    tasks = tiled.cholesky_tasks(t) if kind == "chol" else tiled.lu_tasks(t)
    want = tiled.subgraph_dependencies(tasks)
    assert g.num_tasks == len(tasks)
    for i in range(len(tasks)):
        assert g.deps(i) == want[i], i
    g.close()


@pytest.mark.parametrize("kind", ["chol", "lu"])
def test_tile_edges_give_the_reference_order_over_uneven_tiles(mtd, kind):
    # custom tile edges (a narrower first and last tile): the same task list and dependencies
    # as the reference's order over that many tiles; bad edge lists are refused, and so are
    # edges set after tasks exist
    k = mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU
    edges = [0, 512, 2048, 3584, 4096, 4600]
    g = mtd.TaskGraph(k, 4600, 1536).set_tile_edges(edges).build_tiled()
    t = len(edges) - 1
    tasks = tiled.cholesky_tasks(t) if kind == "chol" else tiled.lu_tasks(t)
    want = tiled.subgraph_dependencies(tasks)
    assert g.num_tasks == len(tasks)
    for i in range(len(tasks)):
        assert g.deps(i) == want[i], i
    with pytest.raises(mtd.MtdError):
        g.set_tile_edges(edges)  # tasks already recorded
    g.close()
    for bad in ([0, 4600], [0, 700, 700, 4600], [1, 4600], [0, 2000, 4000], [0, 3000, 2000, 4600]):
        h = mtd.TaskGraph(k, 4600, 1536)
        if bad == [0, 4600]:
            h.set_tile_edges(bad)  # one tile is allowed
        else:
            with pytest.raises(mtd.MtdError):
                h.set_tile_edges(bad)
        h.close()


def test_creator_mirror_records_reference_calls(mtd):
    # The reference driver's capture sequence for Cholesky T=3 (cholesky_mustard.cu:224-395).
    c = mtd.TiledGraphCreator(mtd.KIND_CUSTOM, 90, 30)
    ops = _oracle_ops("chol")
    for op, write, reads in tiled.cholesky_tasks(3):
        c.beginCaptureOperation(ops[op], write, reads)
        c.endCaptureOperation()
    assert c.subgraphDependencies == tiled.subgraph_dependencies(tiled.cholesky_tasks(3))
    with pytest.raises(mtd.MtdError):
        c.endCaptureOperation()


def test_custom_graph_adds_write_after_read_edges(mtd):
    g = mtd.TaskGraph(mtd.KIND_CUSTOM, 300, 100)
    g.add_task(mtd.OP_POTRF, (0, 0), [(0, 0)])                    # 0
    g.add_task(mtd.OP_TRSM_RLT, (1, 0), [(0, 0), (1, 0)])         # 1 reads (0,0)
    g.add_task(mtd.OP_POTRF, (0, 0), [(0, 0)])                    # 2 overwrites (0,0)
    assert g.deps(2) == [0, 1]  # last writer 0, plus the reader 1 (write-after-read)


@pytest.mark.parametrize("op,write,reads", [
    ("OP_POTRF", (0, 1), [(0, 1)]),                 # off-diagonal POTRF
    ("OP_GEMM_NT", (2, 1), [(2, 1), (2, 0)]),       # missing operand
    ("OP_GEMM_NT", (2, 1), [(2, 1), (1, 0), (2, 0)]),  # operands swapped
    ("OP_TRSM_RLT", (1, 0), [(1, 1), (1, 0)]),      # triangular tile not (k,k) of column k
    ("OP_SYRK_LN", (1, 1), [(1, 0)]),               # output tile not read
    ("OP_GEMM_NN", (1, 1), [(1, 0), (1, 1), (1, 1)]),
    ("OP_POTRF", (5, 5), [(5, 5)]),                 # outside the matrix
])
def test_invalid_tasks_rejected(mtd, op, write, reads):
    g = mtd.TaskGraph(mtd.KIND_CUSTOM, 300, 100)
    with pytest.raises(mtd.MtdError) as e:
        g.add_task(getattr(mtd, op), write, reads)
    assert e.value.status == 1


def test_invalid_graph_arguments(mtd):
    for n, b in [(0, 1), (10, 0), (10, 11), (-5, 2)]:
        with pytest.raises(mtd.MtdError):
            mtd.TaskGraph(mtd.KIND_LU, n, b)
    g = mtd.TaskGraph(mtd.KIND_LU, 100, 10).build_tiled()
    with pytest.raises(mtd.MtdError) as e:
        g.build_tiled()
    assert e.value.status == 2


def test_oversized_task_lists_rejected_before_they_are_built(mtd):
    """The reference's task count is cubic in the tile count: a list past 2^25 tasks is
    refused from the closed form, before anything is built (40960 / 10 -> 4096 tiles,
    ~2.3e10 tasks), and the no-allocation entry point refuses a list longer than its task
    table the same way, before any device work (the pointer is never dereferenced)."""
    import time
    for kind in (mtd.KIND_LU, mtd.KIND_CHOLESKY):
        g = mtd.TaskGraph(kind, 40960, 10)
        t0 = time.perf_counter()
        with pytest.raises(mtd.MtdError) as e:
            g.build_tiled()
        assert e.value.status == 1 and time.perf_counter() - t0 < 1.0
        g.close()
    info = ctypes.c_int(-1)
    t0 = time.perf_counter()
    rc = mtd.lib().mtd_factor_noalloc(mtd.KIND_LU, ctypes.c_void_p(0x1000), 16000, 16000, 8, None,
                                      ctypes.byref(info))
    assert rc == 11 and info.value == 0 and time.perf_counter() - t0 < 1.0
    # the closed form agrees with the oracle's count of the reference's loops
    for t in (1, 2, 6, 8, 47):
        g = mtd.TaskGraph(mtd.KIND_CHOLESKY, 64 * t, 64).build_tiled()
        assert g.num_tasks == tiled.cholesky_task_count(t)
        g.close()
        g = mtd.TaskGraph(mtd.KIND_LU, 64 * t, 64).build_tiled()
        assert g.num_tasks == tiled.lu_task_count(t)
        g.close()


def test_finalize_without_gpu_reports_no_device(mtd):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY, 600, 300).build_tiled()
    with pytest.raises(mtd.MtdError) as e:
        g.finalize()
    assert e.value.status in (3, 8)


def test_trsm_needs_matching_diagonal_factorisation(mtd):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("finalize checks the device first")
    g = mtd.TaskGraph(mtd.KIND_CUSTOM, 200, 100)
    g.add_task(mtd.OP_TRSM_RLT, (1, 0), [(0, 0), (1, 0)])
    with pytest.raises(mtd.MtdError) as e:
        g.finalize()
    assert e.value.status == 7


def _deps_restated(tasks):
    """Last writer of every tile a task reads or writes (mustard/mustard.h:279-296), plus --
    for custom graphs -- every task that read the written tile since its last write."""
    last, readers, out = {}, {}, []
    for idx, (_op, write, reads) in enumerate(tasks):
        d = {last[t] for t in list(reads) + [write] if t in last}
        d |= set(readers.get(write, ()))
        out.append(sorted(d))
        last[write] = idx
        readers[write] = []
        for t in reads:
            if t != write:
                readers.setdefault(t, []).append(idx)
    return out


def _random_cholesky_ops(draw, st, t):
    """One valid Cholesky-shaped task on a t x t tile grid: (op name, write, reads)."""
    kind = draw(st.sampled_from(["OP_POTRF", "OP_TRSM_RLT", "OP_SYRK_LN", "OP_GEMM_NT"]))
    if kind == "OP_POTRF":
        k = draw(st.integers(0, t - 1))
        return kind, (k, k), [(k, k)]
    if kind == "OP_GEMM_NT":
        k = draw(st.integers(0, t - 3))
        i = draw(st.integers(k + 1, t - 2))
        j = draw(st.integers(i + 1, t - 1))
        return kind, (j, i), [(j, i), (j, k), (i, k)]
    k = draw(st.integers(0, t - 2))
    i = draw(st.integers(k + 1, t - 1))
    if kind == "OP_TRSM_RLT":
        return kind, (i, k), [(k, k), (i, k)]
    return kind, (i, i), [(i, k), (i, i)]


def test_custom_graph_dependencies_property(mtd):
    """Random task lists on a 4 x 4 grid: the library's dependency lists equal the restated
    rule (read-after-write, write-after-write and write-after-read edges)."""
    hypothesis = pytest.importorskip("hypothesis")
    st = hypothesis.strategies

    @st.composite
    def task_lists(draw):
        return [_random_cholesky_ops(draw, st, 4) for _ in range(draw(st.integers(1, 40)))]

    @hypothesis.settings(max_examples=150, deadline=None, database=None)
    @hypothesis.given(task_lists())
    def check(tasks):
        g = mtd.TaskGraph(mtd.KIND_CUSTOM, 400, 100)
        try:
            for op, write, reads in tasks:
                g.add_task(getattr(mtd, op), write, reads)
            want = _deps_restated(tasks)
            assert [g.deps(i) for i in range(len(tasks))] == want
        finally:
            g.close()

    check()


def test_header_is_a_c_abi(tmp_path):
    """include/mustard_b200.h compiles as strict C99 and a C program links and calls the
    library (no C++ in the boundary)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib_dir = os.path.join(root, "mustard_b200", "lib")
    src = tmp_path / "abi.c"
    src.write_text('#include "mustard_b200.h"\n'
                   '#include <stdio.h>\n'
                   'int main(void) {\n'
                   '    const char *s = mtd_strerror(MTD_ERR_INVALID_ARG);\n'
                   '    printf("%d %s\\n", mtd_abi_version(), s ? s : "");\n'
                   '    return mtd_abi_version() == MTD_ABI_VERSION ? 0 : 1;\n'
                   '}\n')
    exe = tmp_path / "abi"
    cc = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                         "-I", os.path.join(root, "include"), str(src), "-o", str(exe),
                         "-L", lib_dir, "-lmustard_b200", f"-Wl,-rpath,{lib_dir}"],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr  # the library's ABI version is the header's
    assert len(run.stdout.split()) > 1       # and mtd_strerror names the status
