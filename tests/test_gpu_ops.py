"""Each tile operation, run through the persistent scheduler as a small custom graph,
against the oracle's LAPACK/BLAS tile arithmetic (oracle/tiled.py run_task).
FP64 parity bar: max |diff| / max |oracle| <= 1e-12."""
import numpy as np
import pytest

from oracle import gen, tiled
from tests.gpu_util import from_dev, rel_diff, to_dev

pytestmark = pytest.mark.gpu
TOL = 1e-12

OPS = {"POTRF": "OP_POTRF", "TRSM_RLT": "OP_TRSM_RLT", "SYRK": "OP_SYRK_LN", "GEMM_NT": "OP_GEMM_NT",
       "GETRF": "OP_GETRF", "TRSM_LLNU": "OP_TRSM_LLNU", "TRSM_RUN": "OP_TRSM_RUN", "GEMM_NN": "OP_GEMM_NN"}


def run_custom(mtd, a, tile, tasks):
    n = a.shape[0]
    g = mtd.TaskGraph(mtd.KIND_CUSTOM, n, tile)
    for op, write, reads in tasks:
        g.add_task(getattr(mtd, OPS[op]), write, reads)
    g.finalize()
    d = to_dev(a)
    g.run(d)
    out = from_dev(d)
    g.close()
    ref = a.copy(order="F")
    for task in tasks:
        assert tiled.run_task(ref, tile, task) == 0
    return out, ref


CASES = [
    # (name, tasks, n, tile)
    ("POTRF", [("POTRF", (0, 0), [(0, 0)])], 300, 300),
    ("POTRF", [("POTRF", (1, 1), [(1, 1)])], 328, 200),          # ragged tile 128
    ("POTRF", [("POTRF", (0, 0), [(0, 0)])], 75, 75),            # odd: 8-byte path
    ("POTRF+TRSM_RLT", [("POTRF", (0, 0), [(0, 0)]), ("TRSM_RLT", (1, 0), [(0, 0), (1, 0)])], 600, 300),
    ("POTRF+TRSM_RLT", [("POTRF", (0, 0), [(0, 0)]), ("TRSM_RLT", (1, 0), [(0, 0), (1, 0)])], 350, 256),
    ("SYRK", [("SYRK", (1, 1), [(1, 1), (1, 0)])], 600, 300),
    ("SYRK", [("SYRK", (1, 1), [(1, 1), (1, 0)])], 500, 256),
    ("GEMM_NT", [("GEMM_NT", (2, 1), [(2, 1), (2, 0), (1, 0)])], 900, 300),
    ("GEMM_NT", [("GEMM_NT", (2, 1), [(2, 1), (2, 0), (1, 0)])], 640, 256),
    ("GEMM_NT", [("GEMM_NT", (2, 1), [(2, 1), (2, 0), (1, 0)])], 33, 13),
    ("GETRF", [("GETRF", (0, 0), [(0, 0)])], 300, 300),
    ("GETRF", [("GETRF", (0, 0), [(0, 0)])], 77, 77),
    ("GETRF+TRSM_LLNU", [("GETRF", (0, 0), [(0, 0)]), ("TRSM_LLNU", (0, 1), [(0, 0), (0, 1)])], 600, 300),
    ("GETRF+TRSM_RUN", [("GETRF", (0, 0), [(0, 0)]), ("TRSM_RUN", (1, 0), [(0, 0), (1, 0)])], 600, 300),
    ("GETRF+TRSM_RUN", [("GETRF", (0, 0), [(0, 0)]), ("TRSM_RUN", (1, 0), [(0, 0), (1, 0)])], 420, 256),
    ("GEMM_NN", [("GEMM_NN", (1, 2), [(1, 0), (0, 2), (1, 2)])], 900, 300),
    ("GEMM_NN", [("GEMM_NN", (1, 2), [(1, 0), (0, 2), (1, 2)])], 700, 256),
]


@pytest.mark.parametrize("name,tasks,n,tile", CASES, ids=[f"{c[0]}-{c[2]}-{c[3]}" for c in CASES])
def test_tile_op_parity(mtd, name, tasks, n, tile):
    lu_like = any(op in ("GETRF", "TRSM_LLNU", "TRSM_RUN", "GEMM_NN") for op, _, _ in tasks)
    a = gen.lu_input(n, 17) if lu_like else gen.spd_input(n, 17)
    out, ref = run_custom(mtd, a, tile, tasks)
    assert rel_diff(out, ref) <= TOL
    # tiles nobody writes are untouched, bit for bit
    written = {w for _, w, _ in tasks}
    t = (n + tile - 1) // tile
    for i in range(t):
        for j in range(t):
            if (i, j) not in written:
                sl = (slice(i * tile, min((i + 1) * tile, n)), slice(j * tile, min((j + 1) * tile, n)))
                assert np.array_equal(out[sl], a[sl])


def test_gemm_accumulates_full_k(mtd):
    # K = tile edge 512 through the 16-deep pipeline with a ragged output block
    n, tile = 1500, 512
    a = gen.uniform_pm1(n, n, 3)
    a = np.asfortranarray(a)
    out, ref = run_custom(mtd, a, tile, [("GEMM_NT", (2, 1), [(2, 1), (2, 0), (1, 0)])])
    assert rel_diff(out, ref) <= TOL
