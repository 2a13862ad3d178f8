"""Parity with the reference's own build (mustard/cholesky_mustard.cu, mustard/lu_mustard.cu
compiled for sm_100a by oracle/ref/Makefile into oracle/_ref/): on the reference's default
input (include/gen.h:23-38, srand(420), +n on the diagonal) both builds factor the same
matrix with the same tile edge, the reference through its device-side scheduler
(--subgraph) over cuBLAS / cuSOLVER tile calls, this repository through its persistent
scheduler; the reference's factor is dumped by the verify shim (oracle/ref/shim/verify.h).
Bar: max |diff| / max |reference| <= 1e-12 (lower triangle for Cholesky).

Skipped when the reference's drivers were not built (no reference checkout or no NVSHMEM).
Only tile counts whose --subgraph task count stays within the 120 device graph launches
the reference's scheduler may make are run (oracle/reference_gpu.py says why).
"""
import numpy as np
import pytest

from oracle import gen, reference_gpu
from tests.gpu_util import from_dev, rel_diff, to_dev

TOL = 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["chol", "lu"])
@pytest.mark.parametrize("n,t", [(600, 2), (6000, 6)])
def test_factor_matches_reference_build(mtd, kind, n, t, tmp_path):
    if not reference_gpu.available():
        pytest.skip("the reference's drivers are not built (oracle/ref/Makefile)")
    dump = str(tmp_path / f"{kind}_{n}.bin")
    rec = reference_gpu.run(kind, n, t, "subgraph", runs=1, verify=True, dump=dump, timeout=300)
    assert rec["rc"] == 0, rec.get("tail")
    assert rec.get("passes"), rec
    theirs = reference_gpu.read_dump(dump, n)
    a = gen.ref_spd(n)
    g = mtd.TaskGraph(mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU, n, n // t).build_tiled().finalize()
    d = to_dev(a)
    assert g.run(d) == 0
    g.close()
    ours = from_dev(d)
    if kind == "chol":
        ours, theirs = np.tril(ours), np.tril(theirs)
    assert rel_diff(ours, theirs) <= TOL


def test_reference_refuses_task_counts_past_the_device_launch_limit():
    # Cholesky T = 8 has exactly 120 tasks (allowed); T = 9 has 165; LU T = 7 has 140
    assert reference_gpu.subgraph_tasks("chol", 8) == 120
    assert reference_gpu.subgraph_tasks("lu", 6) == 91
    with pytest.raises(ValueError):
        reference_gpu.run("chol", 900, 9, "subgraph")
    with pytest.raises(ValueError):
        reference_gpu.run("lu", 700, 7, "subgraph")
