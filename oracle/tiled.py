"""Oracle restatement of the reference's tiled task lists, dependency inference and
tile arithmetic (test infrastructure only).

Task list order
  Cholesky: mustard/cholesky_mustard.cu:224-395 -- per step k: POTRF(k,k); TRSM(i,k)
            for i>k; then for each i>k: SYRK(i,i) followed by GEMM(j,i) for j>i.
  LU:       mustard/lu_mustard.cu:345-533 -- per step k: GETRF(k,k) (no pivoting,
            ipiv = NULL at :361-369); TRSM-L writing (k,i) for i>k; then for each
            i>k: TRSM-R writing (i,k) followed by GEMM(i,j) for j>k.
Each task is ``(op, write_tile, read_tiles)`` with tiles ``(row_tile, col_tile)``,
exactly the arguments the reference passes to ``beginCaptureOperation``.

Dependency inference restates ``TiledGraphCreator::getSubgraphDependencies``
(mustard/mustard.h:279-296) and the ``tileIndexByMap`` update in
``endCaptureOperation`` (:177): a task depends on the last writer of every tile in
``reads + [write]``, sorted and de-duplicated.

Tile (i, j) covers rows [i*B, min((i+1)*B, n)) and columns [j*B, min((j+1)*B, n))
(the reference's ``matrix + i*B + j*B*N``, cholesky_mustard.cu:157-160).  The
reference requires B | n; this oracle also accepts a ragged last tile.
"""
import numpy as np
from scipy.linalg import blas, lapack

POTRF, TRSM_RLT, SYRK, GEMM_NT = "POTRF", "TRSM_RLT", "SYRK", "GEMM_NT"
GETRF, TRSM_LLNU, TRSM_RUN, GEMM_NN = "GETRF", "TRSM_LLNU", "TRSM_RUN", "GEMM_NN"


def num_tiles(n: int, b: int) -> int:
    return (n + b - 1) // b


def cholesky_tasks(t: int):
    tasks = []
    for k in range(t):
        tasks.append((POTRF, (k, k), [(k, k)]))
        for i in range(k + 1, t):
            tasks.append((TRSM_RLT, (i, k), [(k, k), (i, k)]))
        for i in range(k + 1, t):
            tasks.append((SYRK, (i, i), [(i, i), (i, k)]))
            for j in range(i + 1, t):
                tasks.append((GEMM_NT, (j, i), [(j, i), (j, k), (i, k)]))
    return tasks


def lu_tasks(t: int):
    tasks = []
    for k in range(t):
        tasks.append((GETRF, (k, k), [(k, k)]))
        for i in range(k + 1, t):
            tasks.append((TRSM_LLNU, (k, i), [(k, k), (k, i)]))
        for i in range(k + 1, t):
            tasks.append((TRSM_RUN, (i, k), [(k, k), (i, k)]))
            for j in range(k + 1, t):
                tasks.append((GEMM_NN, (i, j), [(i, k), (k, j), (i, j)]))
    return tasks


def cholesky_task_count(t: int) -> int:
    """cholesky_mustard.cu:200-204."""
    total = t
    for k in range(t):
        for i in range(k + 1, t):
            total += 2 + (t - (i + 1))
    return total


def lu_task_count(t: int) -> int:
    """lu_mustard.cu:322-326."""
    total = t
    for k in range(t):
        for i in range(k + 1, t):
            total += 2 + (t - (k + 1))
    return total


def subgraph_dependencies(tasks):
    """Per-task predecessor lists: last writer of each tile in reads + [write]."""
    index_by_tile = {}
    deps = []
    for idx, (_op, write, reads) in enumerate(tasks):
        found = [index_by_tile[tile] for tile in list(reads) + [write] if tile in index_by_tile]
        deps.append(sorted(set(found)))
        index_by_tile[write] = idx
    return deps


# ---------------------------------------------------------------------------
# tile arithmetic (LAPACK / BLAS through scipy; no-pivot GETRF restated below)
# ---------------------------------------------------------------------------

def getrf_nopiv(a: np.ndarray, nb: int = 64) -> int:
    """In-place right-looking LU without pivoting (what cusolverDnDgetrf computes with
    ipiv = NULL).  Returns LAPACK-style info: 0, or the 1-based index of the first
    zero pivot."""
    n = a.shape[0]
    for j0 in range(0, n, nb):
        j1 = min(j0 + nb, n)
        for j in range(j0, j1):
            piv = a[j, j]
            if piv == 0.0:
                return j + 1
            a[j + 1:, j] /= piv
            a[j + 1:, j + 1:j1] -= np.outer(a[j + 1:, j], a[j, j + 1:j1])
        if j1 < n:
            a[j0:j1, j1:] = blas.dtrsm(1.0, a[j0:j1, j0:j1], a[j0:j1, j1:], side=0, lower=1, diag=1)
            a[j1:, j1:] -= a[j1:, j0:j1] @ a[j0:j1, j1:]
    return 0


def _tile(a, b, ti, tj):
    n = a.shape[0]
    return a[ti * b:min((ti + 1) * b, n), tj * b:min((tj + 1) * b, n)]


def run_task(a: np.ndarray, b: int, task) -> int:
    """Execute one task in place on the column-major matrix ``a``; returns info."""
    op, (wi, wj), reads = task
    c = _tile(a, b, wi, wj)
    if op == POTRF:
        l, info = lapack.dpotrf(c, lower=1, clean=0)
        c[...] = l
        return info
    if op == GETRF:
        return getrf_nopiv(c)
    if op == TRSM_RLT:      # X = A * L^-T   (cublasDtrsm R, L, T, NonUnit)
        k = wj
        c[...] = blas.dtrsm(1.0, _tile(a, b, k, k), c, side=1, lower=1, trans_a=1, diag=0)
        return 0
    if op == TRSM_LLNU:     # X = L^-1 * A   (cublasDtrsm L, L, N, Unit)
        k = wi
        c[...] = blas.dtrsm(1.0, _tile(a, b, k, k), c, side=0, lower=1, trans_a=0, diag=1)
        return 0
    if op == TRSM_RUN:      # X = A * U^-1   (cublasDtrsm R, U, N, NonUnit)
        k = wj
        c[...] = blas.dtrsm(1.0, _tile(a, b, k, k), c, side=1, lower=0, trans_a=0, diag=0)
        return 0
    if op == SYRK:          # C_lower -= A A^T  (cublasDsyrk L, N, -1, 1)
        src = [t for t in reads if t != (wi, wj)][0]
        c[...] = blas.dsyrk(-1.0, _tile(a, b, *src), beta=1.0, c=c, trans=0, lower=1)
        return 0
    if op == GEMM_NT:       # C -= A B^T  (cublasGemmEx N, T, -1, 1)
        src = [t for t in reads if t != (wi, wj)]
        c[...] = blas.dgemm(-1.0, _tile(a, b, *src[0]), _tile(a, b, *src[1]), beta=1.0, c=c, trans_b=1)
        return 0
    if op == GEMM_NN:       # C -= A B  (cublasGemmEx N, N, -1, 1)
        src = [t for t in reads if t != (wi, wj)]
        c[...] = blas.dgemm(-1.0, _tile(a, b, *src[0]), _tile(a, b, *src[1]), beta=1.0, c=c)
        return 0
    raise ValueError(op)


def tiled_factor(a: np.ndarray, b: int, kind: str) -> int:
    """Run the reference's task list sequentially (its creation order is a topological
    order of the DAG).  ``kind`` is "chol" or "lu".  Returns the LAPACK-style info of
    the first failing diagonal task (global 1-based column), or 0."""
    assert a.flags.f_contiguous and a.dtype == np.float64
    t = num_tiles(a.shape[0], b)
    tasks = cholesky_tasks(t) if kind == "chol" else lu_tasks(t)
    for task in tasks:
        info = run_task(a, b, task)
        if info:
            k = task[1][0]
            return k * b + info
    return 0


def cholesky_lapack(a: np.ndarray) -> np.ndarray:
    l, info = lapack.dpotrf(np.asfortranarray(a), lower=1, clean=0)
    assert info == 0, info
    return l


def lu_nopiv_lapack(a: np.ndarray) -> np.ndarray:
    """LAPACK dgetrf with an identity-pivot assertion (valid for diagonally dominant input)."""
    lu, piv, info = lapack.dgetrf(np.asfortranarray(a))
    assert info == 0, info
    assert np.array_equal(piv, np.arange(a.shape[0])), "partial pivoting swapped rows"
    return lu
