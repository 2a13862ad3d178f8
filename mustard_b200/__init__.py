"""mustard_b200: B200 (sm_100a) runtime for static tiled LU / Cholesky task graphs.

Python view of the C ABI in include/mustard_b200.h (loaded with ctypes from the in-tree
``mustard_b200/lib/libmustard_b200.so``).  The reference's host interface is the C++
``mustard::TiledGraphCreator`` (mustard/mustard.h:132-384); ``TiledGraphCreator`` below
keeps its names -- ``beginCaptureOperation`` / ``endCaptureOperation`` /
``subgraphDependencies`` -- with the captured library call replaced by the operation
code given to ``beginCaptureOperation``.

Matrices are FP64 and column-major.  A torch tensor ``a`` of shape (n, n) is passed as
the column-major matrix ``a.T`` when ``a.T`` is contiguous (``colmajor(x)`` makes one),
i.e. the storage order is the reference's ``matrix[i + j * N]``.

There is no CPU fallback: if the shared library is missing, importing this package
raises ``ImportError``.
"""
import ctypes
import os

from . import _capi
from ._capi import (  # noqa: F401  (re-exported constants)
    BATCH_NUM_SCHEDULES, BATCH_ORDER_INPUT, BATCH_ORDER_LARGEST_FIRST, BATCH_ORDER_SMALLEST_FIRST,
    BATCH_SOLVE_LATE, BATCH_SOLVE_PAIRS, GEN_SPD, GEN_UNIFORM_DIAG, KIND_CHOLESKY, KIND_CUSTOM, KIND_LU, OP_GEMM_NN, OP_GEMM_NT,
    OP_GETRF, OP_NAMES, OP_POTRF, OP_SYRK_LN, OP_TRSM_LLNU, OP_TRSM_RLT, OP_TRSM_RUN,
    PREC_BF16, PREC_FP32, PREC_FP64, PREC_TF32, REFINE_GMRES_IR, REFINE_IR, REFINE_NONE, STATUS_NAMES, MtdError,
    lib, lib_path)

__all__ = [
    "TaskGraph", "TiledGraphCreator", "tiled_cholesky", "tiled_lu", "lu_pivot", "PivotedLU", "generate", "colmajor",
    "probe_fp64_peak", "MtdError", "lib", "lib_path",
]


def _stream_handle(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if hasattr(stream, "cuda_stream"):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def _matrix_ptr(a, n=None):
    """(pointer, n, lda) of a column-major FP64 CUDA matrix given as a torch tensor whose
    transpose is contiguous (shape (n, n), strides (1, lda)), or as an int pointer."""
    if isinstance(a, int):
        if n is None:
            raise ValueError("n is required with a raw pointer")
        return a, n, n
    import torch
    if a.dtype != torch.float64 or not a.is_cuda:
        raise TypeError("expected a float64 CUDA tensor")
    if a.dim() != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("expected a square matrix")
    if a.stride(0) != 1 or a.stride(1) < a.shape[0]:
        raise ValueError("expected column-major storage (use mustard_b200.colmajor)")
    return a.data_ptr(), a.shape[0], a.stride(1)


def colmajor(x):
    """Column-major copy of a square torch tensor (same values, Fortran storage)."""
    return x.t().contiguous().t()


class TaskGraph:
    """Owner of one ``mtd_graph``."""

    def __init__(self, kind, n, tile):
        self._lib = lib()
        h = ctypes.c_void_p()
        _capi.check(self._lib.mtd_graph_create(ctypes.byref(h), kind, n, tile))
        self._h = h
        self.kind, self.n, self.tile = kind, n, tile
        self.tiles = (n + tile - 1) // tile
        self.finalized = False

    # -- construction ------------------------------------------------------
    def add_task(self, op, write, reads):
        flat = [int(v) for tile in reads for v in tile]
        arr = (ctypes.c_int * max(len(flat), 1))(*flat)
        rc = self._lib.mtd_graph_add_task(self._h, op, int(write[0]), int(write[1]), arr, len(reads))
        if rc < 0:
            raise MtdError(-rc)
        return rc

    def build_tiled(self):
        _capi.check(self._lib.mtd_graph_build_tiled(self._h))
        return self

    def set_trace(self, enable=True):
        _capi.check(self._lib.mtd_graph_set_trace(self._h, 1 if enable else 0))
        return self

    def set_tile_edges(self, edges):
        """Tiles at the given element edges (0 < ... < n) instead of uniform ones."""
        arr = (ctypes.c_int64 * len(edges))(*edges)
        _capi.check(self._lib.mtd_graph_set_tile_edges(self._h, arr, len(edges)))
        return self

    def set_nest(self, nest):
        """Sub-tile edge of nested diagonal factorisations (multiple of 64; 0 = off)."""
        _capi.check(self._lib.mtd_graph_set_nest(self._h, int(nest)))
        return self

    def set_timeout(self, seconds):
        _capi.check(self._lib.mtd_graph_set_timeout(self._h, float(seconds)))
        return self

    def finalize(self):
        _capi.check(self._lib.mtd_graph_finalize(self._h))
        self.finalized = True
        return self

    # -- queries -----------------------------------------------------------
    @property
    def num_tasks(self):
        return self._lib.mtd_graph_num_tasks(self._h)

    def deps(self, task):
        cnt = self._lib.mtd_graph_get_deps(self._h, task, None, 0)
        if cnt < 0:
            raise MtdError(-cnt)
        buf = (ctypes.c_int * max(cnt, 1))()
        self._lib.mtd_graph_get_deps(self._h, task, buf, cnt)
        return list(buf[:cnt])

    def task_info(self, task):
        """(op, write tile, read tiles) of host task ``task``, as it was recorded."""
        op, wi, wj = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        buf = (ctypes.c_int * 16)()
        nr = self._lib.mtd_graph_task_info(self._h, task, ctypes.byref(op), ctypes.byref(wi), ctypes.byref(wj), buf, 8)
        if nr < 0:
            raise MtdError(-nr)
        return op.value, (wi.value, wj.value), [(buf[2 * r], buf[2 * r + 1]) for r in range(nr)]

    def items(self, task):
        return self._lib.mtd_graph_task_items(self._h, task)

    def device_task_deps(self, task):
        """Predecessor device tasks of device task ``task`` (after finalize)."""
        cnt = self._lib.mtd_graph_device_task_deps(self._h, task, None, 0)
        if cnt < 0:
            raise MtdError(-cnt)
        buf = (ctypes.c_int * max(cnt, 1))()
        self._lib.mtd_graph_device_task_deps(self._h, task, buf, cnt)
        return list(buf[:cnt])

    def device_task_op(self, task):
        """Operation (OP_*; 100 for a join) of device task ``task``, the index trace records carry."""
        op = self._lib.mtd_graph_device_task_op(self._h, task)
        if op < 0:
            raise MtdError(-op)
        return op

    @property
    def num_device_tasks(self):
        """Device tasks after finalize (nested diagonal factorisations expanded)."""
        return self._lib.mtd_graph_num_device_tasks(self._h)

    # -- execution ---------------------------------------------------------
    def run(self, a, stream=None, sync=True, lda=None):
        """Factor the column-major device matrix ``a`` in place.  With ``sync`` the call
        waits and raises MtdError on failure; otherwise it returns at once and
        ``status()`` reports later."""
        ptr, n, ld = _matrix_ptr(a, self.n)
        if lda is not None:
            ld = lda
        if n != self.n:
            raise ValueError(f"matrix is {n}x{n}, graph expects {self.n}")
        info = ctypes.c_int(0)
        rc = self._lib.mtd_run(self._h, ctypes.c_void_p(ptr), ld, _stream_handle(stream),
                               ctypes.byref(info) if sync else None)
        _capi.check(rc, info.value)
        return info.value

    def set_precision(self, prec):
        _capi.check(self._lib.mtd_graph_set_precision(self._h, int(prec)))
        return self

    def run_f32(self, a, stream=None, sync=True):
        """Run a PREC_TF32 graph on a column-major float32 CUDA matrix."""
        import torch
        if a.dtype != torch.float32 or not a.is_cuda or a.stride(0) != 1:
            raise TypeError("expected a column-major float32 CUDA tensor")
        info = ctypes.c_int(0)
        rc = self._lib.mtd_run_f32(self._h, ctypes.c_void_p(a.data_ptr()), a.stride(1), _stream_handle(stream),
                                   ctypes.byref(info) if sync else None)
        _capi.check(rc, info.value)
        return info.value

    def run_graph(self, a, stream=None, sync=True):
        """Same factorisation through the host-launched CUDA-graph executor (the
        reference's --tiled mode) instead of the persistent scheduler."""
        ptr, n, ld = _matrix_ptr(a, self.n)
        if n != self.n:
            raise ValueError(f"matrix is {n}x{n}, graph expects {self.n}")
        info = ctypes.c_int(0)
        rc = self._lib.mtd_run_graph(self._h, ctypes.c_void_p(ptr), ld, _stream_handle(stream),
                                     ctypes.byref(info) if sync else None)
        _capi.check(rc, info.value)
        return info.value

    def status(self):
        info = ctypes.c_int(0)
        rc = self._lib.mtd_graph_status(self._h, ctypes.byref(info))
        return rc, info.value

    def stats(self):
        s = _capi.RunStats()
        _capi.check(self._lib.mtd_graph_last_stats(self._h, ctypes.byref(s)))
        return {"tasks": s.tasks, "items": s.items, "ctas": s.ctas,
                "busy_fraction": s.busy_fraction, "span_ms": s.span_ms}

    def trace(self, max_records=None):
        """Per-item records of the last traced run: list of (start_ns, end_ns, sm, task, item)."""
        cap = max_records or 1 << 22
        buf = (ctypes.c_ulonglong * (4 * cap))()
        n = self._lib.mtd_graph_copy_trace(self._h, buf, cap)
        if n < 0:
            raise MtdError(-n)
        return [(buf[4 * i], buf[4 * i + 1], buf[4 * i + 2], buf[4 * i + 3] >> 32, buf[4 * i + 3] & 0xFFFFFFFF)
                for i in range(n)]

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mtd_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class TiledGraphCreator:
    """The reference's TiledGraphCreator (mustard/mustard.h:132-384) over the C ABI.

    ``beginCaptureOperation(op, tileToWrite, tilesToRead)`` records a task (the reference
    captures the library call issued between begin and end; here the call is named by
    ``op``), ``endCaptureOperation()`` closes it, and ``subgraphDependencies[i]`` is the
    sorted predecessor list of task i (mustard/mustard.h:279-296)."""

    def __init__(self, kind, n, tile):
        self.graph = TaskGraph(kind, n, tile)
        self._open = None

    def beginCaptureOperation(self, op, tileToWrite, tilesToRead):
        if self._open is not None:
            raise MtdError(_capi.ERR_STATE)
        self._open = (op, tuple(tileToWrite), [tuple(t) for t in tilesToRead])

    def endCaptureOperation(self):
        if self._open is None:
            raise MtdError(_capi.ERR_STATE)
        op, write, reads = self._open
        self._open = None
        return self.graph.add_task(op, write, reads)

    @property
    def subgraphDependencies(self):
        return [self.graph.deps(t) for t in range(self.graph.num_tasks)]


def _rect_ptr(x, rows):
    """(pointer, leading dimension, columns) of a column-major float64 CUDA block (n x k)."""
    import torch
    if x.dtype != torch.float64 or not x.is_cuda:
        raise TypeError("expected a float64 CUDA tensor")
    if x.dim() == 1:
        x = x.unsqueeze(1)
    if x.shape[0] != rows or x.stride(0) != 1:
        raise ValueError("expected a column-major (n, k) block")
    return x.data_ptr(), (x.stride(1) if x.shape[1] > 1 else rows), x.shape[1]


class SpdSolver:
    """Mixed-precision SPD solver (mtd_solver_*): low-precision tiled Cholesky on the task
    scheduler plus FP64 iterative refinement (IR) or GMRES-IR.  ``prec`` is PREC_TF32
    (FP32 factor, TF32 tensor-core products) or PREC_FP64 (the plain FP64 baseline)."""

    def __init__(self, n, tile, prec=_capi.PREC_TF32):
        self._lib = lib()
        h = ctypes.c_void_p()
        _capi.check(self._lib.mtd_solver_create(ctypes.byref(h), n, tile, prec))
        self._h, self.n, self.tile, self.prec = h, n, tile, prec

    def factor(self, a, shift=0.0, stream=None):
        """Factor A + shift*I (A: column-major float64 CUDA matrix, kept by reference)."""
        ptr, n, ld = _matrix_ptr(a, self.n)
        self._a = a
        info = ctypes.c_int(0)
        _capi.check(self._lib.mtd_solver_factor(self._h, ctypes.c_void_p(ptr), ld, float(shift),
                                                _stream_handle(stream), ctypes.byref(info)), info.value)
        return info.value

    def solve(self, b, x, method=_capi.REFINE_IR, tol=1e-13, max_iter=50, stream=None):
        """Solve A X = B into x (both column-major (n, k) float64 CUDA blocks, k <= 16)."""
        pb, ldb, k = _rect_ptr(b, self.n)
        px, ldx, kx = _rect_ptr(x, self.n)
        if k != kx:
            raise ValueError("b and x must have the same number of columns")
        st = _capi.SolveStats()
        rc = self._lib.mtd_solver_solve(self._h, ctypes.c_void_p(pb), ldb, ctypes.c_void_p(px), ldx, k, method,
                                        float(tol), int(max_iter), _stream_handle(stream), ctypes.byref(st))
        _capi.check(rc)
        return {"iterations": st.iterations, "inner_iterations": st.inner_iterations,
                "converged": bool(st.converged), "backward_error": st.backward_error,
                "factor_ms": st.factor_ms, "solve_ms": st.solve_ms}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mtd_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _autotune_call(sizes, prec, stream):
    c = len(sizes)
    n = (ctypes.c_int64 * c)(*sizes)
    t = (ctypes.c_int64 * c)()
    k = (ctypes.c_int * c)()
    ms = ctypes.c_double(0.0)
    _capi.check(lib().mtd_batch_autotune(c, n, prec, t, k, ctypes.byref(ms), _stream_handle(stream)))
    return list(t), list(k), ms.value


def batch_autotune(sizes, prec=_capi.PREC_FP64, stream=None, table=None):
    """(tiles, nests, wall ms) chosen by mtd_batch_autotune for a batch of these sizes.

    ``table``: path of a JSON file of earlier choices (mustard_b200.tune_table), kept per
    device and precision.  Sizes it holds are not tuned again; the others are tuned with
    their share of this batch (so the trial counts are the ones a full call would use), and
    their choices are added to the file."""
    if table is None:
        return _autotune_call(sizes, prec, stream)
    import torch
    from . import tune_table
    device = torch.cuda.get_device_name(torch.cuda.current_device())
    tab = tune_table.load(table)
    todo = tune_table.missing(tab, device, prec, sizes)
    ms = 0.0
    if todo:
        sub = [sizes[i] for i in todo]
        t, k, ms = _autotune_call(sub, prec, stream)
        for n, ti, ki in zip(sub, t, k):
            tune_table.record(tab, device, prec, n, ti, ki)
        tune_table.save(tab, table)
    tiles, nests = [], []
    for n in sizes:
        ti, ki = tune_table.lookup(tab, device, prec, n)
        tiles.append(ti)
        nests.append(ki)
    return tiles, nests, ms


class Batch:
    """Batched Cholesky factorisations and solves (mtd_batch_*): matrices of different sizes
    factored as one merged task graph in one persistent launch.

    ``sizes``: list of n; ``tiles`` / ``nests``: per-matrix tile edge and nested sub-tile
    edge (None: the library's defaults).  Matrices are column-major CUDA tensors (float64
    for PREC_FP64, float32 for PREC_TF32 / PREC_FP32)."""

    def __init__(self, sizes, tiles=None, nests=None, prec=_capi.PREC_FP64):
        self._lib = lib()
        self.count = len(sizes)
        n = (ctypes.c_int64 * self.count)(*sizes)
        t = (ctypes.c_int64 * self.count)(*tiles) if tiles is not None else None
        k = (ctypes.c_int * self.count)(*nests) if nests is not None else None
        h = ctypes.c_void_p()
        _capi.check(self._lib.mtd_batch_create(ctypes.byref(h), self.count, n, t, k, prec))
        self._h, self.sizes, self.prec = h, list(sizes), prec

    @property
    def num_tasks(self):
        return self._lib.mtd_batch_num_tasks(self._h)

    @staticmethod
    def _ptrs(mats):
        p = (ctypes.c_void_p * len(mats))(*[m.data_ptr() for m in mats])
        ld = (ctypes.c_int64 * len(mats))(*[(m.stride(1) if m.dim() == 2 and m.shape[1] > 1 else m.shape[0])
                                             for m in mats])
        return p, ld

    def factor(self, mats, stream=None):
        p, ld = self._ptrs(mats)
        self._keep = mats
        _capi.check(self._lib.mtd_batch_factor(self._h, p, ld, _stream_handle(stream)))

    def status(self, latencies=False):
        info = (ctypes.c_int * self.count)()
        lat = (ctypes.c_double * self.count)() if latencies else None
        rc = self._lib.mtd_batch_status(self._h, info, lat)
        out = (rc, list(info))
        return out + (list(lat),) if latencies else out

    def convert(self, a64, f32, shift=0.0, stream=None):
        pa, la = self._ptrs(a64)
        pf, lf = self._ptrs(f32)
        _capi.check(self._lib.mtd_batch_convert(self._h, pa, la, pf, lf, float(shift), _stream_handle(stream)))

    def solve(self, factors, bs, xs, a64=None, method=_capi.REFINE_NONE, tol=1e-13, max_iter=20, stream=None):
        pf, lf = self._ptrs(factors)
        pb, lb = self._ptrs(bs)
        px, lx = self._ptrs(xs)
        nr = (ctypes.c_int * self.count)(*[(b.shape[1] if b.dim() == 2 else 1) for b in bs])
        pa, la = self._ptrs(a64) if a64 is not None else (None, None)
        st = _capi.BatchSolveStats()
        _capi.check(self._lib.mtd_batch_solve(self._h, pa, la, pf, lf, pb, lb, px, lx, nr, method, float(tol),
                                              int(max_iter), _stream_handle(stream), ctypes.byref(st)))
        return {"iterations": st.iterations, "converged_count": st.converged_count,
                "max_backward_error": st.max_backward_error, "solve_ms": st.solve_ms}

    def _solve_args(self, factors, bs, xs, a64):
        pf, lf = self._ptrs(factors)
        pb, lb = self._ptrs(bs)
        px, lx = self._ptrs(xs)
        nr = (ctypes.c_int * self.count)(*[(b.shape[1] if b.dim() == 2 else 1) for b in bs])
        pa, la = self._ptrs(a64) if a64 is not None else (None, None)
        return pf, lf, pa, la, pb, lb, px, lx, nr

    def factor_solve(self, factors, bs, xs, a64=None, method=_capi.REFINE_NONE, tol=1e-13, max_iter=20,
                     shift=0.0, stream=None):
        """Factor and solve in ONE persistent launch (mtd_batch_factor_solve; stream-ordered,
        CUDA-graph capturable).  FP64 batches factor ``factors`` in place; low-precision
        batches write them from ``a64`` (+ shift I) inside the launch.  Results:
        solve_status()."""
        args = self._solve_args(factors, bs, xs, a64)
        self._keep = (factors, bs, xs, a64)
        _capi.check(self._lib.mtd_batch_factor_solve(self._h, *args, method, float(tol), int(max_iter),
                                                     float(shift), _stream_handle(stream)))

    def solve_status(self):
        """Wait for the last factor_solve: (rc, info, latency_ms, berr, iterations, stats)."""
        c = self.count
        info, lat = (ctypes.c_int * c)(), (ctypes.c_double * c)()
        berr, its = (ctypes.c_double * c)(), (ctypes.c_int * c)()
        st = _capi.BatchSolveStats()
        rc = self._lib.mtd_batch_solve_status(self._h, info, lat, berr, its, ctypes.byref(st))
        stats = {"iterations": st.iterations, "converged_count": st.converged_count,
                 "max_backward_error": st.max_backward_error, "device_ms": st.solve_ms}
        return rc, list(info), list(lat), list(berr), list(its), stats

    @property
    def schedule(self):
        return self._lib.mtd_batch_get_schedule(self._h)

    @schedule.setter
    def schedule(self, value):
        _capi.check(self._lib.mtd_batch_set_schedule(self._h, int(value)))

    def tune_schedule(self, factors, bs, xs, a64=None, source=None, method=_capi.REFINE_NONE, tol=1e-13,
                      max_iter=20, shift=0.0, reps=2, stream=None):
        """Time factor_solve under each CTA-to-task schedule and keep the fastest
        (mtd_batch_tune_schedule).  FP64 batches need ``source``: the inputs ``factors`` is
        restored from before every trial.  Returns (schedule, {schedule: ms})."""
        pf, lf, pa, la, pb, lb, px, lx, nr = self._solve_args(factors, bs, xs, a64)
        ps, ls = self._ptrs(source) if source is not None else (None, None)
        best = ctypes.c_int(0)
        ms = (ctypes.c_double * _capi.BATCH_NUM_SCHEDULES)()
        self._keep = (factors, bs, xs, a64, source)
        _capi.check(self._lib.mtd_batch_tune_schedule(self._h, pf, lf, ps, ls, pa, la, pb, lb, px, lx, nr, method,
                                                      float(tol), int(max_iter), float(shift), int(reps),
                                                      ctypes.byref(best), ms, _stream_handle(stream)))
        sched = [(c % 6 // 2) | (_capi.BATCH_SOLVE_LATE if c % 2 else 0) | (_capi.BATCH_SOLVE_PAIRS if c >= 6 else 0)
                 for c in range(_capi.BATCH_NUM_SCHEDULES)]
        return best.value, {s: ms[c] for c, s in enumerate(sched)}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mtd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CholeskyAdjoint:
    """Blocked Cholesky adjoint (mtd_adjoint_*): for factors L_m (lower) and Lbar_m =
    dLoss/dL_m, overwrite each Lbar_m's lower triangle with Abar_m = dLoss/dA_m (gradient
    with respect to the lower triangle of A_m).  Many matrices of different sizes run as
    one merged reverse task graph in one persistent launch.  Matrices are column-major
    CUDA tensors: float64 for PREC_FP64, float32 for PREC_FP32 (split-TF32 products)."""

    def __init__(self, sizes, tile=128, prec=_capi.PREC_FP64):
        self._lib = lib()
        self.count = len(sizes)
        n = (ctypes.c_int64 * self.count)(*sizes)
        h = ctypes.c_void_p()
        _capi.check(self._lib.mtd_adjoint_create(ctypes.byref(h), self.count, n, tile, prec))
        self._h, self.sizes, self.tile, self.prec = h, list(sizes), tile, prec

    def num_tasks(self):
        return self._lib.mtd_adjoint_num_tasks(self._h)

    def run(self, factors, lbars, stream=None):
        """Stream-ordered; returns immediately (wait with status())."""
        pl, ll = Batch._ptrs(factors)
        pb, lb = Batch._ptrs(lbars)
        self._keep = (factors, lbars)
        _capi.check(self._lib.mtd_adjoint_run(self._h, pl, ll, pb, lb, _stream_handle(stream)))

    def status(self):
        """Wait for the last run; returns its device time in ms."""
        ms = ctypes.c_double(0.0)
        _capi.check(self._lib.mtd_adjoint_status(self._h, ctypes.byref(ms)))
        return ms.value

    ADJOINT_OP_NAMES = {20: "X L^-1", 21: "C -= A B", 22: "C -= A^T B", 23: "diagonal adjoint"}

    def set_trace(self, enable=True):
        _capi.check(self._lib.mtd_adjoint_set_trace(self._h, int(enable)))
        return self

    def op_times(self):
        """Per operation of the last traced run: items and summed / median item time (us)."""
        import statistics
        cap = 1 << 22
        buf = (ctypes.c_ulonglong * (4 * cap))()
        n = self._lib.mtd_adjoint_copy_trace(self._h, buf, cap)
        if n < 0:
            _capi.check(-n)
        per = {}
        for i in range(n):
            s, e, task = buf[4 * i], buf[4 * i + 1], buf[4 * i + 3] >> 32
            if e <= s:
                continue
            op = self._lib.mtd_adjoint_task_op(self._h, int(task))
            per.setdefault(self.ADJOINT_OP_NAMES.get(op, op), []).append((e - s) * 1e-3)
        return {k: {"items": len(v), "total_us": sum(v), "median_us": statistics.median(v)} for k, v in per.items()}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mtd_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cholesky_adjoint(factor, lbar, tile=128, stream=None):
    """One matrix, synchronous: ``lbar``'s lower triangle becomes dLoss/dA (see
    CholeskyAdjoint).  Both column-major CUDA tensors of the same dtype."""
    import torch
    prec = _capi.PREC_FP64 if factor.dtype == torch.float64 else _capi.PREC_FP32
    (pl,), (ll,) = Batch._ptrs([factor])
    (pb,), (lb,) = Batch._ptrs([lbar])
    _capi.check(lib().mtd_cholesky_adjoint(prec, ctypes.c_void_p(pl), ll, ctypes.c_void_p(pb), lb, factor.shape[0],
                                           tile, _stream_handle(stream)))


def _one_call(kind, a, tile, stream):
    ptr, n, ld = _matrix_ptr(a)
    info = ctypes.c_int(0)
    fn = lib().mtd_tiled_cholesky if kind == KIND_CHOLESKY else lib().mtd_tiled_lu
    rc = fn(ctypes.c_void_p(ptr), n, ld, tile, _stream_handle(stream), ctypes.byref(info))
    _capi.check(rc, info.value)
    return info.value


def tiled_cholesky(a, tile, stream=None):
    """In-place lower Cholesky of the column-major CUDA matrix ``a`` (tiledCholesky,
    mustard/cholesky_mustard.cu:135)."""
    return _one_call(KIND_CHOLESKY, a, tile, stream)


def tiled_lu(a, tile, stream=None):
    """In-place no-pivot LU of the column-major CUDA matrix ``a`` (tiledLU,
    mustard/lu_mustard.cu:256)."""
    return _one_call(KIND_LU, a, tile, stream)


class PivotedLU:
    """LU with partial pivoting (mtd_lupiv): P A = L U with LAPACK dgetrf's interchanges, as
    one persistent launch over a task graph built once for (n, tile).  No counterpart in
    the reference, which factors without pivoting."""

    def __init__(self, n, tile=128):
        self._lib = lib()
        h = ctypes.c_void_p()
        _capi.check(self._lib.mtd_lupiv_create(ctypes.byref(h), n, tile))
        self._h, self.n, self.tile = h, n, tile

    @property
    def num_tasks(self):
        return self._lib.mtd_lupiv_num_tasks(self._h)

    def run(self, a, ipiv, stream=None):
        """Factor the column-major float64 CUDA matrix ``a`` in place; ``ipiv``: an int32
        CUDA tensor of n entries (LAPACK's 1-based pivots on completion).  Stream-ordered."""
        ptr, n, ld = _matrix_ptr(a)
        if n != self.n or ipiv.numel() < n or not ipiv.is_cuda or ipiv.element_size() != 4:
            raise ValueError("matrix size or pivot vector does not match")
        self._keep = (a, ipiv)
        _capi.check(self._lib.mtd_lupiv_run(self._h, ctypes.c_void_p(ptr), ld, ctypes.c_void_p(ipiv.data_ptr()),
                                            _stream_handle(stream)))

    def status(self):
        """Wait for the last run; returns LAPACK's info (0, or the first zero pivot's column)."""
        info = ctypes.c_int(0)
        _capi.check(self._lib.mtd_lupiv_status(self._h, ctypes.byref(info)))
        return info.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mtd_lupiv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def lu_pivot(a, tile=128, stream=None):
    """In-place LU with partial pivoting of the column-major float64 CUDA matrix ``a``
    (dgetrf's result); returns (info, ipiv) with ipiv an int32 CUDA tensor, 1-based."""
    import torch
    ptr, n, ld = _matrix_ptr(a)
    ipiv = torch.empty(n, dtype=torch.int32, device=a.device)
    info = ctypes.c_int(0)
    _capi.check(lib().mtd_lu_pivot(ctypes.c_void_p(ptr), n, ld, tile, ctypes.c_void_p(ipiv.data_ptr()),
                                   _stream_handle(stream), ctypes.byref(info)))
    return info.value, ipiv


def generate(a, which, seed=0, alpha=1.0, stream=None):
    """Fill the column-major CUDA matrix ``a`` with a seeded benchmark input."""
    ptr, n, ld = _matrix_ptr(a)
    _capi.check(lib().mtd_generate(ctypes.c_void_p(ptr), n, ld, which, ctypes.c_uint64(seed),
                                   ctypes.c_double(alpha), _stream_handle(stream)))


def generate_reference_host(n):
    """The reference's host input (include/gen.h:23-38) as a numpy array (symmetric)."""
    import numpy as np
    out = np.empty((n, n), dtype=np.float64)
    _capi.check(lib().mtd_generate_reference_host(out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))
    return out


def probe_fp64_peak():
    """Measured FP64 tensor-core (DMMA) rate of the current device, TFLOP/s."""
    v = ctypes.c_double(0.0)
    _capi.check(lib().mtd_probe_fp64_peak(ctypes.byref(v)))
    return v.value


LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

lib()  # fail at import when the native library is missing: there is no fallback path
