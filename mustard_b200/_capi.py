"""ctypes declarations for include/mustard_b200.h."""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libmustard_b200.so")

OK = 0
ERR_INVALID_ARG, ERR_STATE, ERR_CUDA, ERR_TIMEOUT = 1, 2, 3, 4
ERR_NOT_POSITIVE_DEFINITE, ERR_SINGULAR, ERR_BAD_DAG = 5, 6, 7
ERR_NO_DEVICE, ERR_OUT_OF_MEMORY, ERR_QUEUE, ERR_TOO_LARGE = 8, 9, 10, 11
STATUS_NAMES = {
    0: "MTD_OK", 1: "MTD_ERR_INVALID_ARG", 2: "MTD_ERR_STATE", 3: "MTD_ERR_CUDA",
    4: "MTD_ERR_TIMEOUT", 5: "MTD_ERR_NOT_POSITIVE_DEFINITE", 6: "MTD_ERR_SINGULAR",
    7: "MTD_ERR_BAD_DAG", 8: "MTD_ERR_NO_DEVICE", 9: "MTD_ERR_OUT_OF_MEMORY", 10: "MTD_ERR_QUEUE",
    11: "MTD_ERR_TOO_LARGE",
}

KIND_LU, KIND_CHOLESKY, KIND_CUSTOM = 0, 1, 2
OP_POTRF, OP_TRSM_RLT, OP_SYRK_LN, OP_GEMM_NT = 0, 1, 2, 3
OP_GETRF, OP_TRSM_LLNU, OP_TRSM_RUN, OP_GEMM_NN = 4, 5, 6, 7
OP_NAMES = {0: "POTRF", 1: "TRSM_RLT", 2: "SYRK", 3: "GEMM_NT", 4: "GETRF", 5: "TRSM_LLNU",
            6: "TRSM_RUN", 7: "GEMM_NN"}
GEN_UNIFORM_DIAG, GEN_SPD = 0, 1

# Every symbol the header declares, with its ctypes signature.
_vp, _i, _i64, _d = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double


class RunStats(ctypes.Structure):
    _fields_ = [("tasks", ctypes.c_int64), ("items", ctypes.c_int64), ("ctas", ctypes.c_int64),
                ("busy_fraction", ctypes.c_double), ("span_ms", ctypes.c_double)]


PREC_FP64, PREC_TF32, PREC_FP32, PREC_BF16 = 0, 1, 2, 3
REFINE_NONE, REFINE_IR, REFINE_GMRES_IR = 0, 1, 2
BATCH_ORDER_INPUT, BATCH_ORDER_LARGEST_FIRST, BATCH_ORDER_SMALLEST_FIRST = 0, 1, 2
BATCH_SOLVE_LATE, BATCH_SOLVE_PAIRS, BATCH_NUM_SCHEDULES = 4, 8, 12


class SolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("inner_iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("backward_error", ctypes.c_double), ("factor_ms", ctypes.c_double), ("solve_ms", ctypes.c_double)]


class BatchSolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged_count", ctypes.c_int),
                ("max_backward_error", ctypes.c_double), ("solve_ms", ctypes.c_double)]


_pp, _pi64 = ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int64)

SIGNATURES = {
    "mtd_batch_create": (_i, [ctypes.POINTER(_vp), _i, _pi64, _pi64, ctypes.POINTER(_i), _i]),
    "mtd_batch_num_tasks": (_i, [_vp]),
    "mtd_batch_factor": (_i, [_vp, _pp, _pi64, _vp]),
    "mtd_batch_status": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_d)]),
    "mtd_batch_convert": (_i, [_vp, _pp, _pi64, _pp, _pi64, _d, _vp]),
    "mtd_batch_solve": (_i, [_vp, _pp, _pi64, _pp, _pi64, _pp, _pi64, _pp, _pi64, ctypes.POINTER(_i), _i, _d, _i, _vp,
                             ctypes.POINTER(BatchSolveStats)]),
    "mtd_batch_factor_solve": (_i, [_vp, _pp, _pi64, _pp, _pi64, _pp, _pi64, _pp, _pi64, ctypes.POINTER(_i), _i, _d,
                                    _i, _d, _vp]),
    "mtd_batch_solve_status": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_d), ctypes.POINTER(_d),
                                    ctypes.POINTER(_i), ctypes.POINTER(BatchSolveStats)]),
    "mtd_batch_set_schedule": (_i, [_vp, _i]),
    "mtd_batch_get_schedule": (_i, [_vp]),
    "mtd_batch_tune_schedule": (_i, [_vp, _pp, _pi64, _pp, _pi64, _pp, _pi64, _pp, _pi64, _pp, _pi64,
                                     ctypes.POINTER(_i), _i, _d, _i, _d, _i, ctypes.POINTER(_i), ctypes.POINTER(_d),
                                     _vp]),
    "mtd_batch_destroy": (_i, [_vp]),
    "mtd_batch_autotune": (_i, [_i, _pi64, _i, _pi64, ctypes.POINTER(_i), ctypes.POINTER(_d), _vp]),
    "mtd_lupiv_create": (_i, [ctypes.POINTER(_vp), _i64, _i64]),
    "mtd_lupiv_num_tasks": (_i, [_vp]),
    "mtd_lupiv_run": (_i, [_vp, _vp, _i64, _vp, _vp]),
    "mtd_lupiv_status": (_i, [_vp, ctypes.POINTER(_i)]),
    "mtd_lupiv_destroy": (_i, [_vp]),
    "mtd_lu_pivot": (_i, [_vp, _i64, _i64, _i64, _vp, _vp, ctypes.POINTER(_i)]),
    "mtd_adjoint_create": (_i, [ctypes.POINTER(_vp), _i, _pi64, _i64, _i]),
    "mtd_adjoint_num_tasks": (_i, [_vp]),
    "mtd_adjoint_run": (_i, [_vp, _pp, _pi64, _pp, _pi64, _vp]),
    "mtd_adjoint_status": (_i, [_vp, ctypes.POINTER(_d)]),
    "mtd_adjoint_set_trace": (_i, [_vp, _i]),
    "mtd_adjoint_copy_trace": (ctypes.c_longlong, [_vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_longlong]),
    "mtd_adjoint_task_op": (_i, [_vp, _i]),
    "mtd_adjoint_destroy": (_i, [_vp]),
    "mtd_cholesky_adjoint": (_i, [_i, _vp, _i64, _vp, _i64, _i64, _i64, _vp]),
    "mtd_graph_set_precision": (_i, [_vp, _i]),
    "mtd_run_f32": (_i, [_vp, _vp, _i64, _vp, ctypes.POINTER(_i)]),
    "mtd_solver_create": (_i, [ctypes.POINTER(_vp), _i64, _i64, _i]),
    "mtd_solver_factor": (_i, [_vp, _vp, _i64, _d, _vp, ctypes.POINTER(_i)]),
    "mtd_solver_solve": (_i, [_vp, _vp, _i64, _vp, _i64, _i64, _i, _d, _i, _vp, ctypes.POINTER(SolveStats)]),
    "mtd_solver_destroy": (_i, [_vp]),
    "mtd_graph_create": (_i, [ctypes.POINTER(_vp), _i, _i64, _i64]),
    "mtd_graph_add_task": (_i, [_vp, _i, _i, _i, ctypes.POINTER(_i), _i]),
    "mtd_graph_build_tiled": (_i, [_vp]),
    "mtd_graph_num_tasks": (_i, [_vp]),
    "mtd_graph_get_deps": (_i, [_vp, _i, ctypes.POINTER(_i), _i]),
    "mtd_graph_task_info": (_i, [_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i),
                                 ctypes.POINTER(_i), _i]),
    "mtd_graph_task_items": (_i, [_vp, _i]),
    "mtd_graph_device_task_op": (_i, [_vp, _i]),
    "mtd_graph_device_task_deps": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_int), _i]),
    "mtd_graph_num_device_tasks": (_i, [_vp]),
    "mtd_graph_finalize": (_i, [_vp]),
    "mtd_graph_set_trace": (_i, [_vp, _i]),
    "mtd_graph_set_timeout": (_i, [_vp, _d]),
    "mtd_graph_set_nest": (_i, [_vp, _i]),
    "mtd_graph_set_tile_edges": (_i, [_vp, _pi64, _i]),
    "mtd_run": (_i, [_vp, _vp, _i64, _vp, ctypes.POINTER(_i)]),
    "mtd_run_graph": (_i, [_vp, _vp, _i64, _vp, ctypes.POINTER(_i)]),
    "mtd_graph_status": (_i, [_vp, ctypes.POINTER(_i)]),
    "mtd_graph_last_stats": (_i, [_vp, ctypes.POINTER(RunStats)]),
    "mtd_graph_copy_trace": (ctypes.c_longlong, [_vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_longlong]),
    "mtd_graph_destroy": (_i, [_vp]),
    "mtd_tiled_cholesky": (_i, [_vp, _i64, _i64, _i64, _vp, ctypes.POINTER(_i)]),
    "mtd_tiled_lu": (_i, [_vp, _i64, _i64, _i64, _vp, ctypes.POINTER(_i)]),
    "mtd_factor_noalloc": (_i, [_i, _vp, _i64, _i64, _i64, _vp, ctypes.POINTER(_i)]),
    "mtd_generate": (_i, [_vp, _i64, _i64, _i, ctypes.c_uint64, _d, _vp]),
    "mtd_generate_reference_host": (_i, [ctypes.POINTER(_d), _i64]),
    "mtd_probe_fp64_peak": (_i, [ctypes.POINTER(_d)]),
    "mtd_strerror": (ctypes.c_char_p, [_i]),
    "mtd_abi_version": (_i, []),
}

_lib = None


def lib_path():
    return _LIB_PATH


def lib():
    """Load the runtime library (raises ImportError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError(f"mustard_b200 native library missing: {_LIB_PATH} "
                              "(build it with `python mustard_b200/build.py`)")
        handle = ctypes.CDLL(_LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class MtdError(RuntimeError):
    def __init__(self, status, info=0):
        self.status = status
        self.info = info
        msg = lib().mtd_strerror(status).decode() if _lib is not None else STATUS_NAMES.get(status, "?")
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}" + (f" (info={info})" if info else ""))


def check(rc, info=0):
    if rc != OK:
        raise MtdError(rc, info)
