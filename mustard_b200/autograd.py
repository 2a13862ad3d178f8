"""torch.autograd.Function over the scheduler's batched Cholesky and its blocked adjoint.

    L = cholesky(A, tile=256, recompute=False)     # A: (n, n) or (B, n, n), SPD

Forward: one merged task graph factors every matrix of the batch (mtd_batch_*: FP64 for
float64 input; FP32 storage with FP32-accurate split-TF32 products for float32).
Backward: the blocked reverse sweep (mtd_adjoint_*) over the same tiles turns dLoss/dL
into dLoss/dA, returned in torch's symmetric convention ((Abar + Abar^T) / 2, the diagonal
kept), as torch.linalg.cholesky's gradient is.  ``recompute=True`` keeps only A between the
passes and factors again in backward (less memory held by autograd, one more
factorisation); ``recompute=False`` keeps L.
"""
import ctypes

import torch

from . import _capi
from ._capi import lib

_batches = {}
_adjoints = {}


def _prec(dtype):
    if dtype == torch.float64:
        return _capi.PREC_FP64
    if dtype == torch.float32:
        return _capi.PREC_FP32
    raise TypeError("cholesky: float64 or float32 input")


def _table(x):
    """Pointer and leading-dimension arrays of the (B, n, n) contiguous stack x, each
    matrix read as column-major (its row-major storage holds the transpose)."""
    b, n = x.shape[0], x.shape[-1]
    step = n * n * x.element_size()
    base = x.data_ptr()
    p = (ctypes.c_void_p * b)(*[base + i * step for i in range(b)])
    ld = (ctypes.c_int64 * b)(*([n] * b))
    return p, ld


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _factor(a, tile):
    """(B, n, n) SPD -> (B, n, n) lower factors, via one merged task graph.  The result is a
    transposed view of one contiguous buffer whose (column-major) storage is L itself, so
    the adjoint reads it without a copy."""
    b, n = a.shape[0], a.shape[-1]
    prec = _prec(a.dtype)
    key = (b, n, tile, prec)
    h = _batches.get(key)
    if h is None:
        h = ctypes.c_void_p()
        sizes = (ctypes.c_int64 * b)(*([n] * b))
        _capi.check(lib().mtd_batch_create(ctypes.byref(h), b, sizes, None, None, prec))  # library's tiles
        _batches[key] = h
    # symmetric A: its row-major storage is A in column-major order; the factor is written
    # to the column-major lower triangle, i.e. the row-major upper triangle
    w = a.detach().contiguous().clone()
    p, ld = _table(w)
    _capi.check(lib().mtd_batch_factor(h, p, ld, _stream()))
    info = (ctypes.c_int * b)()
    _capi.check(lib().mtd_batch_status(h, info, None))
    bad = [i for i in range(b) if info[i]]
    if bad:
        raise _capi.MtdError(_capi.ERR_NOT_POSITIVE_DEFINITE, info[bad[0]])
    L = w.transpose(-1, -2)
    L.tril_()  # zero what is left of A above the diagonal, in w itself
    return L


def _adjoint(L, gl, tile):
    """Symmetric gradient dLoss/dA for factors L (as _factor returns them) and gradients
    gl = dLoss/dL, both (B, n, n)."""
    b, n = L.shape[0], L.shape[-1]
    prec = _prec(L.dtype)
    key = (b, n, tile, prec)
    h = _adjoints.get(key)
    if h is None:
        h = ctypes.c_void_p()
        sizes = (ctypes.c_int64 * b)(*([n] * b))
        _capi.check(lib().mtd_adjoint_create(ctypes.byref(h), b, sizes, tile, prec))
        _adjoints[key] = h
    lc = L.transpose(-1, -2)
    if not lc.is_contiguous():
        lc = lc.contiguous()
    # gc's storage read column-major is tril(gl); the adjoint turns it into Abar, after which
    # gc (row-major) is Abar^T with zeros below the diagonal
    gc = gl.transpose(-1, -2).contiguous()
    gc.triu_()
    pl, ll = _table(lc)
    pg, lg = _table(gc)
    _capi.check(lib().mtd_adjoint_run(h, pl, ll, pg, lg, _stream()))
    _capi.check(lib().mtd_adjoint_status(h, None))
    grad = gc + gc.transpose(-1, -2)
    grad.mul_(0.5)
    return grad


class CholeskyFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, a, tile, recompute):
        batched = a.dim() == 3
        a3 = a if batched else a.unsqueeze(0)
        L = _factor(a3, tile)
        ctx.tile, ctx.recompute, ctx.batched = tile, recompute, batched
        ctx.save_for_backward(a3 if recompute else L)
        return L if batched else L[0]

    @staticmethod
    def backward(ctx, gl):
        (saved,) = ctx.saved_tensors
        L = _factor(saved, ctx.tile) if ctx.recompute else saved
        g3 = gl if ctx.batched else gl.unsqueeze(0)
        grad = _adjoint(L, g3.to(L.dtype), ctx.tile)
        return (grad if ctx.batched else grad[0]), None, None


def cholesky(a, tile=256, recompute=False):
    """Lower Cholesky factor of the SPD matrix (or stack) ``a`` on the task scheduler,
    differentiable through the blocked adjoint."""
    return CholeskyFunction.apply(a, tile, recompute)


def release_cached():
    """Free the cached task graphs (one per batch shape, tile and precision)."""
    for h in _batches.values():
        lib().mtd_batch_destroy(h)
    for h in _adjoints.values():
        lib().mtd_adjoint_destroy(h)
    _batches.clear()
    _adjoints.clear()
