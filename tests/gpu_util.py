"""Helpers shared by the GPU tests: column-major transfers and the parity metric."""
import numpy as np


def to_dev(a):
    """numpy (n, n) -> column-major float64 CUDA tensor with the same entries."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)).cuda().t()


def from_dev(t):
    """column-major CUDA tensor -> numpy (n, n) in Fortran order."""
    return np.asfortranarray(t.t().contiguous().cpu().numpy().T)


def rel_diff(x, y):
    """max |x - y| / max |y| (the factor parity metric; FP64 bar 1e-12)."""
    return float(np.abs(np.asarray(x) - np.asarray(y)).max() / max(np.abs(np.asarray(y)).max(), 1e-300))


def device_probe_residual(a, f, kind, probes=8, seed=7):
    """||(A - L U) X||_F / ||A X||_F over `probes` random columns, on the device in FP64:
    a is the input and f the in-place factor, both column-major CUDA tensors.  LU: unit
    lower L below the diagonal, U on and above it; Cholesky: L = lower triangle of f.  An
    O(n^2) check that stays cheap at n = 24000 (torch matmuls serve only as the checker)."""
    import torch
    n = a.shape[0]
    gen = torch.Generator(device=a.device).manual_seed(seed)
    x = torch.randn(n, probes, dtype=torch.float64, device=a.device, generator=gen)
    ax = a @ x
    if kind == "chol":
        l = torch.tril(f)
        r = ax - l @ (l.t() @ x)
    else:
        u = torch.triu(f)
        ux = u @ x
        del u
        r = ax - (torch.tril(f, -1) @ ux + ux)
    return float(torch.linalg.norm(r) / torch.linalg.norm(ax))
