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
