"""Residual checks of a finished factorisation on the device (the large-n counterpart of
the reference's --verify, include/verify.h:17-129, whose O(n^3) host product is only
practical for small n).

``probe_residual(a, f, kind)`` = ||(A - L U) X||_F / ||A X||_F over a few random columns X,
in FP64 on the device: O(n^2) work, so it stays cheap at n = 24000.  ``a`` is the input and
``f`` the in-place factor, both column-major CUDA float64 tensors; LU: unit-lower L below
the diagonal and U on and above it; Cholesky: L = lower triangle of ``f``.
"""


def probe_residual(a, f, kind, probes=8, seed=7):
    import torch
    if kind not in ("lu", "chol"):
        raise ValueError(kind)
    n = a.shape[0]
    gen = torch.Generator(device=a.device).manual_seed(seed)
    x = torch.randn(n, probes, dtype=torch.float64, device=a.device, generator=gen)
    ax = a @ x
    if kind == "chol":
        l = torch.tril(f)
        r = ax - l @ (l.t() @ x)
        del l
    else:
        u = torch.triu(f)
        ux = u @ x
        del u
        r = ax - (torch.tril(f, -1) @ ux + ux)
    return float(torch.linalg.norm(r) / torch.linalg.norm(ax))
