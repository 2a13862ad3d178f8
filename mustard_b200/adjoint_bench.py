"""Cholesky forward + adjoint benchmark (one B200).

    python -m mustard_b200.adjoint_bench [--batch 64] [--n 2048] [--dtypes float64,float32]

A = K + 0.1 I with K the RBF kernel (lengthscale 1) over X in R^{n x 8}, X and y i.i.d.
N(0, 1) (seeded, built on the device); loss = 0.5 y^T A^-1 y + sum(log diag L).  For each
dtype and for the store / recompute variants of the autograd function: device time of the
forward factorisation (one merged task graph for the whole batch), of the backward pass
(the blocked adjoint's reverse task graph, plus the re-factorisation when recomputing),
and the peak memory allocated by torch over forward + backward; the gradient is compared
with torch.linalg.cholesky's (timed the same way, for reference).  One JSON line each.
Rates: forward n^3/3, adjoint 2 n^3/3 flop per matrix.
"""
import argparse
import json

import torch

from mustard_b200 import autograd


def rbf_batch(batch, n, d, seed, dtype):
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn((batch, n, d), generator=g, device="cuda", dtype=torch.float64)
    y = torch.randn((batch, n), generator=g, device="cuda", dtype=torch.float64)
    sq = (x * x).sum(-1)
    d2 = (sq.unsqueeze(-1) + sq.unsqueeze(-2) - 2.0 * x @ x.transpose(-1, -2)).clamp_min(0.0)
    a = torch.exp(-0.5 * d2) + 0.1 * torch.eye(n, device="cuda", dtype=torch.float64)
    return a.to(dtype), y.to(dtype)


def gp_loss(L, y):
    z = torch.linalg.solve_triangular(L, y.unsqueeze(-1), upper=False).squeeze(-1)
    return 0.5 * (z * z).sum() + torch.log(torch.diagonal(L, dim1=-2, dim2=-1)).sum()


def linear_loss(L, w):
    """sum(L * w): nothing downstream keeps L, so what the Cholesky function itself keeps
    between the passes shows in the held memory."""
    return (L * w).sum()


def timed_pass(a, y, chol, loss_fn):
    """(forward ms, backward ms, peak bytes, bytes held between the passes, grad) of one
    forward + backward; memory counted above what the caller already holds (A, y)."""
    a = a.detach().clone().requires_grad_(True)
    torch.cuda.synchronize()
    base = torch.cuda.memory_allocated()
    torch.cuda.reset_peak_memory_stats()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record()
    L = chol(a)
    e[1].record()
    loss = loss_fn(L, y)
    del L  # whatever autograd keeps stays alive
    torch.cuda.synchronize()
    held = torch.cuda.memory_allocated() - base
    e[2].record()
    loss.backward()
    e[3].record()
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated() - base
    return e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3]), peak, held, a.grad


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--tile", type=int, default=256)
    ap.add_argument("--dtypes", default="float64,float32")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--losses", default="gp,linear")
    args = ap.parse_args()
    b, n = args.batch, args.n
    f_fwd, f_adj = b * n ** 3 / 3.0, b * 2.0 * n ** 3 / 3.0
    for dt_name in args.dtypes.split(","):
        dt = getattr(torch, dt_name)
        a, y = rbf_batch(b, n, 8, args.seed, dt)
        variants = [("store", lambda x: autograd.cholesky(x, tile=args.tile, recompute=False)),
                    ("recompute", lambda x: autograd.cholesky(x, tile=args.tile, recompute=True)),
                    ("torch.linalg.cholesky", torch.linalg.cholesky)]
        for loss_name in args.losses.split(","):
            if loss_name == "gp":
                loss_fn, aux = gp_loss, y
            else:
                g = torch.Generator(device="cuda").manual_seed(args.seed + 7)
                aux = torch.randn((b, n, n), generator=g, device="cuda", dtype=torch.float64).tril().to(dt)
                loss_fn = linear_loss
            grads = {}
            for name, chol in variants:
                best = None
                for _ in range(args.reps):
                    fwd, bwd, peak, held, grad = timed_pass(a, aux, chol, loss_fn)
                    if best is None or fwd + bwd < best[0] + best[1]:
                        best = (fwd, bwd, peak, held)
                grads[name] = grad
                rec = {"bench": "cholesky_adjoint", "loss": loss_name, "variant": name, "dtype": dt_name,
                       "batch": b, "n": n, "tile": args.tile, "forward_ms": best[0], "backward_ms": best[1],
                       "peak_mem_mb": best[2] / 2 ** 20, "held_between_passes_mb": best[3] / 2 ** 20,
                       "forward_tflops": f_fwd / (best[0] * 1e-3) / 1e12}
                if name != "torch.linalg.cholesky":
                    # adjoint flop count over the whole backward (loss backward included, and the
                    # second factorisation when recomputing)
                    rec["backward_adjoint_tflops"] = f_adj / (best[1] * 1e-3) / 1e12
                print(json.dumps(rec), flush=True)
            ref = grads["torch.linalg.cholesky"].double()
            for name in ("store", "recompute"):
                rel = ((grads[name].double() - ref).abs().max() / ref.abs().max()).item()
                print(json.dumps({"bench": "cholesky_adjoint", "loss": loss_name,
                                  "check": f"{name} vs torch.linalg.cholesky grad", "dtype": dt_name,
                                  "max_rel_diff": rel}), flush=True)
            del aux, grads
        del a, y
        autograd.release_cached()
        torch.cuda.empty_cache()


if __name__ == "__main__":
    main()
