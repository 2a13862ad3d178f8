"""Mixed-precision factor + FP64 refinement against the plain FP64 solve (one B200).

    python -m mustard_b200.mixed_bench [--n 32768] [--tile 1536] [--kappas 1e2,1e5,1e8]
                                       [--nrhs 1,16] [--out results.jsonl]

For each condition number kappa: A = B B^T / n + alpha I (B = U[-1,1), alpha = (4/3)/(kappa-1),
built on the device by the seeded generator), right-hand sides i.i.d. N(0,1).  The plain FP64
time-to-solution (FP64 tiled Cholesky + one FP64 solve) is compared with each
low-precision variant: TF32, BF16-update (tcgen05 kind::f16 updates, TF32 panels) or
FP32-accurate (split TF32) factor of A + shift*I followed by
IR or GMRES-IR to a normwise backward error of 1e-13.  One JSON line per run: iterations,
backward error (FP64, on the device), forward error against the FP64 solution, times, and
the FP64-equivalent rate (n^3/3 + 2 n^2 nrhs) / time-to-solution.
"""
import argparse
import json
import time

import torch

import mustard_b200 as mtd

PREC_NAMES = {mtd.PREC_FP64: "fp64", mtd.PREC_TF32: "tf32", mtd.PREC_FP32: "fp32(3xtf32)", mtd.PREC_BF16: "bf16"}
METHOD_NAMES = {mtd.REFINE_NONE: "none", mtd.REFINE_IR: "ir", mtd.REFINE_GMRES_IR: "gmres-ir"}
UNIT_ROUNDOFF = {mtd.PREC_TF32: 2.0 ** -11, mtd.PREC_FP32: 2.0 ** -24, mtd.PREC_BF16: 2.0 ** -8}


def colmajor(n, k):
    return torch.empty((k, n), dtype=torch.float64, device="cuda").t()


def time_to_solution(a, b, n, tile, prec, method, shift, tol, max_iter):
    s = mtd.SpdSolver(n, tile, prec)
    x = colmajor(n, b.shape[1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    try:
        s.factor(a, shift=shift)
    except mtd.MtdError as e:
        s.close()
        return None, {"factor_error": str(e)}
    st = s.solve(b, x, method=method, tol=tol, max_iter=max_iter)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    s.close()
    return x, dict(st, time_to_solution_ms=(t1 - t0) * 1e3)


def run_case(n, tile, kappa, nrhs, seed, variants, tol, max_iter, reps):
    a = colmajor(n, n)
    mtd.generate(a, mtd.GEN_SPD, seed=seed, alpha=(4.0 / 3.0) / (kappa - 1.0))
    g = torch.Generator(device="cuda").manual_seed(seed + 1)
    b = torch.randn((nrhs, n), dtype=torch.float64, device="cuda", generator=g).t()
    maxdiag = float(a.diagonal().max())
    out = []
    # plain FP64: best of reps
    best, x64 = None, None
    for _ in range(reps):
        x, st = time_to_solution(a, b, n, tile, mtd.PREC_FP64, mtd.REFINE_NONE, 0.0, tol, 1)
        if best is None or st["time_to_solution_ms"] < best["time_to_solution_ms"]:
            best, x64 = st, x
    flops = n ** 3 / 3.0 + 2.0 * n * n * nrhs
    base = dict(best, n=n, tile=tile, kappa=kappa, nrhs=nrhs, prec="fp64", method="none", shift=0.0,
                fp64_equiv_tflops=flops / (best["time_to_solution_ms"] * 1e-3) / 1e12, ratio_vs_fp64=1.0)
    out.append(base)
    for prec, method, shift_c in variants:
        shift = shift_c * UNIT_ROUNDOFF[prec] * maxdiag
        bestv, xv = None, None
        for _ in range(reps):
            x, st = time_to_solution(a, b, n, tile, prec, method, shift, tol, max_iter)
            if x is None:
                bestv = st
                break
            if bestv is None or st["time_to_solution_ms"] < bestv["time_to_solution_ms"]:
                bestv, xv = st, x
        rec = dict(bestv, n=n, tile=tile, kappa=kappa, nrhs=nrhs, prec=PREC_NAMES[prec], method=METHOD_NAMES[method],
                   shift=shift)
        if xv is not None:
            ferr = ((xv - x64).abs().amax(dim=0) / x64.abs().amax(dim=0)).max().item()
            rec["forward_error_vs_fp64"] = ferr
            rec["fp64_equiv_tflops"] = flops / (bestv["time_to_solution_ms"] * 1e-3) / 1e12
            rec["ratio_vs_fp64"] = bestv["time_to_solution_ms"] / base["time_to_solution_ms"]
        out.append(rec)
    del a, b
    torch.cuda.empty_cache()
    return out


DEFAULT_VARIANTS = [
    (mtd.PREC_TF32, mtd.REFINE_IR, 0.0),
    (mtd.PREC_TF32, mtd.REFINE_GMRES_IR, 0.0),
    (mtd.PREC_BF16, mtd.REFINE_IR, 0.0),
    (mtd.PREC_BF16, mtd.REFINE_GMRES_IR, 0.0),
    (mtd.PREC_FP32, mtd.REFINE_IR, 0.0),
    (mtd.PREC_FP32, mtd.REFINE_GMRES_IR, 2.0),
]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=32768)
    ap.add_argument("--tile", type=int, default=1536)
    ap.add_argument("--kappas", default="1e2,1e5,1e8")
    ap.add_argument("--nrhs", default="1,16")
    ap.add_argument("--tol", type=float, default=1e-13)
    ap.add_argument("--max-iter", type=int, default=30)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    fh = open(args.out, "a") if args.out else None
    for kappa in [float(k) for k in args.kappas.split(",")]:
        for nrhs in [int(k) for k in args.nrhs.split(",")]:
            variants = [v for v in DEFAULT_VARIANTS if not (v[1] == mtd.REFINE_GMRES_IR and nrhs != 1)]
            for rec in run_case(args.n, args.tile, kappa, nrhs, args.seed, variants, args.tol, args.max_iter,
                                args.reps):
                line = json.dumps(rec)
                print(line, flush=True)
                if fh:
                    fh.write(line + "\n")
    if fh:
        fh.close()


if __name__ == "__main__":
    main()
