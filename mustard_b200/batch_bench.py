"""Batched Cholesky solves benchmark (one B200).

    python -m mustard_b200.batch_bench [--count 4096] [--precs fp64,fp32] [--reps 3]

`count` independent SPD matrices, N drawn uniformly from {32, 64, ..., 1024} (seeded), each
B B^T / N + I with B = U[-1, 1) (as the reference's N=600 case), with 1 to 16 right-hand
sides each (uniform count, entries N(0, 1)).  Per precision (fp64: FP64 factor and one
solve; fp32: FP32 storage with split-TF32 products, then FP64 iterative refinement to
normwise backward error 1e-13):
  autotune   per-size tile and nested tile from mtd_batch_autotune (wall time reported);
  factor     ONE persistent launch for the whole batch, captured in a CUDA graph and
             replayed (inputs restored by device copies outside the timed replay):
             aggregate TFLOP/s (sum n^3/3 over device time) and p50 / p99 per-matrix
             latency (completion of the matrix's last task after the launch's first work,
             on the device clock);
  solve      factor replay + per-matrix solves, time-to-solution and max backward error;
  one launch factor AND solve (+ refinement; + conversion from FP64 for fp32) as ONE
             persistent launch (mtd_batch_factor_solve), captured in a CUDA graph and
             replayed: device time, wall time-to-solution, latencies, backward errors; first
             the schedule tuner times the twelve CTA-to-task schedules and keeps the fastest;
  defaults   the same factor launch with the library's default tiles (what tuning buys);
  torch      torch.linalg.cholesky + cholesky_solve per size group, for reference.
One JSON line per measurement.
"""
import argparse
import json
import time

import numpy as np
import torch

import mustard_b200 as mtd

PRECS = {"fp64": (mtd.PREC_FP64, torch.float64), "fp32": (mtd.PREC_FP32, torch.float32)}


def make_batch(count, seed):
    rng = np.random.default_rng(seed)
    sizes = [int(32 * v) for v in rng.integers(1, 33, size=count)]
    nrhs = [int(v) for v in rng.integers(1, 17, size=count)]
    g = torch.Generator(device="cuda").manual_seed(seed)
    groups = {}
    for n in sorted(set(sizes)):
        idx = [i for i, v in enumerate(sizes) if v == n]
        b = torch.rand((len(idx), n, n), generator=g, device="cuda", dtype=torch.float64) * 2.0 - 1.0
        a = b @ b.transpose(-1, -2) / n + torch.eye(n, device="cuda", dtype=torch.float64)
        groups[n] = (idx, a)
    rhs = [torch.randn((k, n), generator=g, device="cuda", dtype=torch.float64).t() for n, k in zip(sizes, nrhs)]
    return sizes, nrhs, groups, rhs


def views(groups, count, dtype=None):
    """Per-matrix column-major views (symmetric: a row-major matrix is its own transpose)."""
    out = [None] * count
    for n, (idx, a) in groups.items():
        src = a if dtype is None else a.to(dtype)
        for j, i in enumerate(idx):
            out[i] = src[j].t()
    return out


def one_launch(b, pname, prec, work, restore, rhs, a64, groups, base, flops_s, reps):
    """Factor + solve (+ IR) as ONE persistent launch: tune the CTA-to-task schedule, capture
    the launch in a CUDA graph and time its replays."""
    fp64 = prec == mtd.PREC_FP64
    kw = dict(a64=a64, method=mtd.REFINE_NONE) if fp64 else \
        dict(a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=30)
    xs = [torch.zeros_like(r) for r in rhs]
    src = views({n: (idx, a) for n, (idx, a) in groups.items()}, len(rhs)) if fp64 else None
    t0 = time.perf_counter()
    sched, trial = b.tune_schedule(work, rhs, xs, source=src, reps=2, **kw)
    tune_s = time.perf_counter() - t0
    names = {0: "input order", 1: "largest first", 2: "smallest first"}
    label = {s_: names[s_ & 3] + (", solves late" if s_ & mtd.BATCH_SOLVE_LATE else ", solves early")
             + (", two matrices per solve task" if s_ & mtd.BATCH_SOLVE_PAIRS else "") for s_ in trial}
    print(json.dumps(dict(base, prec=pname, step="schedule tuner", wall_s=tune_s, chosen=label[sched],
                          device_ms={label[k]: v for k, v in trial.items()})), flush=True)
    restore()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            b.factor_solve(work, rhs, xs, stream=s, **kw)
    best = None
    for _ in range(reps):
        restore()
        for x in xs:
            x.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        ms = e0.elapsed_time(e1)
        rc, info, lat, berr, its, st = b.solve_status()
        assert rc == 0 and not any(info), rc
        if best is None or ms < best[0]:
            best = (ms, wall, lat, st)
    ms, wall, lat, st = best
    lat = np.asarray(lat)
    print(json.dumps(dict(base, prec=pname, step="factor+solve", launches="ONE graph-captured persistent launch",
                          schedule=label[sched], device_ms=ms, time_to_solution_ms=wall,
                          tflops=flops_s / (wall * 1e-3) / 1e12, iterations=st["iterations"],
                          converged=st["converged_count"], max_backward_error=st["max_backward_error"],
                          latency_p50_ms=float(np.percentile(lat, 50)), latency_p99_ms=float(np.percentile(lat, 99)))),
          flush=True)
    del g


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--precs", default="fp64,fp32")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--tune-table", default=None,
                    help="JSON table of autotuner choices to reuse and extend (mustard_b200.tune_table)")
    args = ap.parse_args()
    sizes, nrhs, groups, rhs = make_batch(args.count, args.seed)
    count = args.count
    flops_f = sum(n ** 3 / 3.0 for n in sizes)
    flops_s = flops_f + sum(2.0 * n * n * k for n, k in zip(sizes, nrhs))
    a64 = views(groups, count)
    base = {"bench": "batched_cholesky", "count": count, "sizes": "U{32..1024 step 32}", "rhs": "U{1..16}",
            "total_factor_gflop": flops_f / 1e9}
    for pname in args.precs.split(","):
        prec, dt = PRECS[pname]
        # working copies of the factor inputs, one contiguous block per size group
        work_groups = {n: (idx, a.to(dt).clone()) for n, (idx, a) in groups.items()}
        pristine = {n: a.to(dt).clone() for n, (idx, a) in groups.items()}
        work = views(work_groups, count)

        def restore():
            for n, (idx, w) in work_groups.items():
                w.copy_(pristine[n])

        tiles, nests, tune_ms = mtd.batch_autotune(sizes, prec, table=args.tune_table)
        chosen = {n: (tiles[sizes.index(n)], nests[sizes.index(n)]) for n in sorted(set(sizes))}
        print(json.dumps(dict(base, prec=pname, step="autotune", wall_ms=tune_ms,
                              choice={str(n): list(v) for n, v in chosen.items()})), flush=True)

        for label, tl, ns in (("autotuned", tiles, nests), ("defaults", None, None)):
            b = mtd.Batch(sizes, tiles=tl, nests=ns, prec=prec)
            restore()
            b.factor(work)  # warm-up, outside the capture
            rc, info = b.status()
            assert rc == 0 and not any(info), info
            s = torch.cuda.Stream()
            g = torch.cuda.CUDAGraph()
            restore()
            torch.cuda.synchronize()
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    b.factor(work, stream=s)
            best, lat = None, None
            for _ in range(args.reps):
                restore()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                g.replay()
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                rc, info, lt = b.status(latencies=True)
                assert rc == 0 and not any(info)
                if best is None or ms < best:
                    best, lat = ms, lt
            lat = np.asarray(lat)
            rec = dict(base, prec=pname, step="factor", tiles=label, launches="1 graph-captured persistent launch",
                       device_ms=best, tflops=flops_f / (best * 1e-3) / 1e12,
                       latency_p50_ms=float(np.percentile(lat, 50)), latency_p99_ms=float(np.percentile(lat, 99)),
                       latency_max_ms=float(lat.max()), tasks=b.num_tasks)
            print(json.dumps(rec), flush=True)
            if label == "autotuned":
                # time-to-solution: factor replay + solves (+ FP64 refinement for fp32)
                xs = [torch.zeros_like(r) for r in rhs]
                best_t, st = None, None
                for _ in range(args.reps):
                    restore()
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    g.replay()
                    if prec == mtd.PREC_FP64:
                        s_ = b.solve(work, rhs, xs, a64=a64, method=mtd.REFINE_NONE)
                    else:
                        s_ = b.solve(work, rhs, xs, a64=a64, method=mtd.REFINE_IR, tol=1e-13, max_iter=30)
                    torch.cuda.synchronize()
                    t = (time.perf_counter() - t0) * 1e3
                    if best_t is None or t < best_t:
                        best_t, st = t, s_
                print(json.dumps(dict(base, prec=pname, step="factor+solve", launches="factor graph + solve launches",
                                      time_to_solution_ms=best_t,
                                      tflops=flops_s / (best_t * 1e-3) / 1e12, iterations=st["iterations"],
                                      converged=st["converged_count"], max_backward_error=st["max_backward_error"])),
                      flush=True)
                one_launch(b, pname, prec, work, restore, rhs, a64, groups, base, flops_s, args.reps)
            del g
            b.close()
        del work_groups, pristine, work
        torch.cuda.empty_cache()

    # reference point: torch.linalg.cholesky + cholesky_solve, one batched call per size group
    # (right-hand sides zero-padded to 16 columns inside a group)
    padded = {}
    for n, (idx, a) in groups.items():
        bb = torch.zeros((len(idx), n, 16), device="cuda", dtype=torch.float64)
        for j, i in enumerate(idx):
            bb[j, :, : nrhs[i]] = rhs[i]
        padded[n] = bb
    best = None
    for _ in range(args.reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for n, (idx, a) in groups.items():
            torch.cholesky_solve(padded[n], torch.linalg.cholesky(a))
        torch.cuda.synchronize()
        t = (time.perf_counter() - t0) * 1e3
        best = t if best is None else min(best, t)
    print(json.dumps(dict(base, prec="fp64", step="torch.linalg.cholesky+cholesky_solve, one call per size group",
                          time_to_solution_ms=best, tflops=flops_s / (best * 1e-3) / 1e12)), flush=True)


if __name__ == "__main__":
    main()
