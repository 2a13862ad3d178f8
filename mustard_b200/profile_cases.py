"""Small, self-contained workloads for ncu captures of the persistent kernel.

    python -m mustard_b200.profile_cases gemm  --n 6144 --tile 768
        one Cholesky update step only: every GEMM_NT(j, i) of step k = 0 for j > i >= 1,
        all independent, so the capture shows the GEMM work items and the scheduler
        without the critical path
    python -m mustard_b200.profile_cases chol --n 6144 --tile 512
    python -m mustard_b200.profile_cases lu   --n 6144 --tile 512
        a whole tiled factorisation
    python -m mustard_b200.profile_cases lupiv --n 8192 --tile 128
        LU with partial pivoting (mtd_lupiv) of a U[-1, 1) matrix (no diagonal boost, so most
        rows are interchanged)
    python -m mustard_b200.profile_cases batch --n 512 --prec fp64
        the batched factor-and-solve launch (mtd_batch_factor_solve) of `--n` matrices with
        sizes and right-hand sides drawn as config 3 draws them (batch_bench.make_batch),
        library default tiles; fp32: conversion + split-TF32 factor + FP64 refinement
    python -m mustard_b200.profile_cases gemm --n 8192 --tile 1024 --prec tf32
        the same cases on a float32 matrix with TF32 tensor-core products (tcgen05 GEMM /
        SYRK items fed by TMA; Cholesky and the GEMM-only step only); --prec bf16 (BF16
        updates) and --prec fp32 (FP32-accurate: three TF32 passes) likewise

Each case runs `--runs` launches (default 2: the first is the one to capture with
`-c 1`), checks the run status, and prints the device time of the last launch.  With
`--trace` the runs record per-item timestamps and the line adds, per tile operation, the
items, median and summed item time, the busy fraction (time inside items over SMs x span)
and the critical path's composition (mustard_b200.trace_analysis); `--trace-out FILE`
also writes the records, task spans and critical path as JSON.
Inputs are the seeded generators of the benchmark (larger than L2 from n = 4096).
"""
import argparse
import json

import torch

import mustard_b200 as mtd


OP_NAMES = {mtd.OP_POTRF: "POTRF", mtd.OP_TRSM_RLT: "TRSM_RLT", mtd.OP_SYRK_LN: "SYRK_LN",
            mtd.OP_GEMM_NT: "GEMM_NT", mtd.OP_GETRF: "GETRF", mtd.OP_TRSM_LLNU: "TRSM_LLNU",
            mtd.OP_TRSM_RUN: "TRSM_RUN", mtd.OP_GEMM_NN: "GEMM_NN"}


def op_breakdown(g):
    """Per-operation item statistics of the last traced run."""
    tr = g.trace()
    if not tr:
        return {}
    t0 = min(r[0] for r in tr)
    t1 = max(r[1] for r in tr)
    per = {}
    for s, e, _sm, task, _item in tr:
        per.setdefault(OP_NAMES.get(g.device_task_op(task), "other"), []).append((e - s) * 1e-3)
    total = sum(sum(v) for v in per.values())
    ops = {}
    for name, d in sorted(per.items()):
        d.sort()
        ops[name] = {"items": len(d), "median_us": d[len(d) // 2], "sum_ms": sum(d) * 1e-3,
                     "share": sum(d) / total}
    # gaps between consecutive items of one CTA: completing one item and claiming the next
    # (or waiting for work)
    by_sm = {}
    for s, e, sm, _task, _item in tr:
        by_sm.setdefault(sm, []).append((s, e))
    gaps = []
    for v in by_sm.values():
        v.sort()
        gaps += [(b[0] - a[1]) * 1e-3 for a, b in zip(v, v[1:])]
    gaps.sort()
    gap = {"count": len(gaps), "median_us": gaps[len(gaps) // 2] if gaps else 0.0,
           "p90_us": gaps[(9 * len(gaps)) // 10] if gaps else 0.0, "sum_ms": sum(gaps) * 1e-3}
    from mustard_b200 import trace_analysis
    return {"span_ms": (t1 - t0) * 1e-6, "busy": trace_analysis.busy_fraction(tr),
            "busy_by_twentieth": [round(v, 3) for v in trace_analysis.busy_profile(tr, 20)], "ops": ops, "gaps": gap}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["gemm", "chol", "lu", "lupiv", "batch"])
    ap.add_argument("--n", type=int, default=6144)
    ap.add_argument("--tile", type=int, default=768)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--prec", choices=["fp64", "tf32", "bf16", "fp32"], default="fp64")
    ap.add_argument("--nest", type=int, default=None, help="nested sub-tile edge of the diagonal factorisations")
    ap.add_argument("--first", type=int, default=0, help="a narrower first tile of this edge")
    ap.add_argument("--last", type=int, default=0, help="the end of the matrix in tiles of at most this edge")
    ap.add_argument("--trace", action="store_true", help="per-operation item-time breakdown")
    ap.add_argument("--trace-out", default=None,
                    help="also write the records, task spans and critical path to this JSON file")
    args = ap.parse_args()
    if args.prec != "fp64" and args.case == "lu":
        ap.error("the low-precision paths factor SPD matrices only (chol, gemm)")
    n, b = args.n, args.tile
    t = (n + b - 1) // b
    if args.case == "lupiv":
        return run_pivoted(n, b, args.runs)
    if args.case == "batch":
        return run_batch(n, args.prec, args.runs)
    a = torch.empty((n, n), dtype=torch.float64, device="cuda").t()
    edges = tile_edges(n, b, args.first, args.last) if (args.first or args.last) else None
    if args.case == "lu":
        mtd.generate(a, mtd.GEN_UNIFORM_DIAG, seed=3)
        g = mtd.TaskGraph(mtd.KIND_LU, n, b)
        if edges:
            g.set_tile_edges(edges)
        g.build_tiled()
        flops = 2.0 * n ** 3 / 3
    elif args.case == "chol":
        mtd.generate(a, mtd.GEN_SPD, seed=3)
        g = mtd.TaskGraph(mtd.KIND_CHOLESKY, n, b)
        if edges:
            g.set_tile_edges(edges)
        g.build_tiled()
        flops = n ** 3 / 3.0
    else:
        mtd.generate(a, mtd.GEN_SPD, seed=3)
        g = mtd.TaskGraph(mtd.KIND_CUSTOM, n, b)
        flops = 0.0
        ext = [min(b, n - i * b) for i in range(t)]
        for i in range(1, t):
            for j in range(i + 1, t):
                g.add_task(mtd.OP_GEMM_NT, (j, i), [(j, i), (j, 0), (i, 0)])
                flops += 2.0 * ext[j] * ext[i] * ext[0]
    if args.prec != "fp64":
        g.set_precision({"tf32": mtd.PREC_TF32, "bf16": mtd.PREC_BF16, "fp32": mtd.PREC_FP32}[args.prec])
        a = a.t().contiguous().float().t()
    if args.nest is not None:
        g.set_nest(args.nest)
    if args.trace_out:
        args.trace = True
    if args.trace:
        g.set_trace(True)
    g.finalize()
    src = a.clone()
    s = torch.cuda.current_stream()
    ms = 0.0
    for _ in range(args.runs):
        a.copy_(src)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        if args.prec != "fp64":
            g.run_f32(a, stream=s, sync=False)
        else:
            g.run(a, stream=s, sync=False)
        e1.record(s)
        torch.cuda.synchronize()
        rc, info = g.status()
        if rc:
            raise mtd.MtdError(rc, info)
        ms = e0.elapsed_time(e1)
    rec = {"case": args.case, "prec": args.prec, "n": n, "tile": b, "tasks": g.num_tasks, "ms": ms,
           "tflops": flops / (ms * 1e-3) / 1e12}
    if args.trace:
        rec.update(op_breakdown(g))
        from mustard_b200 import trace_analysis
        recs = g.trace()
        rec["critical_path"] = (trace_analysis.dump_json(args.trace_out, g, recs) if args.trace_out
                                else trace_analysis.summary(g, recs))["critical_path"]
    print(json.dumps(rec))
    g.close()


def tile_edges(n, b, first, last):
    """0, first, then b-wide tiles while at least `last` elements (or one b tile) remain, the
    rest in near-equal tiles of at most `last` (multiples of 64)."""
    edges = [0]
    if first:
        edges.append(first)
    tail = last or b
    while n - edges[-1] > b + tail:
        edges.append(edges[-1] + b)
    rest = n - edges[-1]
    pieces = max(1, -(-rest // tail))
    for i in range(1, pieces):
        edges.append(edges[-1] + ((rest // pieces) // 64) * 64)
    edges.append(n)
    return edges


def run_batch(count, prec, runs):
    from mustard_b200 import batch_bench
    if prec not in ("fp64", "fp32"):
        raise SystemExit("batch: --prec fp64 or fp32")
    sizes, nrhs, groups, rhs = batch_bench.make_batch(count, 7)
    a64 = batch_bench.views(groups, count)
    p, dt = batch_bench.PRECS[prec]
    work_groups = {k: (idx, a.to(dt).clone()) for k, (idx, a) in groups.items()}
    work = batch_bench.views(work_groups, count)
    xs = [torch.zeros_like(r) for r in rhs]
    b = mtd.Batch(sizes, prec=p)
    kw = dict(method=mtd.REFINE_NONE) if prec == "fp64" else dict(method=mtd.REFINE_IR, tol=1e-13, max_iter=30)
    s = torch.cuda.current_stream()
    ms = 0.0
    for _ in range(runs):
        for k, (idx, w) in work_groups.items():
            w.copy_(groups[k][1].to(dt))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        b.factor_solve(work, rhs, xs, a64=a64, stream=s, **kw)
        e1.record(s)
        rc, info, lat, berr, its, st = b.solve_status()
        if rc:
            raise mtd.MtdError(rc)
        ms = e0.elapsed_time(e1)
    flops = sum(k ** 3 / 3.0 for k in sizes)
    print(json.dumps({"case": "batch", "prec": prec, "count": count, "tasks": b.num_tasks, "ms": ms,
                      "tflops": flops / (ms * 1e-3) / 1e12, "max_backward_error": st["max_backward_error"],
                      "converged": st["converged_count"]}))
    b.close()


def run_pivoted(n, b, runs):
    gen = torch.Generator(device="cuda").manual_seed(3)
    src = (torch.rand((n, n), generator=gen, dtype=torch.float64, device="cuda") * 2.0 - 1.0).t()
    a = torch.empty_like(src)
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    h = mtd.PivotedLU(n, b)
    s = torch.cuda.current_stream()
    ms = 0.0
    for _ in range(runs):
        a.copy_(src)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        h.run(a, ipiv, stream=s)
        e1.record(s)
        info = h.status()
        ms = e0.elapsed_time(e1)
    swapped = int((ipiv.cpu() != torch.arange(1, n + 1, dtype=torch.int32)).sum())
    print(json.dumps({"case": "lupiv", "prec": "fp64", "n": n, "tile": b, "tasks": h.num_tasks, "ms": ms,
                      "tflops": 2.0 * n ** 3 / 3 / (ms * 1e-3) / 1e12, "info": info, "rows_interchanged": swapped}))
    h.close()


if __name__ == "__main__":
    main()
