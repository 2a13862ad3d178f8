"""Tile sweep of the FP64 factorisations at N = 24000 (the configuration the reference's
published numbers use).

    python -m mustard_b200.tile_sweep [--n 24000] [--runs 11]
                                      [--tiles 512,768,1024,1536,2048,500,750,1000,1500,2000]

For every tile edge -- the power-of-two-ish set (ragged last tile) and the set that divides
N as the reference requires -- a tiled LU of U[-1,1) + N*I and a tiled Cholesky of
B B^T / N + I run `--runs` times on a fresh device copy of their input; each run is timed
with CUDA events around the launch (as the reference's drivers time theirs), run 0 is
dropped, and the mean and the minimum of the rest are reported with their TFLOP/s (LU
2N^3/3, Cholesky N^3/3).  One JSON line per (kind, tile).
"""
import argparse
import json

import torch

import mustard_b200 as mtd


def sweep(n, tiles, runs, seed):
    a_lu = mtd.colmajor(torch.empty((n, n), dtype=torch.float64, device="cuda"))
    a_ch = mtd.colmajor(torch.empty((n, n), dtype=torch.float64, device="cuda"))
    mtd.generate(a_lu, mtd.GEN_UNIFORM_DIAG, seed=seed)
    mtd.generate(a_ch, mtd.GEN_SPD, seed=seed + 1)
    work = mtd.colmajor(torch.empty((n, n), dtype=torch.float64, device="cuda"))
    s = torch.cuda.current_stream()
    out = []
    for tile in tiles:
        for kind, src, flops in (("lu", a_lu, 2.0 * n ** 3 / 3), ("chol", a_ch, n ** 3 / 3.0)):
            g = mtd.TaskGraph(mtd.KIND_LU if kind == "lu" else mtd.KIND_CHOLESKY, n, tile).build_tiled().finalize()
            times = []
            for _ in range(runs):
                work.copy_(src)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                g.run(work, stream=s, sync=False)
                e1.record(s)
                torch.cuda.synchronize()
                rc, info = g.status()
                if rc:
                    raise mtd.MtdError(rc, info)
                times.append(e0.elapsed_time(e1))
            g.close()
            kept = times[1:]
            mean = sum(kept) / len(kept)
            rec = {"kind": kind, "n": n, "tile": tile, "divides_n": n % tile == 0, "runs": len(kept),
                   "mean_ms": mean, "min_ms": min(kept), "tflops_mean": flops / (mean * 1e-3) / 1e12,
                   "tflops_best": flops / (min(kept) * 1e-3) / 1e12}
            print(json.dumps(rec), flush=True)
            out.append(rec)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=24000)
    ap.add_argument("--runs", type=int, default=11)
    ap.add_argument("--tiles", default="512,768,1024,1536,2048,500,750,1000,1500,2000")
    ap.add_argument("--seed", type=int, default=2024)
    args = ap.parse_args()
    if args.runs < 2:
        ap.error("--runs must be at least 2 (run 0 is dropped)")
    sweep(args.n, [int(t) for t in args.tiles.split(",")], args.runs, args.seed)


if __name__ == "__main__":
    main()
