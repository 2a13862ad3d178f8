"""Runs the reference's own GPU drivers (test and measurement infrastructure, not product).

oracle/ref/Makefile builds the reference's `cholesky_mustard` and `lu_mustard`
(mustard/cholesky_mustard.cu, mustard/lu_mustard.cu) for sm_100a into oracle/_ref/, with
oracle/ref/shim/verify.h in front of include/verify.h (factor dump, O(n^2) probe residual
at large n).  This module runs them on one GPU, one process, and parses their output:

  - the timed loop's `device 0 | r run | time (s): x` lines (cholesky_mustard.cu:470-489,
    lu_mustard.cu:605-624; run 0 is a warm-up the reference's own scripts drop,
    scripts/calc.py:293),
  - `error = ` (the reference's verify, small n) or `probe_residual = ` (the shim, large n),
  - `Result passes verification: `.

Modes: "subgraph" (the device-side scheduler, the path this repository replaces),
"tiled" (one host-launched CUDA graph) and "single" (one cuSOLVER call).

The device-side scheduler (mustard/mustard.h:108-129) launches every task as a
fire-and-forget device graph launch, and CUDA allows a graph at most 120 of those per
execution.  A launch past that limit is lost, its dependency updates never run, and the
scheduler's unbounded spin (mustard/mustard.h:116) never ends: the GPU hangs.  So
"subgraph" runs are refused here unless the task count -- the drivers' own totalNodes
(cholesky_mustard.cu:398-402, lu_mustard.cu:321-326) -- is at most 120: T <= 8 for
Cholesky, T <= 6 for LU.  Those are the tile counts of the reference's published 1-GPU
logs (scripts/results/*/24000/log2_24000_{6,8}_1GPU.log).
"""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
DEVICE_LAUNCH_LIMIT = 120

_RUN = re.compile(r"device\s+\d+\s*\|\s*(\d+)\s+run\s*\|\s*time \(s\):\s*([0-9.eE+-]+)")
_ERR = re.compile(r"^error = ([0-9.eE+-]+|nan|inf)", re.M)
_PROBE = re.compile(r"^probe_residual = ([0-9.eE+-]+|nan|inf)", re.M)
_PASS = re.compile(r"Result passes verification:\s*(\d)")


def binary(kind: str) -> str:
    return os.path.join(REF_BIN, "cholesky_mustard" if kind == "chol" else "lu_mustard")


def available() -> bool:
    return all(os.access(binary(k), os.X_OK) for k in ("chol", "lu"))


def subgraph_tasks(kind: str, t: int) -> int:
    """The drivers' totalNodes for T tiles per dimension."""
    total = t
    for k in range(t):
        for i in range(k + 1, t):
            total += 2 + (t - (i + 1) if kind == "chol" else t - (k + 1))
    return total


def flops(kind: str, n: int) -> float:
    return (2.0 if kind == "lu" else 1.0) * n ** 3 / 3.0


def run(kind: str, n: int, t: int = 1, mode: str = "subgraph", runs: int = 2, sm: int = 20,
        verify: bool = False, dump: str = None, timeout: float = 600.0, extra_env: dict = None) -> dict:
    """One invocation; returns the parsed times (s), residuals and the raw output."""
    if mode not in ("subgraph", "tiled", "single"):
        raise ValueError(mode)
    if mode == "single":
        t = 1
    if n % t:
        raise ValueError("the reference needs T | N")
    if mode == "subgraph" and subgraph_tasks(kind, t) > DEVICE_LAUNCH_LIMIT:
        raise ValueError(f"--subgraph with T={t} has {subgraph_tasks(kind, t)} tasks, above the "
                         f"{DEVICE_LAUNCH_LIMIT} device graph launches the reference's scheduler may make")
    cmd = [binary(kind), f"-n={n}", f"-t={t}", f"-r={runs}", f"--sm={sm}"]
    if mode != "single":
        cmd.append("--" + mode)
    if verify or dump:
        cmd.append("--verify")
    env = dict(os.environ)
    # one PE, no launcher; the symmetric heap holds the matrix in --subgraph mode
    env.setdefault("NVSHMEM_REMOTE_TRANSPORT", "none")
    env.setdefault("NVSHMEM_DISABLE_NVLS", "1")  # no NVLink multicast objects for one PE
    env.setdefault("NVSHMEM_SYMMETRIC_SIZE", str(int(n * n * 8 * 1.1) + (1 << 30)))
    if dump:
        env["MTD_REF_DUMP"] = dump
    if extra_env:
        env.update(extra_env)
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    out = p.stdout + p.stderr
    times = [float(m.group(2)) for m in _RUN.finditer(out)]
    rec = {"kind": kind, "n": n, "t": t, "b": n // t, "mode": mode, "sm": sm, "runs": runs, "rc": p.returncode,
           "times_s": times, "cmd": " ".join(os.path.basename(c) if i == 0 else c for i, c in enumerate(cmd))}
    if mode == "subgraph":
        rec["tasks"] = subgraph_tasks(kind, t)
    kept = times[1:] if len(times) > 1 else times
    if kept:
        rec["mean_s"] = sum(kept) / len(kept)
        rec["best_s"] = min(kept)
        rec["tflops_mean"] = flops(kind, n) / rec["mean_s"] / 1e12
        rec["tflops_best"] = flops(kind, n) / rec["best_s"] / 1e12
    m = _ERR.search(out)
    if m:
        rec["verify_error"] = float(m.group(1))
    m = _PROBE.search(out)
    if m:
        rec["probe_residual"] = float(m.group(1))
    m = _PASS.search(out)
    if m:
        rec["passes"] = m.group(1) == "1"
    if p.returncode != 0 or not times:
        rec["tail"] = out[-2000:]
    return rec


def read_dump(path: str, n: int):
    """The dumped factor as an (n, n) Fortran-ordered array (column-major on disk)."""
    import numpy as np
    return np.fromfile(path, dtype=np.float64, count=n * n).reshape((n, n), order="F")


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="time the reference's own drivers on this GPU")
    ap.add_argument("--kind", choices=["lu", "chol"], required=True)
    ap.add_argument("--n", type=int, default=24000)
    ap.add_argument("--t", type=int, default=6)
    ap.add_argument("--mode", choices=["subgraph", "tiled", "single"], default="subgraph")
    ap.add_argument("--runs", type=int, default=4)
    ap.add_argument("--sm", type=int, default=20)
    ap.add_argument("--verify", action="store_true")
    a = ap.parse_args()
    r = run(a.kind, a.n, a.t, a.mode, a.runs, a.sm, a.verify)
    print(json.dumps(r), flush=True)
