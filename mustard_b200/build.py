"""Build recipe: nvcc for sm_100a -> mustard_b200/lib/libmustard_b200.so and the
lu_mustard / cholesky_mustard command-line drivers (mustard_b200/bin/)."""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
CLI = os.path.join(PKG, "cli")
LIB_DIR = os.path.join(PKG, "lib")
BIN_DIR = os.path.join(PKG, "bin")
BUILD_DIR = os.path.join(PKG, "_build")
LIB = os.path.join(LIB_DIR, "libmustard_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
# engine-shape overrides for tuning builds, e.g. MTD_NVCC_EXTRA="-DMTD_PANEL_STAGES=4"
CUDA_FLAGS += os.environ.get("MTD_NVCC_EXTRA", "").split()

LIB_SOURCES = ["runtime.cu", "batch_run.cu", "gen.cu", "dag.cpp", "solver.cu", "batch.cu", "adjoint.cu", "lupiv.cu"]
CLI_PROGRAMS = {"lu_mustard": "lu_mustard.cpp", "cholesky_mustard": "cholesky_mustard.cpp"}
PROBES = {"dmma_probe": os.path.join(PKG, "probe", "dmma_probe.cu")}  # measurement tools


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    out = []
    for d in (CSRC, CLI, os.path.join(ROOT, "include")):
        if os.path.isdir(d):
            out += [os.path.join(d, f) for f in os.listdir(d)
                    if f.endswith((".cu", ".cuh", ".cpp", ".hpp", ".h"))]
    return out


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    os.makedirs(BIN_DIR, exist_ok=True)
    deps = _deps()
    objs, jobs = [], []
    for src in LIB_SOURCES:
        obj = os.path.join(BUILD_DIR, src + ".o")
        objs.append(obj)
        if _newer(obj, deps) or ptxas_verbose:
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            jobs.append([NVCC] + CUDA_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj])
    # the translation units compile independently (the two persistent-kernel units take most
    # of the time), so in parallel
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_run, cmd, verbose) for cmd in jobs]:
            f.result()
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"], verbose)
    for prog, src in CLI_PROGRAMS.items():
        path = os.path.join(CLI, src)
        if not os.path.exists(path):
            continue
        out = os.path.join(BIN_DIR, prog)
        if _newer(out, deps + [LIB]):
            _run([NVCC, "-O2", "-std=c++17", "-x", "cu", path, "-o", out,
                  "-I", os.path.join(ROOT, "include"), "-L", LIB_DIR, "-lmustard_b200",
                  "-Xlinker", "-rpath,$ORIGIN/../lib"] + ARCH, verbose)
    for prog, path in PROBES.items():
        out = os.path.join(BIN_DIR, prog)
        if _newer(out, [path]):
            _run([NVCC, "-O3", "-std=c++17", path, "-o", out] + ARCH, verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
