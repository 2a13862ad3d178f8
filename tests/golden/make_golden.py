"""Regenerate the golden fixtures that pin the oracle to the reference's own code.

Runs oracle/_ref/ref_driver -- the reference's include/gen.h generator and
include/verify.h verifier compiled in place by oracle/ref/Makefile -- and writes:

  ref_gen.json     the generator's output: all entries for n = 15 (hex floats) and a
                   SHA-256 of the row-major bytes for n in (64, 300, 600)
  ref_verify.json  the verifier's printed "error = %.6f" line and pass flag for factors
                   of the n = 600 generator matrix (2 x 2 tiles of 300), as computed and
                   after deliberate perturbations

Needs the reference checkout (this script reads it at generation time only); the
fixtures it writes are committed, so the tests never need the reference.
Usage: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import tiled  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
OUT = os.path.dirname(os.path.abspath(__file__))


def ref_gen(n):
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        path = f.name
    subprocess.check_call([DRIVER, "gen", str(n), path])
    a = np.fromfile(path, dtype=np.float64).reshape(n, n)
    os.unlink(path)
    return a


def ref_verify(kind, a_rowmajor, f_colmajor):
    n = a_rowmajor.shape[0]
    with tempfile.TemporaryDirectory() as d:
        pa, pf = os.path.join(d, "a.bin"), os.path.join(d, "f.bin")
        np.ascontiguousarray(a_rowmajor).tofile(pa)
        np.asfortranarray(f_colmajor).T.copy().tofile(pf)  # column-major bytes
        out = subprocess.check_output([DRIVER, "verify_" + kind, str(n), pa, pf]).decode()
    err_line = [ln for ln in out.splitlines() if ln.startswith("error = ")][0]
    passed = int([ln for ln in out.splitlines() if ln.startswith("pass=")][0].split("=")[1])
    return err_line, passed


def main():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref")])
    gen = {"n15": [float(v).hex() for v in ref_gen(15).ravel()], "sha256": {}}
    for n in (64, 300, 600):
        gen["sha256"][str(n)] = hashlib.sha256(ref_gen(n).tobytes()).hexdigest()
    with open(os.path.join(OUT, "ref_gen.json"), "w") as f:
        json.dump(gen, f, indent=1)

    n, b = 600, 300
    a = ref_gen(n)
    cases = []
    for kind in ("lu", "chol"):
        f = np.asfortranarray(a.copy())
        assert tiled.tiled_factor(f, b, "chol" if kind == "chol" else "lu") == 0
        for label, scale in (("exact", 0.0), ("perturbed_small", 1e-9), ("perturbed_large", 1e-3)):
            g = f.copy(order="F")
            if scale:
                rng = np.random.default_rng(11)
                idx = rng.integers(0, n, size=(40, 2))
                for i, j in idx:
                    if kind == "chol" and i < j:
                        i, j = j, i
                    g[i, j] += scale
            err_line, passed = ref_verify(kind, a, g)
            cases.append({"kind": kind, "n": n, "tile": b, "case": label, "scale": scale,
                          "perturb_seed": 11, "perturb_count": 40,
                          "error_line": err_line, "pass": passed})
    with open(os.path.join(OUT, "ref_verify.json"), "w") as f:
        json.dump({"cases": cases}, f, indent=1)
    print("wrote", os.path.join(OUT, "ref_gen.json"), os.path.join(OUT, "ref_verify.json"))


if __name__ == "__main__":
    main()
