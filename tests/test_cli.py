"""The lu_mustard / cholesky_mustard drivers: the reference's flags and output lines
(include/cli.h:21-97, cholesky_mustard.cu:486-526)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "mustard_b200", "bin")


def run(prog, *args, timeout=300):
    p = subprocess.run([os.path.join(BIN, prog), *args], capture_output=True, text=True, timeout=timeout)
    return p.returncode, p.stdout, p.stderr


@pytest.mark.parametrize("prog", ["lu_mustard", "cholesky_mustard"])
def test_help_and_argument_errors(prog):
    rc, out, err = run(prog, "--help")
    assert rc == 1 and "Usage:" in err and "--subgraph" in err
    rc, out, err = run(prog, "-n=600", "-t=7")
    assert rc == 1 and "N must be divisible by T" in err
    rc, out, err = run(prog, "-n=abc")
    assert rc == 1 and "valid N" in err
    rc, out, err = run(prog, "--bogus")
    assert rc == 1 and "unknown option" in err


@pytest.mark.gpu
@pytest.mark.parametrize("prog", ["lu_mustard", "cholesky_mustard"])
@pytest.mark.parametrize("mode", ["--subgraph", "--tiled"])
def test_reference_example_runs_and_verifies(prog, mode):
    rc, out, err = run(prog, "-n=600", "-t=2", mode, "--verify", "-r=2")
    assert rc == 0, err
    assert ("SUBGRAPH" if mode == "--subgraph" else "TILED") + " with N=600 (2 of 300x300 tiles)" in out
    assert len(re.findall(r"device 0 \| \d run \| time \(s\): \d+\.\d{4}", out)) == 2
    assert "error = 0.000000" in out
    assert "Result passes verification: 1" in out
    assert "Total time used (s):" in out


@pytest.mark.gpu
def test_ragged_tile_and_generators():
    rc, out, err = run("cholesky_mustard", "-n=3000", "--tile=512", "--subgraph", "--gen=spd", "--verify")
    assert rc == 0, err
    assert "(6 of 512x512 tiles)" in out and "Result passes verification: 1" in out
    rc, out, err = run("lu_mustard", "-n=2500", "--tile=768", "--subgraph", "--gen=uniform", "--verify", "-v")
    assert rc == 0, err
    assert "Result passes verification: 1" in out and "totalNodes=" in out


@pytest.mark.gpu
def test_dot_dump_has_the_reference_dependencies(tmp_path):
    # --dot writes ./graph.dot (cholesky_mustard.cu:447-450): one edge per predecessor
    from oracle import tiled
    p = subprocess.run([os.path.join(BIN, "cholesky_mustard"), "-n=900", "-t=3", "--subgraph", "--dot"],
                       capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert p.returncode == 0, p.stderr
    text = (tmp_path / "graph.dot").read_text()
    assert text.startswith("digraph tasks {") and text.rstrip().endswith("}")
    edges = sorted(tuple(map(int, m)) for m in re.findall(r"(\d+) -> (\d+);", text))
    deps = tiled.subgraph_dependencies(tiled.cholesky_tasks(3))
    assert edges == sorted((d, t) for t, ds in enumerate(deps) for d in ds)
