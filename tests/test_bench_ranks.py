"""bench.py's multi-rank host logic, on CPU: two gloo ranks take the same steps the NCCL ranks
of `bench.py --gpus 2` take (barrier, max over ranks of the step time, whole-job rate)."""
import datetime
import os
import socket

import pytest

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        ms = bench.max_over_ranks(10.0 + rank, dist, "cpu")  # rank 1 is the slower one
        q.put((rank, ms, bench.aggregate_rate(world, 1e12, ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_single_process_passes_the_time_through():
    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.aggregate_rate(1, 2e12, 100.0) == pytest.approx(20.0)


def test_two_ranks_report_the_slowest_rank_and_the_whole_job_rate():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        out = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    assert [r for r, _, _ in out] == [0, 1]
    assert all(ms == 11.0 for _, ms, _ in out)  # both ranks see the slowest rank's time
    # two replicas of 1e12 flop per step in 11 ms: 181.8 TFLOP/s for the whole job
    assert all(v == pytest.approx(2 * 1e12 / 11e-3 / 1e12) for _, _, v in out)


def _reference_arm(env_extra):
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, **env_extra)
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3", "--cpu-n", "600", "--cpu-tile", "300"],
                         capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    return [json.loads(l) for l in lines]


def test_reference_arm_line_and_other_ranks():
    (line,) = _reference_arm({"RANK": "0", "WORLD_SIZE": "1"})
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "TFLOP/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    # the config states the sample it ran and the metric's workload size
    cfg = line["config"]
    assert cfg["n"] == 600 and cfg["metric_n"] == 24000 and "sampled at N=600" in cfg["workload"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == line["value"] and cb["cores"] >= 1 and "N=600" in cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    # under torchrun only rank 0 works and prints
    assert _reference_arm({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
