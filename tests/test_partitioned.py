"""The partitioned LU plan (mustard_b200/partitioned.py), executed on CPU ranks.

Each gloo rank stands for one GPU.  It holds only its tile rows (the others start as NaN) and
runs the plan step by step with the oracle's tile arithmetic:

- the owner of step k factors the diagonal tile and solves its row;
- the owner broadcasts tile row k to the step's receivers;
- every rank solves and updates its own rows.

Rank 0 gathers the rows.  The factor must equal the single-process tiled LU bit for bit:
each tile sees the same calls with the same operands in the same order.  No rank may read a
NaN: every tile it reads is its own or arrived with a broadcast.
"""
import datetime
import socket

import numpy as np
import pytest

from oracle import gen, tiled


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, n, tile, q):
    import torch
    import torch.distributed as dist

    from mustard_b200.partitioned import build_plan, owner
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        T = tiled.num_tiles(n, tile)
        plan = build_plan(T, world)
        a = np.array(gen.lu_input(n, 3), order="F")
        rows = lambda i: slice(i * tile, min((i + 1) * tile, n))
        cols = lambda j: slice(j * tile, min((j + 1) * tile, n))
        for i in range(T):
            if owner(i, world) != rank:
                a[rows(i), :] = np.nan

        def run(task):
            _op, write, reads = task
            for ti, tj in list(reads) + [write]:
                assert not np.isnan(a[rows(ti), cols(tj)]).any(), (task, rank)
            assert tiled.run_task(a, tile, task) == 0

        for step in plan.steps:
            k = step.k
            if rank == step.owner:
                for task in step.owner_tasks:
                    run(task)
            # tile row k, columns k .. : one broadcast group per step (every rank takes part, so
            # the collective calls match; ranks outside the receivers ignore the data)
            buf = torch.from_numpy(np.ascontiguousarray(a[rows(k), k * tile:]))
            dist.broadcast(buf, src=step.source)
            if rank in step.receivers:
                a[rows(k), k * tile:] = buf.numpy()
            for task in step.rank_tasks.get(rank, []):
                run(task)
        mine = np.zeros((n, n))
        for i in range(T):
            if owner(i, world) == rank:
                mine[rows(i), :] = a[rows(i), :]
        full = torch.from_numpy(np.ascontiguousarray(mine))
        dist.all_reduce(full)
        if rank == 0:
            q.put(full.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_lu_equals_single_process(world):
    import torch.multiprocessing as mp
    n, tile = 500, 100
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, tile, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0] * world
    want = np.array(gen.lu_input(n, 3), order="F")
    assert tiled.tiled_factor(want, tile, "lu") == 0
    assert np.array_equal(got, want)


def test_plan_matches_the_reference_layout_and_chain():
    from mustard_b200.partitioned import build_plan, chain, owner, slice_bytes, slices_of
    T = 7
    for world in (1, 2, 3, 4, 8):
        plan = build_plan(T, world)
        # 1-D block-cyclic slices: every tile row on exactly one rank, ceil(T / P) at most
        held = sorted(i for r in range(world) for i in slices_of(r, T, world))
        assert held == list(range(T))
        assert max(len(slices_of(r, T, world)) for r in range(world)) == -(-T // world)
        # every task of the tiled LU exactly once, each on the owner of the tile it writes
        tasks = plan.tasks()
        assert sorted(map(str, tasks)) == sorted(map(str, tiled.lu_tasks(T)))
        for step in plan.steps:
            assert all(owner(w[0], world) == step.owner for _op, w, _r in step.owner_tasks)
            for r, ts in step.rank_tasks.items():
                assert all(owner(w[0], world) == r for _op, w, _r in ts)
                # a rank with update work in step k receives slice k (or owns it)
                assert r == step.owner or r in step.receivers
            # the chain: the owner's neighbours in order, no further than the rows left
            assert step.receivers == chain(step.k, T, world)
            assert step.owner not in step.receivers
            assert len(step.receivers) == min(world - 1, T - step.k - 1)
    # one slice's broadcast part: its rows x the columns from its diagonal on
    assert slice_bytes(1000, 300, 3) == 100 * 100 * 8
    assert slice_bytes(1000, 300, 0) == 300 * 1000 * 8
