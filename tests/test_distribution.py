"""The multi-GPU distribution plan (mustard_b200/distribution.py), executed on CPU ranks.

Each gloo rank stands for one GPU: it holds only the tiles it owns (the others start as
NaN), runs the tasks the plan gives it in the reference's task order with the oracle's tile
arithmetic, receives the tile versions the plan says it needs before a task, and sends the
copies the plan lists after one.  Rank 0 then gathers every rank's tiles: the distributed
factor must equal the single-process oracle's bit for bit (same tile calls, same operands,
same order per tile), and no rank may ever have read a NaN (a missing copy).
"""
import datetime
import os
import socket

import numpy as np
import pytest

from oracle import gen, tiled


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _graph(kind, n, tile):
    import mustard_b200 as mtd
    return mtd.TaskGraph(mtd.KIND_CHOLESKY if kind == "chol" else mtd.KIND_LU, n, tile).build_tiled()


def _input(kind, n):
    return gen.spd_input(n, 3) if kind == "chol" else gen.lu_input(n, 3)


def _rank(rank, world, port, kind, n, tile, q):
    import torch
    import torch.distributed as dist

    from mustard_b200 import OP_NAMES
    from mustard_b200.distribution import build_plan, owner
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        g = _graph(kind, n, tile)
        plan = build_plan(g, world)
        a = np.array(_input(kind, n), order="F")
        T = plan.tiles

        def block(tile):
            i, j = tile
            return (slice(i * tile_b, min((i + 1) * tile_b, n)), slice(j * tile_b, min((j + 1) * tile_b, n)))

        tile_b = tile
        for i in range(T):
            for j in range(T):
                if owner((i, j), world) != rank:
                    a[block((i, j))] = np.nan
        pending = []

        def send(tile, dest, version):
            buf = torch.from_numpy(np.ascontiguousarray(a[block(tile)]))
            pending.append((dist.isend(buf, dst=dest, tag=plan.version_tag(tile, version)), buf))

        def recv(tile, version):
            rs, cs = block(tile)
            buf = torch.empty((rs.stop - rs.start, cs.stop - cs.start), dtype=torch.float64)
            dist.recv(buf, src=owner(tile, world), tag=plan.version_tag(tile, version))
            a[rs, cs] = buf.numpy()

        for tile, src, dest in plan.initial_sends:
            if src == rank:
                send(tile, dest, -1)
        for t, (op, write, reads) in enumerate(plan.tasks):
            if plan.rank_of[t] != rank:
                continue
            for tile, version in plan.needs[t]:
                recv(tile, version)
            for tile in list(reads) + [write]:
                assert not np.isnan(a[block(tile)]).any(), (t, tile)
            assert tiled.run_task(a, tile_b, (OP_NAMES[op], write, reads)) == 0
            for tile, dest in plan.sends[t]:
                send(tile, dest, t)
        for w, _buf in pending:
            w.wait()
        # gather: every rank contributes its own tiles
        mine = np.zeros((n, n))
        for i in range(T):
            for j in range(T):
                if owner((i, j), world) == rank:
                    mine[block((i, j))] = a[block((i, j))]
        full = torch.from_numpy(np.ascontiguousarray(mine))
        dist.all_reduce(full)
        if rank == 0:
            q.put(full.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["chol", "lu"])
@pytest.mark.parametrize("world", [2, 3])
def test_distributed_factor_equals_single_process(kind, world):
    import torch.multiprocessing as mp
    n, tile = 500, 100
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, kind, n, tile, q)) for r in range(world)]
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
    want = np.array(_input(kind, n), order="F")
    assert tiled.tiled_factor(want, tile, kind) == 0
    if kind == "chol":  # the strict upper triangle is never written: compare what is
        got, want = np.tril(got), np.tril(want)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("kind", ["chol", "lu"])
def test_plan_covers_every_remote_read_once(kind):
    from mustard_b200.distribution import build_plan, owner, reference_copies
    g = _graph(kind, 2400, 200)  # 12 x 12 tiles
    for world in (1, 2, 4, 8):
        plan = build_plan(g, world)
        deps = [g.deps(t) for t in range(g.num_tasks)]
        assert all(plan.rank_of[t] == owner(w, world) for t, (_o, w, _r) in enumerate(plan.tasks))
        if world == 1:
            assert plan.transfers() == 0 and plan.cross_rank_edges(deps) == 0
            continue
        # every read of a tile owned elsewhere is satisfied by exactly one copy to that rank
        delivered = set()
        for tile, src, dest in plan.initial_sends:
            delivered.add((tile, -1, dest))
        for t, copies in enumerate(plan.sends):
            for tile, dest in copies:
                assert (tile, t, dest) not in delivered
                delivered.add((tile, t, dest))
        last = {}
        for t, (_op, write, reads) in enumerate(plan.tasks):
            r = plan.rank_of[t]
            for tile in set(reads) | {write}:
                if owner(tile, world) != r:
                    assert (tile, last.get(tile, -1), r) in delivered
            last[write] = t
        # fewer copies than the reference's funnel through PE 0
        assert plan.transfers() < reference_copies(plan.tasks, world)
