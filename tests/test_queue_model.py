"""A model of the persistent scheduler's device protocol (scheduler.cuh), checked on CPU under
random interleavings of CTAs.

Each CTA is a coroutine that yields at every step the device performs as one global memory
operation, so a random scheduler explores interleavings the GPU may produce:

- claim (claim_item): read `avail`; fetch-and-add -1 on `avail`, undone if the old value
  was not positive; fetch-and-add +1 on `head`; wait for the reserved slot to be written;
- run the item, then complete it (complete_item): decrement the task's items-left counter;
  the last item decrements each successor's predecessor counter, and a successor that
  reaches zero is pushed (release_task): fetch-and-add on `tail`, write the slots, then
  fetch-and-add their number on `avail`.  Every task has at least one item: a join (the
  stand-in of a nested factorisation with several sinks) has one no-op item, so a release
  never recurses.

The tcgen05 kernel's variant (`deferred`): a GEMM / SYRK item is completed only during the
CTA's next claim, the completion and the claim interleaving step by step.

Checked, in both: every work item runs exactly once, no task starts before every item of its
predecessors has run, every queue slot is claimed once, and the run terminates (a CTA holding
a pending item never waits on itself).
"""
import random

import pytest

EMPTY = None


class Queue:
    def __init__(self, cap):
        self.avail = 0
        self.head = 0
        self.tail = 0
        self.slots = [EMPTY] * cap


class Model:
    def __init__(self, n_items, succ, deps, queue_of, n_queues):
        assert all(n >= 1 for n in n_items)    # a join is one no-op item
        self.n_items = n_items                 # per task
        self.succ = succ
        self.deps = list(deps)                 # predecessor counters
        self.items_left = list(n_items)
        self.queue_of = queue_of
        self.queues = [Queue(sum(n for t, n in enumerate(n_items) if queue_of[t] == q) + 1)
                       for q in range(n_queues)]
        self.tasks_done = 0
        self.n_tasks = len(n_items)
        self.finished = [0] * len(n_items)     # items of each task whose work is done
        self.data_done = set()                 # tasks whose every item (or join) is done
        self.done_tasks = set()                # tasks counted in tasks_done
        self.runs = []                         # (task, item) in execution order
        self.started = {}

    # release_task: reserve slots on `tail`, write them, then publish them on `avail`
    def release(self, task):
        n = self.n_items[task]
        q = self.queues[self.queue_of[task]]
        base = q.tail
        q.tail += n
        yield
        for i in range(n):
            q.slots[base + i] = (task, i)
            yield
        q.avail += n                           # after the slots (the device fences in between)
        yield

    def complete(self, task):
        self.items_left[task] -= 1
        left = self.items_left[task]
        yield
        if left != 0:
            return
        for s in self.succ[task]:
            self.deps[s] -= 1
            left_s = self.deps[s]
            yield
            if left_s == 0:
                yield from self.release(s)
        self.done_tasks.add(task)
        self.tasks_done += 1
        yield

    def claim(self):
        """One attempt (claim_item); returns (task, item), "exit" or None."""
        if self.tasks_done >= self.n_tasks:
            return "exit"
        avail = [q.avail for q in self.queues]  # one round trip
        yield
        for qi, q in enumerate(self.queues):
            if avail[qi] <= 0:
                continue
            old = q.avail
            q.avail -= 1
            yield
            if old <= 0:                      # taken meanwhile: give the unit back
                q.avail += 1
                yield
                continue
            h = q.head
            q.head += 1
            yield
            while q.slots[h] is EMPTY:        # reserved: its producer is between tail and write
                yield
            claimed = q.slots[h]
            q.slots[h] = "claimed"
            return claimed
        return None

    def run_item(self, task, item):
        self.started.setdefault(task, set(self.data_done))
        self.runs.append((task, item))
        yield                                 # the item's work
        self.finished[task] += 1
        if self.finished[task] == self.n_items[task]:
            self.data_done.add(task)

    def cta(self):
        while True:
            claimed = yield from self.claim()
            if claimed == "exit":
                return
            if claimed is None:
                yield                         # back off and retry
                continue
            yield from self.run_item(*claimed)
            yield from self.complete(claimed[0])

    def cta_deferred(self, deferred_ops, rng):
        """The tcgen05 kernel's loop: an item of a deferred kind is completed only at the
        next claim, by other threads of the CTA, while thread 0 claims (the two interleave
        step by step); an item of another kind finds nothing pending and completes at once."""
        pending = None
        while True:
            gens = {"claim": self.claim()}
            if pending is not None:
                gens["complete"] = self.complete(pending)
            result = None
            while gens:
                k = rng.choice(sorted(gens))
                try:
                    next(gens[k])
                except StopIteration as e:
                    if k == "claim":
                        result = e.value
                    del gens[k]
                yield
            pending = None
            if result == "exit":
                return
            if result is None:
                yield
                continue
            task, item = result
            yield from self.run_item(task, item)
            if self.op[task] in deferred_ops:
                pending = task
            else:
                yield from self.complete(task)


    def claim_waiting(self):
        """pop_item: claim attempts until one succeeds (or the run is over)."""
        while True:
            r = yield from self.claim()
            if r is not None:
                return r
            yield

    def cta_ws(self, ws_ops, rng, waiting_claim_in_round=False):
        """The warp-specialised tcgen05 loop (persistent_loop_ws): an item of a ws kind runs
        (loads and MMAs) while thread 0 tries once to claim the next item and the drain warps
        complete the previous ws item, all interleaved; it is itself completed in the next
        round.  When the attempt found nothing, the next round starts with thread 0 waiting
        for an item while the drain warps complete the pending one.  Any other item finds
        nothing pending, runs, completes, then thread 0 waits for the next.  With
        waiting_claim_in_round (a planted mistake) thread 0 waits for its claim inside the ws
        round, before the round's own item can complete."""
        pending, nxt = None, None

        def interleave(gens):
            results = {}
            while gens:
                k = rng.choice(sorted(gens))
                try:
                    next(gens[k])
                except StopIteration as e:
                    results[k] = e.value
                    del gens[k]
                yield
            return results

        while True:
            if nxt is None:
                gens = {"claim": self.claim_waiting()}
                if pending is not None:
                    gens["complete"] = self.complete(pending)
                res = yield from interleave(gens)
                pending, nxt = None, res["claim"]
            if nxt == "exit":
                if pending is not None:
                    yield from self.complete(pending)
                return
            task, item = nxt
            nxt = None
            if self.op[task] in ws_ops:
                gens = {"run": self.run_item(task, item),
                        "claim": self.claim_waiting() if waiting_claim_in_round else self.claim()}
                if pending is not None:
                    gens["complete"] = self.complete(pending)
                res = yield from interleave(gens)
                nxt = res["claim"]
                pending = task
            else:
                if pending is not None:
                    yield from self.complete(pending)
                    pending = None
                yield from self.run_item(task, item)
                yield from self.complete(task)
                nxt = yield from self.claim_waiting()


def cholesky_dag(t):
    """The reference's tiled Cholesky task list (cholesky_mustard.cu:224-395) as tasks with
    items, last-writer predecessors, and the three-queue assignment (0: POTRF/TRSM/SYRK and
    the updates one column ahead, 1: two to three ahead, 2: the rest)."""
    tasks, write_of = [], {}
    for k in range(t):
        tasks.append(("POTRF", (k, k), [(k, k)], 0))
        for i in range(k + 1, t):
            tasks.append(("TRSM", (i, k), [(k, k), (i, k)], 0))
        for i in range(k + 1, t):
            tasks.append(("SYRK", (i, i), [(i, i), (i, k)], 0))
            for j in range(i + 1, t):
                ahead = i - k
                tasks.append(("GEMM", (j, i), [(j, i), (j, k), (i, k)], 0 if ahead <= 1 else 1 if ahead <= 3 else 2))
    preds = []
    for idx, (_op, w, reads, _q) in enumerate(tasks):
        preds.append(sorted({write_of[x] for x in reads + [w] if x in write_of}))
        write_of[w] = idx
    succ = [[] for _ in tasks]
    for i, ps in enumerate(preds):
        for p in ps:
            succ[p].append(i)
    return tasks, preds, succ


def run_model(tasks, preds, succ, n_items, n_ctas, seed, deferred=False, max_steps=2_000_000, ws=False,
              ws_bug=False):
    rng = random.Random(seed)
    m = Model(n_items, succ, [len(p) for p in preds], [q for *_, q in tasks], 3)
    m.op = [op for op, *_ in tasks]
    for r in (i for i, p in enumerate(preds) if not p):  # kernel_populate_queue
        for _ in m.release(r):
            pass
    if ws:
        ctas = [m.cta_ws({"GEMM", "SYRK"}, random.Random(seed * 37 + c), ws_bug) for c in range(n_ctas)]
    else:
        ctas = [m.cta_deferred({"GEMM", "SYRK"}, random.Random(seed * 31 + c)) if deferred else m.cta()
                for c in range(n_ctas)]
    live = list(range(n_ctas))
    steps = 0
    while live:
        i = rng.choice(live)
        try:
            next(ctas[i])
        except StopIteration:
            live.remove(i)
        steps += 1
        assert steps < max_steps, "no termination"
    return m


@pytest.mark.parametrize("mode", ["plain", "deferred", "ws"])
@pytest.mark.parametrize("t,n_ctas,seed", [(3, 2, 1), (4, 4, 2), (5, 8, 3), (6, 3, 4), (6, 16, 5), (2, 1, 6), (3, 1, 7)])
def test_cholesky_dag_runs_each_item_once_in_dependency_order(t, n_ctas, seed, mode):
    tasks, preds, succ = cholesky_dag(t)
    rng = random.Random(seed)
    # a few items per task (a join's single no-op item is one of them)
    n_items = [1 if (idx % 7 == 3 and preds[idx]) else rng.randint(1, 3) for idx in range(len(tasks))]
    m = run_model(tasks, preds, succ, n_items, n_ctas, seed, deferred=mode == "deferred", ws=mode == "ws")
    want = sorted((tk, i) for tk, n in enumerate(n_items) for i in range(n))
    assert sorted(m.runs) == want                       # every item exactly once
    assert m.tasks_done == len(tasks) and m.done_tasks == set(range(len(tasks)))
    for tk, done_before in m.started.items():          # predecessors' work done before a start
        assert set(preds[tk]) <= done_before, tk
    for q in m.queues:                                  # every pushed slot claimed once
        assert q.head == q.tail and q.avail == 0
        assert all(s in (EMPTY, "claimed") for s in q.slots)
        assert q.slots[:q.tail] == ["claimed"] * q.tail


def test_model_detects_a_broken_claim():
    """The checks catch a mistake: a claim that skips the avail count (reads head blindly)
    ends with items run twice or never, or claims a slot nobody reserved."""
    tasks, preds, succ = cholesky_dag(4)
    n_items = [2] * len(tasks)

    class Broken(Model):
        def cta(self):
            while self.tasks_done < self.n_tasks:
                q = self.queues[0]
                if q.head >= len(q.slots) - 1:
                    return
                h = q.head
                yield
                q.head = h + 1                # not atomic: two CTAs can take the same slot
                yield
                if q.slots[h] in (EMPTY, "claimed"):
                    return
                task, item = q.slots[h]
                self.runs.append((task, item))
                yield from self.complete(task)

    rng = random.Random(7)
    m = Broken(n_items, succ, [len(p) for p in preds], [0] * len(tasks), 3)
    for r in (i for i, p in enumerate(preds) if not p):
        for _ in m.release(r):
            pass
    ctas = [m.cta() for _ in range(6)]
    live = list(range(6))
    for _ in range(200_000):
        if not live:
            break
        i = rng.choice(live)
        try:
            next(ctas[i])
        except StopIteration:
            live.remove(i)
    want = sorted((tk, i) for tk, n in enumerate(n_items) for i in range(n))
    assert sorted(m.runs) != want


def test_ws_model_catches_a_waiting_claim_inside_the_round():
    """The mistake the warp-specialised loop first had: thread 0 waited for its next claim
    inside the round of a TMA item, whose completion comes only in the next round.  On one
    CTA the last update before a diagonal factorisation then waits for ever."""
    tasks, preds, succ = cholesky_dag(3)
    with pytest.raises(AssertionError, match="no termination"):
        run_model(tasks, preds, succ, [1] * len(tasks), 1, 3, ws=True, ws_bug=True, max_steps=200_000)
