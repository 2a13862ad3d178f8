"""A model of the tcgen05 TMA pipeline's barrier bookkeeping (tcgen05.cuh, mainloop_tma /
mainloop_tma_bf16), checked on CPU.

Thread 0 runs one item after another through `stages` shared-memory stages.  Per stage it
uses two mbarriers: full[s] completes when the stage's loads land, mbar[s] when the MMAs that
read it are done.  A wait names the parity of the phase it waits for; the thread keeps one
parity bit per barrier, across items.  The loads land in any order, some time after they are
issued; the commits complete in issue order, some time after the MMAs are issued.

Checked, over items of random depth (shorter and longer than the stage count) and random
completion timing: every wait returns on the completion it is meant for (the loads of that
k-slice, the MMAs of that k-slice) and never on a stale or a later one, no MMA reads a stage
whose load has not landed, every item ends with all its commits consumed, and nothing
deadlocks.
"""
import random

import pytest


class Barrier:
    """Phases complete one after another; phase c has parity c & 1."""

    def __init__(self):
        self.completed = []              # label of each completed phase, in order

    def passes(self, parity):
        # try_wait.parity(P) succeeds once the phase with parity P has completed, i.e. the
        # current (incomplete) phase has the other parity
        return (len(self.completed) & 1) != parity


def run(items, stages, seed, reset_bits=False):
    rng = random.Random(seed)
    full = [Barrier() for _ in range(stages)]
    mbar = [Barrier() for _ in range(stages)]
    in_flight_loads = []                 # (stage, label) landing in any order
    in_flight_commits = []               # (stage, label) completing in issue order
    stage_holds = [None] * stages        # label of the k-slice whose load landed in the stage
    ph = fph = 0                         # thread 0's parity bits, kept across items

    def settle(force=False):
        # let some asynchronous completions happen (all of them when the thread would block)
        while in_flight_loads and (force or rng.random() < 0.5):
            s, label = in_flight_loads.pop(rng.randrange(len(in_flight_loads)))
            stage_holds[s] = label
            full[s].completed.append(label)
            if not force:
                break
        while in_flight_commits and (force or rng.random() < 0.5):
            s, label = in_flight_commits.pop(0)
            mbar[s].completed.append(label)
            if not force:
                break

    def wait(bar, parity, want):
        for _ in range(4):
            if bar.passes(parity):
                break
            settle()
        if not bar.passes(parity):
            settle(force=True)
        assert bar.passes(parity), f"deadlock waiting for {want}"
        assert bar.completed[-1] == want, (bar.completed[-1], want)

    for it, nk in enumerate(items):
        if reset_bits:                   # a planted mistake: parity not carried across items
            ph = fph = 0

        def issue(s, kt):
            in_flight_loads.append((s, (it, kt)))

        for s in range(min(stages, nk)):
            issue(s, s)
        for kt in range(nk):
            s = kt % stages
            wait(full[s], (fph >> s) & 1, (it, kt))
            fph ^= 1 << s
            assert stage_holds[s] == (it, kt)        # the MMAs read this k-slice's operands
            in_flight_commits.append((s, (it, kt)))  # the MMAs, committed to mbar[s]
            settle()
            if kt > 0 and kt - 1 + stages < nk:      # reload the stage of k-slice kt - 1
                sp = (kt - 1) % stages
                wait(mbar[sp], (ph >> sp) & 1, (it, kt - 1))
                ph ^= 1 << sp
                issue(sp, kt - 1 + stages)
        for kt in range(max(nk - stages, 0), nk):    # the commits not waited above
            s = kt % stages
            wait(mbar[s], (ph >> s) & 1, (it, kt))
            ph ^= 1 << s
        # the accumulator is final and every stage free before the next item
        assert not in_flight_loads and not in_flight_commits
    return full, mbar


@pytest.mark.parametrize("stages", [3, 6])
@pytest.mark.parametrize("seed", range(6))
def test_pipeline_waits_see_their_own_completions(stages, seed):
    rng = random.Random(1000 + seed)
    # depths of 64-column k-slices: 1536 / 64 = 24 at the configs' tiles, down to a single
    # slice for the shallow updates of nested diagonal factorisations
    items = [rng.choice([1, 2, 3, 4, 5, 7, 8, 24]) for _ in range(40)]
    full, mbar = run(items, stages, seed)
    for s in range(stages):              # one load and one commit per k-slice held
        held = sum((nk - s + stages - 1) // stages for nk in items if s < nk)
        assert len(full[s].completed) == len(mbar[s].completed) == held


def test_model_catches_a_parity_bit_not_carried_across_items():
    """A mistake planted in the model: the parity bits reset at every item.  Then some wait
    returns on an earlier item's completion, or never."""
    caught = 0
    for seed in range(6):
        rng = random.Random(seed)
        items = [rng.choice([1, 2, 3, 4, 5, 7]) for _ in range(12)]
        try:
            run(items, 3, seed, reset_bits=True)
        except AssertionError:
            caught += 1
    assert caught == 6


# ---- the warp-specialised pipeline (tcgen05.cuh ws_load / ws_mma / ws_drain) ---------------
#
# Three actors share one ring that runs on across items: the loader (thread 0) puts slice g
# (counted over the CTA's whole run) into stage g % stages once the MMAs of slice g - stages
# are done (waiting on empty[s] with parity (g / stages - 1) & 1); the MMA thread waits for
# full[s] with parity (g / stages) & 1, issues the slice's MMAs and commits them to empty[s];
# after an item's last slice it commits to accf[buf] (buf alternating per item); the drain
# warps wait on accf[buf] with parity (items drained from buf so far) & 1.  A round ends
# when the loader has issued the item's slices, the MMA thread its MMAs and the drain warps
# the previous item's update.  Loads land in any order; commits complete in issue order.


def run_ws(items, stages, seed, drop_use_parity=False):
    rng = random.Random(seed)
    full = [Barrier() for _ in range(stages)]
    empty = [Barrier() for _ in range(stages)]
    accf = [Barrier(), Barrier()]
    loads, commits = [], []              # in flight
    holds = [None] * stages              # which slice a stage holds (after its load landed)
    reading = [None] * stages            # slice whose MMAs are reading the stage
    st = {"prod": 0, "cons": 0}
    drained = [0, 0]

    def settle_one():
        # one asynchronous completion, if any is in flight
        if loads and (not commits or rng.random() < 0.5):
            s, label = loads.pop(rng.randrange(len(loads)))
            assert reading[s] is None, "a load overwrote a stage the MMAs still read"
            holds[s] = label
            full[s].completed.append(label)
            return True
        if commits:
            kind, idx, label = commits.pop(0)
            if kind == "empty":
                reading[idx] = None
                empty[idx].completed.append(label)
            else:
                accf[idx].completed.append(label)
            return True
        return False

    def wait(bar, parity, want):         # a coroutine: yields until the phase completed
        while not bar.passes(parity):
            yield
        assert bar.completed[-1] == want, (bar.completed[-1], want)

    def loader(nk):
        for _ in range(nk):
            g, s = st["prod"], st["prod"] % stages
            if g >= stages:
                par = 0 if drop_use_parity else ((g // stages) - 1) & 1
                yield from wait(empty[s], par, ("slice", g - stages))
            loads.append((s, ("slice", g)))
            st["prod"] += 1
            yield

    def mma(nk, buf, it):
        for _ in range(nk):
            g, s = st["cons"], st["cons"] % stages
            yield from wait(full[s], (g // stages) & 1, ("slice", g))
            assert holds[s] == ("slice", g)
            reading[s] = ("slice", g)
            commits.append(("empty", s, ("slice", g)))
            st["cons"] += 1
            yield
        commits.append(("accf", buf, ("item", it)))

    def drain(pending):
        if pending is None:
            return
        pb, pit = pending
        yield from wait(accf[pb], drained[pb] & 1, ("item", pit))
        drained[pb] += 1

    def run_round(actors):               # random interleaving of the actors and completions
        live = list(actors)
        stalls = 0
        while live:
            a = rng.choice(live)
            try:
                next(a)
            except StopIteration:
                live.remove(a)
            if rng.random() < 0.5 and settle_one():
                stalls = 0
            stalls += 1
            if stalls > 10_000:
                while settle_one():
                    pass
                assert stalls < 20_000, "deadlock"

    pending = None
    for it, nk in enumerate(items):
        buf = it & 1
        run_round([loader(nk), mma(nk, buf, it), drain(pending)])
        pending = (buf, it)
    run_round([drain(pending)])
    while settle_one():
        pass
    assert not loads and not commits
    return st["prod"], drained


@pytest.mark.parametrize("seed", range(8))
def test_ws_pipeline_waits_see_their_own_completions(seed):
    rng = random.Random(2000 + seed)
    # slices of 32 (TF32) / 64 (BF16) columns: 48 / 24 at tile 1536, 1 for shallow nested updates
    items = [rng.choice([1, 2, 3, 5, 6, 7, 12, 24, 48]) for _ in range(30)]
    prod, drained = run_ws(items, 6, seed)
    assert prod == sum(items) and sum(drained) == len(items)


def test_ws_model_catches_a_wrong_stage_parity():
    """A mistake planted in the model: the loader waits on empty[s] with parity 0 for every
    use of the stage.  Some wait then returns on a stale completion, or the load overwrites a
    stage the MMAs still read."""
    caught = 0
    for seed in range(6):
        rng = random.Random(seed)
        items = [rng.choice([2, 3, 5, 7, 12]) for _ in range(10)]
        try:
            run_ws(items, 6, seed, drop_use_parity=True)
        except AssertionError:
            caught += 1
    assert caught == 6
