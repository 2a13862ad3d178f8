"""Per-item device traces -> per-task spans, scheduler idle fraction, critical path, JSON.

A traced run (``TaskGraph.set_trace(True)``) records, per work item, the %globaltimer times
at which its CTA started and finished it, the SM and the device task.  From those records:

- a task's span runs from its first item's start to its last item's end;
- the busy fraction is the time each SM spent inside at least one item, summed over SMs,
  over (SMs x the run's span); the idle fraction is the rest (queue waits, dependency
  stalls, the tail).  Items of one SM may overlap: the tensor-core kernel finishes an item's
  C update while its next item's loads and MMAs already run;
- the critical path is walked back from the task that ended last, each time to the
  predecessor (device task dependencies) that ended last; along it, ``wait`` is the time
  from that predecessor's end to the task's first item start (the scheduler's hand-off
  plus any wait for a free SM).

``graph`` needs ``device_task_op(t)`` and ``device_task_deps(t)`` (a finalized TaskGraph).
"""
import json

from ._capi import OP_NAMES


def task_spans(graph, records):
    """{task: {"op", "start", "end", "items", "item_ns"}} (times in ns)."""
    spans = {}
    for s, e, _sm, task, _item in records:
        t = spans.get(task)
        if t is None:
            spans[task] = t = {"op": OP_NAMES.get(graph.device_task_op(task), "join"), "start": s, "end": e,
                               "items": 0, "item_ns": 0}
        t["start"] = min(t["start"], s)
        t["end"] = max(t["end"], e)
        t["items"] += 1
        t["item_ns"] += e - s
    return spans


def busy_fraction(records):
    if not records:
        return 0.0
    t0 = min(r[0] for r in records)
    t1 = max(r[1] for r in records)
    per_sm = {}
    for s, e, sm, _, _ in records:
        per_sm.setdefault(sm, []).append((s, e))
    busy = 0
    for iv in per_sm.values():  # union of the SM's item intervals
        iv.sort()
        cs, ce = iv[0]
        for s, e in iv[1:]:
            if s > ce:
                busy += ce - cs
                cs, ce = s, e
            else:
                ce = max(ce, e)
        busy += ce - cs
    return busy / (len(per_sm) * (t1 - t0))


def busy_profile(records, bins=20):
    """The busy fraction per time bin: the run's span cut into ``bins`` equal parts, and for
    each the SM-time inside items (overlapping items of one SM counted once) over the SMs seen
    x the bin's length.  Shows where the idle time sits (start-up, tail, in between)."""
    if not records or bins < 1:
        return []
    t0 = min(r[0] for r in records)
    t1 = max(r[1] for r in records)
    width = (t1 - t0) / bins
    if width <= 0:
        return [1.0] * bins
    per_sm = {}
    for s, e, sm, _, _ in records:
        per_sm.setdefault(sm, []).append((s, e))
    busy = [0.0] * bins
    for iv in per_sm.values():
        iv.sort()
        merged = []
        for s, e in iv:
            if merged and s <= merged[-1][1]:
                merged[-1][1] = max(merged[-1][1], e)
            else:
                merged.append([s, e])
        for s, e in merged:
            b0 = min(bins - 1, int((s - t0) / width))
            b1 = min(bins - 1, int((e - t0) / width))
            for b in range(b0, b1 + 1):
                lo = max(s, t0 + b * width)
                hi = min(e, t0 + (b + 1) * width)
                if hi > lo:
                    busy[b] += hi - lo
    return [v / (len(per_sm) * width) for v in busy]


def critical_path(graph, spans):
    """Tasks on the critical path, first to last: dicts with task, op, start, end, wait (ns)."""
    if not spans:
        return []
    task = max(spans, key=lambda t: spans[t]["end"])
    path = []
    while task is not None:
        sp = spans[task]
        preds = [p for p in graph.device_task_deps(task) if p in spans]
        prev = max(preds, key=lambda p: spans[p]["end"]) if preds else None
        wait = sp["start"] - spans[prev]["end"] if prev is not None else 0
        path.append({"task": task, "op": sp["op"], "start": sp["start"], "end": sp["end"], "wait": wait})
        task = prev
    path.reverse()
    return path


def summary(graph, records):
    """Busy fraction, span and the critical path's composition (per op: tasks, time in the
    task, waits before it), in ms."""
    spans = task_spans(graph, records)
    path = critical_path(graph, spans)
    t0 = min(r[0] for r in records)
    t1 = max(r[1] for r in records)
    per = {}
    for step in path:
        d = per.setdefault(step["op"], {"tasks": 0, "in_task_ms": 0.0, "wait_ms": 0.0})
        d["tasks"] += 1
        d["in_task_ms"] += (step["end"] - step["start"]) * 1e-6
        d["wait_ms"] += step["wait"] * 1e-6
    first = path[0]["start"] if path else t0
    return {"span_ms": (t1 - t0) * 1e-6, "busy": busy_fraction(records),
            "critical_path": {"tasks": len(path), "start_offset_ms": (first - t0) * 1e-6, "per_op": per}}


def dump_json(path, graph, records):
    """Write the records, the task spans and the critical path to ``path``."""
    spans = task_spans(graph, records)
    out = {"records": [list(r) for r in records],
           "tasks": {str(k): v for k, v in sorted(spans.items())},
           "critical_path": critical_path(graph, spans),
           "summary": summary(graph, records)}
    with open(path, "w") as f:
        json.dump(out, f)
    return out["summary"]
