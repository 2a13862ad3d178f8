"""Trace analysis on a synthetic trace (host logic, no GPU)."""
import json

from mustard_b200 import trace_analysis


class FakeGraph:
    # 0 POTRF -> 1 TRSM -> 3 GEMM ; 0 -> 2 TRSM -> 3 ; 3 -> 4 POTRF
    ops = {0: 0, 1: 1, 2: 1, 3: 3, 4: 0}
    deps = {0: [], 1: [0], 2: [0], 3: [1, 2], 4: [3]}

    def device_task_op(self, t):
        return self.ops[t]

    def device_task_deps(self, t):
        return self.deps[t]


# (start, end, sm, task, item), ns
RECORDS = [
    (0, 100, 0, 0, 0),
    (110, 200, 0, 1, 0), (110, 300, 1, 1, 1),   # task 1 ends at 300
    (105, 250, 2, 2, 0),                         # task 2 ends at 250
    (320, 400, 0, 3, 0), (330, 420, 1, 3, 1),
    (450, 500, 2, 4, 0),
]


def test_spans_busy_and_critical_path(tmp_path):
    g = FakeGraph()
    spans = trace_analysis.task_spans(g, RECORDS)
    assert spans[1] == {"op": "TRSM_RLT", "start": 110, "end": 300, "items": 2, "item_ns": 280}
    path = trace_analysis.critical_path(g, spans)
    assert [p["task"] for p in path] == [0, 1, 3, 4]  # through the later-ending TRSM
    assert [p["wait"] for p in path] == [0, 10, 20, 30]
    busy = trace_analysis.busy_fraction(RECORDS)
    assert abs(busy - (100 + 90 + 190 + 145 + 80 + 90 + 50) / (3 * 500)) < 1e-12
    s = trace_analysis.dump_json(str(tmp_path / "t.json"), g, RECORDS)
    assert s["critical_path"]["tasks"] == 4
    assert abs(s["critical_path"]["per_op"]["POTRF"]["in_task_ms"] - 150e-6) < 1e-15
    out = json.load(open(tmp_path / "t.json"))
    assert len(out["records"]) == len(RECORDS) and set(out["tasks"]) == {"0", "1", "2", "3", "4"}


def test_busy_counts_overlapping_items_of_an_sm_once():
    # SM 0: an item whose C update (100..130) overlaps the next item (110..200), then a gap
    recs = [(0, 130, 0, 0, 0), (110, 200, 0, 1, 0), (250, 300, 0, 2, 0), (0, 300, 1, 3, 0)]
    assert abs(trace_analysis.busy_fraction(recs) - (250 + 300) / (2 * 300)) < 1e-12


def test_op_breakdown_of_a_traced_run():
    from mustard_b200 import profile_cases

    class Traced(FakeGraph):
        def trace(self):
            return RECORDS

    out = profile_cases.op_breakdown(Traced())
    assert abs(out["span_ms"] - 500e-6) < 1e-15
    assert abs(out["busy"] - trace_analysis.busy_fraction(RECORDS)) < 1e-12
    ops = out["ops"]
    assert set(ops) == {"POTRF", "TRSM_RLT", "GEMM_NT"}
    assert ops["POTRF"]["items"] == 2 and ops["TRSM_RLT"]["items"] == 3 and ops["GEMM_NT"]["items"] == 2
    assert abs(sum(o["share"] for o in ops.values()) - 1.0) < 1e-12
    assert abs(ops["TRSM_RLT"]["sum_ms"] - (90 + 190 + 145) * 1e-6) < 1e-15


def test_busy_profile_bins_the_idle_time():
    # two SMs over [0, 100): SM 0 busy all the time, SM 1 only in [0, 50) (two overlapping items)
    recs = [(0, 100, 0, 1, 0), (0, 30, 1, 2, 0), (20, 50, 1, 2, 1)]
    prof = trace_analysis.busy_profile(recs, bins=4)
    assert prof == [1.0, 1.0, 0.5, 0.5]
    assert abs(sum(prof) / 4 - trace_analysis.busy_fraction(recs)) < 1e-12
    assert trace_analysis.busy_profile([], bins=4) == []
