"""Violation drain and timing report (restates src/event_buffer.rs:254-390,
src/timing_report.rs, WordSymbolMap of src/flatten.rs:128-181)."""
import numpy as np

from jacquard_b200 import timing


def ev(kind, cycle, word, slack, arr, cons):
    return [kind, word, cycle, 0, word, slack & 0xFFFFFFFF, arr, cons]


def test_describe_word_formats():
    m = timing.WordSymbolMap({3: [("a", 0), ("b", 5), ("c", 9)]})
    assert m.describe_word(3, 2) == "a[bit 0], b[bit 5], +1 more [word=3]"
    assert m.describe_word(3, 8) == "a[bit 0], b[bit 5], c[bit 9] [word=3]"
    assert m.describe_word(7) == "<no DFF in word> [word=7]"
    assert m.num_sites() == 3 and m.num_words() == 1


def test_word_symbol_map_from_positions():
    m = timing.WordSymbolMap.from_positions([33, 0xFFFFFFFF, 32, 5], names=["x", "y", "z", "w"])
    assert m.word_to_dffs[1] == [("z", 0), ("x", 1)]
    assert m.word_to_dffs[0] == [("w", 5)]


def test_process_events_counts_and_dropped():
    st = timing.new_stats()
    evs = np.array([ev(4, 1, 2, -100, 900, 200), ev(5, 1, 3, -40, 10, 50), [2, 0, 0, 0, 0, 0, 0, 0]],
                   np.uint32)
    b = timing.ReportBuilder({"clock_period_ps": 1000})
    timing.process_events(evs, 1030, 1024, st, b)
    assert st == {"setup_violations": 1, "hold_violations": 1, "events_dropped": 6}
    r = b.finalize(10, st)
    assert r["violations"][0]["slack_ps"] == -100 and r["violations"][1]["kind"] == "hold"
    assert r["metadata"]["cycles_run"] == 10 and r["stats"]["violations_truncated"] == 0


def test_worst_slack_top_n_and_truncation():
    b = timing.ReportBuilder({}, worst_slack_n=2, max_violations=3)
    for i, s in enumerate([-5, -50, -1, -70, -20]):
        b.observe({"cycle": i, "kind": "setup", "word_id": i % 2, "site": "s",
                   "arrival_ps": 100 + i, "constraint_ps": 30, "slack_ps": s})
    r = b.finalize(5, timing.new_stats())
    assert [v["slack_ps"] for v in r["worst_slack"]["setup"]] == [-70, -50]
    assert len(r["violations"]) == 3 and r["stats"]["violations_truncated"] == 2
    pw = {p["word_id"]: p for p in r["per_word"]}
    assert pw[0]["setup_violations"] == 3 and pw[0]["worst_setup_slack_ps"] == -20
    assert pw[1]["worst_setup_slack_ps"] == -70 and pw[1]["worst_arrival_ps"] == 103
    assert [p["word_id"] for p in r["per_word"]] == [0, 1]
