"""Setup/hold violation drain and timing report.

This restates the reference's host side of the timed path:
- the event-buffer drain: process_events, src/event_buffer.rs:254-390,
  violation arms only;
- the word-to-DFF resolver: WordSymbolMap, src/flatten.rs:128-181 and
  :1852-1879;
- the JSON timing report accumulator: src/timing_report.rs, ReportBuilder
  and TimingReport.

CUDA never wired this in the reference; it only existed on Metal. Here the
plain interpreter's status entry point takes an event buffer of any capacity,
and `run_timed` drains it window by window.
"""
import json

import numpy as np

SCHEMA_VERSION = "1.1.0"
EVENT_SETUP, EVENT_HOLD = 4, 5
DEFAULT_MAX_VIOLATIONS = 100_000


class WordSymbolMap:
    """State word -> DFF sites ((name, bit) sorted by bit)."""

    def __init__(self, word_to_dffs):
        self.word_to_dffs = word_to_dffs

    @classmethod
    def from_positions(cls, dff_data_pos, names=None):
        """dff_data_pos[i] = state bit position of DFF i's D (0xFFFFFFFF = none)."""
        m = {}
        for i, pos in enumerate(np.asarray(dff_data_pos).tolist()):
            if pos == 0xFFFFFFFF:
                continue
            name = names[i] if names is not None else f"dff[{i}]"
            m.setdefault(pos // 32, []).append((name, pos % 32))
        for v in m.values():
            v.sort(key=lambda x: x[1])
        return cls(m)

    def describe_word(self, word_id, max_names=4):
        dffs = self.word_to_dffs.get(word_id)
        if not dffs:
            return f"<no DFF in word> [word={word_id}]"
        total = len(dffs)
        shown = min(total, max(1, max_names))
        parts = [f"{n}[bit {b}]" for n, b in dffs[:shown]]
        if total > shown:
            parts.append(f"+{total - shown} more")
        return f"{', '.join(parts)} [word={word_id}]"

    def num_sites(self):
        return sum(len(v) for v in self.word_to_dffs.values())

    def num_words(self):
        return len(self.word_to_dffs)


def _s32(u):
    u = int(u) & 0xFFFFFFFF
    return u - (1 << 32) if u & 0x80000000 else u


class ReportBuilder:
    """Per-word aggregates, top-N worst slacks, bounded violation list."""

    def __init__(self, metadata, worst_slack_n=10, max_violations=DEFAULT_MAX_VIOLATIONS):
        self.metadata = dict(metadata)
        self.violations = []
        self.per_word = {}
        self.worst = {"setup": [], "hold": []}
        self.n = max(1, worst_slack_n)
        self.max_violations = max_violations
        self.truncated = 0

    def _worst_push(self, kind, v):
        items = self.worst[kind]
        if len(items) < self.n:
            items.append(v)
            return
        idx = max(range(len(items)), key=lambda i: items[i]["slack_ps"])
        if v["slack_ps"] < items[idx]["slack_ps"]:
            items[idx] = v

    def observe(self, v):
        self._worst_push(v["kind"], v)
        e = self.per_word.setdefault(v["word_id"], {
            "word_id": v["word_id"], "site": v["site"], "setup_violations": 0,
            "hold_violations": 0, "worst_setup_slack_ps": None, "worst_hold_slack_ps": None,
            "worst_arrival_ps": None})
        k = v["kind"]
        e[f"{k}_violations"] += 1
        key = f"worst_{k}_slack_ps"
        e[key] = v["slack_ps"] if e[key] is None else min(e[key], v["slack_ps"])
        e["worst_arrival_ps"] = v["arrival_ps"] if e["worst_arrival_ps"] is None else \
            max(e["worst_arrival_ps"], v["arrival_ps"])
        if self.max_violations is not None and len(self.violations) >= self.max_violations:
            self.truncated += 1
        else:
            self.violations.append(v)

    def finalize(self, cycles_run, stats):
        md = dict(self.metadata)
        md["cycles_run"] = cycles_run
        st = dict(stats)
        st["violations_truncated"] = self.truncated
        per_word = sorted(self.per_word.values(),
                          key=lambda e: (-(e["setup_violations"] + e["hold_violations"]), e["word_id"]))
        worst = {k: sorted(v, key=lambda r: (r["slack_ps"], r["cycle"])) for k, v in self.worst.items()}
        return {"schema_version": SCHEMA_VERSION, "metadata": md, "stats": st,
                "violations": self.violations, "per_word": per_word, "worst_slack": worst}


def process_events(events, count, capacity, stats, builder=None, resolver=None):
    """Drain one buffer's violation records into `stats` (and `builder`).

    events: (n, 8) u32 records; count: the buffer's counter, which counts
    every event, dropped ones included.  The reference counts
    `count - MAX_EVENTS` dropped events when it overflowed."""
    if count > capacity:
        stats["events_dropped"] += count - capacity
    for ev in np.asarray(events, dtype=np.uint32).reshape(-1, 8):
        et = int(ev[0])
        if et not in (EVENT_SETUP, EVENT_HOLD):
            continue
        word_id, slack, arr, cons = int(ev[4]), _s32(ev[5]), int(ev[6]), int(ev[7])
        kind = "setup" if et == EVENT_SETUP else "hold"
        stats[f"{kind}_violations"] += 1
        if builder is not None:
            builder.observe({"cycle": int(ev[2]), "kind": kind, "word_id": word_id,
                             "site": resolver(word_id) if resolver else f"word={word_id}",
                             "arrival_ps": arr, "constraint_ps": cons, "slack_ps": slack})


def count_events(events, count, capacity, stats, streams=None):
    """Vectorised drain of a buffer's violation records into `stats` (counts
    only; for the many records of batched runs).  With `streams`, also
    per-stream counts: stats['per_stream_setup'] / ['per_stream_hold'],
    arrays indexed by the records' stream field (`reserved`)."""
    if count > capacity:
        stats["events_dropped"] += count - capacity
    ev = np.asarray(events, dtype=np.uint32).reshape(-1, 8)
    setup = ev[:, 0] == EVENT_SETUP
    hold = ev[:, 0] == EVENT_HOLD
    stats["setup_violations"] += int(setup.sum())
    stats["hold_violations"] += int(hold.sum())
    if streams is not None:
        for kind, sel in (("setup", setup), ("hold", hold)):
            key = f"per_stream_{kind}"
            c = np.bincount(ev[sel, 3].astype(np.int64), minlength=streams)[:streams]
            stats[key] = stats.get(key, np.zeros(streams, np.int64)) + c
    return stats


def constraint_buffer(design, script, clock_ps, setup_ps, hold_ps, clock_arrival_ps):
    """Timing constraint buffer [clock_ps, per-word setup<<16 | hold] for every
    DFF of a design (build_timing_constraint_buffer, src/flatten.rs:1891-1924,
    with the clock-arrival fold of :97-123): per-DFF setup/hold/clock arrival
    arrays (or scalars), folded to the per-word minimum."""
    import ctypes
    from .frontend import _lib
    n = int(design.num_dffs)
    su = np.broadcast_to(np.asarray(setup_ps, np.uint16), (n,)).copy()
    ho = np.broadcast_to(np.asarray(hold_ps, np.uint16), (n,)).copy()
    ca = np.broadcast_to(np.asarray(clock_arrival_ps, np.int16), (n,)).copy()
    pos = np.ascontiguousarray(script.dff_data_pos, dtype=np.uint32)
    out = np.zeros(script.reg_io_state_size, np.uint32)
    clk = ctypes.c_uint32()
    vp = ctypes.c_void_p
    rc = _lib().jqf_constraint_buffer(ctypes.c_uint32(script.reg_io_state_size),
                                      ctypes.c_uint64(clock_ps), ctypes.c_size_t(n),
                                      su.ctypes.data_as(vp), ho.ctypes.data_as(vp),
                                      ca.ctypes.data_as(vp), pos.ctypes.data_as(vp),
                                      ctypes.byref(clk), out.ctypes.data_as(vp))
    if rc:
        raise ValueError("constraint buffer: bad arguments")
    return np.concatenate([[np.uint32(clk.value)], out]).astype(np.uint32)


def new_stats():
    return {"setup_violations": 0, "hold_violations": 0, "events_dropped": 0}


def run_timed(ds, states, cycles, state_size, sram, sram_x, constraints, window, capacity,
              arrival_state_offset, builder=None, resolver=None, stream=None, first_cycle=0,
              stats=None, events=None):
    """Timed simulation in windows of `window` cycles on the plain interpreter;
    each window's event buffer is drained into the stats and report.  `states`
    holds the (cycles+1) snapshots on the device; events are numbered from
    `first_cycle`.  `stats` (accumulated) and `events` (a buffer of
    `capacity` records) may be passed in to reuse them.  Returns the stats."""
    import torch
    from . import sim
    stats = new_stats() if stats is None else stats
    ev = sim.new_event_buffer(capacity, device=states.device) if events is None else events
    for c0 in range(0, cycles, window):
        n = min(window, cycles - c0)
        ev[:2].zero_()
        view = states[c0 * state_size:]
        sim.simulate(ds, view, n, state_size, sram, sram_x, constraints=constraints, events=ev,
                     event_capacity=capacity, arrival_state_offset=arrival_state_offset,
                     first_cycle=first_cycle + c0, stream=stream)
        rc = sim.status(stream)
        if rc not in (0,):
            raise RuntimeError(sim.lib().jq_strerror(rc).decode())
        recs, count, _ = sim.read_events(ev)
        process_events(recs, count, capacity, stats, builder, resolver)
    torch.cuda.synchronize()
    return stats


def write_report(report, path):
    with open(path, "w") as f:
        json.dump(report, f, indent=2)
