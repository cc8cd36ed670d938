"""VCD stimulus parsing and waveform writing (jacquard_b200.vcd), on the
host: the reference's timed-writer known-answer tests
(src/sim/vcd_io.rs:1336-1500), value-change and X encoding of the plain
writer, header and input matching, and stimulus round trips through the
parser on a generated design."""
import io

import numpy as np
import pytest

import cases
from jacquard_b200 import state, vcd


def timed_output(states, arrivals, ots, out2vcd_pos, timescale):
    buf = io.StringIO()
    w = vcd.VcdWriter(buf)
    w.timescale(*timescale)
    w.add_module("test")
    codes = [w.add_wire(1, name) for name in ("A", "B")[:len(out2vcd_pos)]]
    w.upscope()
    w.enddefinitions()
    w.begin_dumpvars()
    out2vcd = [(2 + 2 * i, pos, codes[i]) for i, pos in enumerate(out2vcd_pos)]
    vcd.write_output_vcd_timed(w, out2vcd, ots, states, arrivals, timescale=timescale)
    return buf.getvalue()


def test_timed_writer_offsets_transitions_by_arrival():
    # two outputs at bits 0 and 32 flip at the 10000 ps edge, arrivals 350 / 885
    text = timed_output([0, 0, 1, 1], [0, 0, 350, 885], [(0, 0), (2, 10000)], [0, 32], (1, "ps"))
    assert "#10350" in text and "#10885" in text and "#0" in text
    assert text.index("#10350") < text.index("#10885")


def test_timed_writer_rounds_half_away_from_zero():
    # 500 ps at a 1 ns timescale is 0.5 units -> 1: transition at #11
    text = timed_output([0, 1], [0, 500], [(0, 0), (1, 10)], [0], (1, "ns"))
    assert "#11" in text


def test_timed_writer_zero_arrival_stays_at_edge():
    text = timed_output([0, 1], [0, 0], [(0, 0), (1, 5000)], [0], (1, "ps"))
    assert "#5000" in text


def body_changes(text):
    """[(timestamp, [(code, value)])] of a written VCD body."""
    r = vcd.VcdReader(text)
    out = []
    for tok in r.tokens():
        if tok[0] == "t":
            out.append((tok[1], []))
        else:
            out[-1][1].append((tok[1], tok[2]))
    return out


def test_plain_writer_emits_changes_only_and_x():
    buf = io.StringIO()
    w = vcd.VcdWriter(buf)
    w.timescale(1, "ns")
    w.add_module("top")
    a, b, c = w.add_wire(1, "a"), w.add_wire(1, "b"), w.add_wire(1, "k")
    w.upscope()
    w.enddefinitions()
    w.begin_dumpvars()
    out2vcd = [(2, 0, a), (4, 33, b), (1, vcd.U32_MAX, c)]  # c: constant aigpin 1
    # 4 snapshots of 2 value words and their X words
    vals = np.array([[0, 0], [1, 2], [1, 2], [0, 0]], np.uint32).reshape(-1)
    xm = np.array([[0, 0], [0, 0], [1, 0], [0, 0]], np.uint32).reshape(-1)
    ots = [(0, vcd.U64_MAX), (2, 10), (4, 20), (6, 30)]
    nx = vcd.write_output_vcd(w, out2vcd, ots, vals, xm)
    got = body_changes(buf.getvalue())
    assert got == [(10, [(a, "1"), (b, "1"), (c, "1")]),
                   (20, [(a, "x")]),
                   (30, [(a, "0"), (b, "0")])]
    assert nx == 1


def test_reader_header_vectors_and_scope_detection():
    text = """$timescale 10ps $end
$scope module tb $end
$scope module dut $end
$var wire 1 ! clk $end
$var wire 4 " data [3:0] $end
$var wire 3 # sel $end
$upscope $end
$upscope $end
$enddefinitions $end
#0
0!
b101 "
b1 #
#5
1!
"""
    r = vcd.VcdReader(text)
    assert r.timescale == (10, "ps")
    path, sc = vcd.auto_detect_vcd_scope(r.scopes, ["clk", "data", "sel"])
    assert path == "tb/dut"
    pins = {("clk", None): "c", **{("data", i): f"d{i}" for i in range(4)},
            **{("sel", i): f"s{i}" for i in range(3)}}
    m = vcd.match_vcd_inputs(sc, pins)
    # [3:0] and an unindexed vector are both most significant first
    assert m[('"', 0)] == "d3" and m[('"', 3)] == "d0"
    assert m[("#", 0)] == "s2" and m[("#", 2)] == "s0"
    toks = list(r.tokens())
    # vector values are used as written (no extension to the variable width)
    assert ("v", '"', "101") in toks and ("v", "#", "1") in toks


@pytest.mark.parametrize("kind,nb,split", [("tiny", 8, (5,)), ("sram", 16, (8,))])
def test_stimulus_round_trip(kind, nb, split):
    d = cases.design(kind)
    s = cases.script(kind, nb, split)
    ports = vcd.DesignPorts(d, s)
    vals = state.stimulus_inputs(s, d, 12, seed=5, p_toggle=0.4, reset_cycles=2)
    buf = io.StringIO()
    vcd.write_stimulus_vcd(buf, ports, vals, s.input_layout, d.clock_flag_pin, period=10)
    r = vcd.VcdReader(buf.getvalue())
    _, sc = vcd.auto_detect_vcd_scope(r.scopes, ["clk"])
    m = vcd.match_vcd_inputs(sc, ports.input_pins)
    snaps, ots = vcd.parse_input_vcd(r, m, ports.input_pos, ports.clock_pins, s.reg_io_state_size)
    want = state.pack_inputs(s, vals)
    assert np.array_equal(snaps[1:1 + want.shape[0]], want)
    # one written timestamp per rising edge after the first
    assert [t for _, t in ots[:3]] == [vcd.U64_MAX, 0, 5]
    assert [o for o, _ in ots] == [(k + 1) * s.reg_io_state_size for k in range(len(ots))]
    # the posedge flag is set only in the edge snapshots
    fpos = ports.clock_pins["clk"][0]
    assert not (snaps[0][fpos >> 5] >> (fpos & 31)) & 1


def test_max_clock_edges_stops_reading():
    d = cases.design("tiny")
    s = cases.script("tiny", 8, (5,))
    ports = vcd.DesignPorts(d, s)
    vals = state.stimulus_inputs(s, d, 12, seed=5, p_toggle=0.4)
    buf = io.StringIO()
    vcd.write_stimulus_vcd(buf, ports, vals, s.input_layout, d.clock_flag_pin)
    r = vcd.VcdReader(buf.getvalue())
    _, sc = vcd.auto_detect_vcd_scope(r.scopes, ["clk"])
    m = vcd.match_vcd_inputs(sc, ports.input_pins)
    snaps, ots = vcd.parse_input_vcd(r, m, ports.input_pos, ports.clock_pins, s.reg_io_state_size,
                                     max_clock_edges=4)
    assert len(ots) == 4 and snaps.shape[0] == 5
