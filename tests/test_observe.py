"""Display formatting (src/display.rs known answers) and the display /
assertion post-scan on the host, over oracle-simulated netlist designs."""
import io
import os

import numpy as np

import oracle_lib
import test_netlist_golden as golden
from jacquard_b200 import netlist, observe, vcd

HERE = os.path.dirname(os.path.abspath(__file__))


def test_format_known_answers():
    lits, specs = observe.parse_format_string("Counter = {8:>02h-u}\\n")
    assert lits == ["Counter = ", "\n"] and len(specs) == 1
    assert (specs[0].width, specs[0].radix, specs[0].signed) == (8, "h", False)
    assert observe.format_display_message("value = {8:>02h-u}", [255], [8]) == "value = ff"
    assert observe.format_display_message("Counter reached 5, data_in = {8:>02h-u}\\n",
                                          [0x42], [8]) == "Counter reached 5, data_in = 42\n"


def test_format_signed_padding_and_alignment():
    f = observe.format_display_message
    assert f("{8:d}", [0xFF], [8]) == "-1"          # signed by default
    assert f("{8:d-u}", [0xFF], [8]) == "255"
    assert f("[{8:>5d-u}]", [7], [8]) == "[    7]"
    assert f("[{8:^5b-u}]", [5], [8]) == "[ 101 ]"
    assert f("[{8:<5d-u}]", [7], [8]) == "[7]"      # left alignment pads nothing
    assert f("{4:h} and {4:h}", [1], [4]) == "1 and "  # more specs than arguments


def stimulus(n, reset_cycles=2, period=10):
    """clk / rst stimulus VCD for the display counter."""
    buf = io.StringIO()
    w = vcd.VcdWriter(buf)
    w.timescale(1, "ns")
    w.add_module("tb")
    w.add_module("dut")
    clk, rst = w.add_wire(1, "clk"), w.add_wire(1, "rst")
    w.upscope()
    w.upscope()
    w.enddefinitions()
    w.begin_dumpvars()
    for k in range(n):
        w.timestamp(k * period)
        w.change_scalar(clk, "0")
        w.change_scalar(rst, "1" if k < reset_cycles else "0")
        w.timestamp(k * period + period // 2)
        w.change_scalar(clk, "1")
    w.timestamp(n * period)
    w.change_scalar(clk, "0")
    w.flush()
    return buf.getvalue()


def simulate_oracle(nd, text):
    s = nd.design.build_script(num_blocks=1)
    ports = netlist.NetlistPorts(nd, s)
    r, snaps, ots = golden.parse(ports, s, text)
    st = np.ascontiguousarray(snaps).reshape(-1).copy()
    oracle_lib.simulate(s, st, snaps.shape[0] - 1, s.reg_io_state_size)
    return s, ports, st, snaps.shape[0] - 1


def test_display_counter_post_scan():
    with open(os.path.join(HERE, "golden", "display_counter.gv")) as f:
        nd = netlist.read_netlist(f.read())
    s, ports, st, cycles = simulate_oracle(nd, stimulus(14))
    disp = ports.display_positions(s)
    assert len(disp) == 1 and disp[0][2] == "count is {2:>02h-u}\\n" and disp[0][4] == [2]
    assert len(disp[0][3]) == 2  # the 30 constant MSG_ID bits have no position
    msgs, stats = observe.post_scan(st, cycles, s.reg_io_state_size, displays=disp)
    # the counter leaves reset and counts 0, 1, 2, 3, 0, ...: the display
    # fires every fourth cycle, formatting the first argument bit (counter[1])
    fired = [c for c, _, _ in msgs]
    assert len(fired) >= 2 and all(b - a == 4 for a, b in zip(fired, fired[1:]))
    assert all(m == "count is 01\n" for _, _, m in msgs)
    assert stats["assertion_failures"] == 0


def test_assert_fixture_post_scan():
    nd, s, ports = golden.build("assert_synth.gv")
    r, snaps, ots = golden.parse(ports, s, golden.read("assert_test.vcd"))
    st = np.ascontiguousarray(snaps).reshape(-1).copy()
    oracle_lib.simulate(s, st, snaps.shape[0] - 1, s.reg_io_state_size)
    asserts = ports.assertion_positions(s)
    assert len(asserts) == 1
    msgs, stats = observe.post_scan(st, snaps.shape[0] - 1, s.reg_io_state_size,
                                    assertions=asserts)
    assert msgs == []
    assert stats["assertion_failures"] == len(stats["fired"])
