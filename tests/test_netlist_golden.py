"""End-to-end parity with the reference's own simulation fixtures: a
gate-level aigpdk netlist read into a design, its stimulus VCD parsed into
snapshots, every cycle simulated by the oracle, and the output VCD written as
the reference writes it, compared byte for byte with the VCD the reference
produced (tests/golden/ref_fixtures, copied by make_ref_fixtures.py)."""
import io
import os

import numpy as np
import pytest

import oracle_lib
from jacquard_b200 import netlist, vcd

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_fixtures")
CASES = [("dff_test_synth.gv", "dff_test.vcd", "dff_test_output.vcd"),
         ("assert_synth.gv", "assert_test.vcd", "assert_test_output.vcd")]


def read(name):
    with open(os.path.join(FIX, name)) as f:
        return f.read()


def build(gv):
    nd = netlist.read_netlist(read(gv))
    s = nd.design.build_script(num_blocks=1)
    return nd, s, netlist.NetlistPorts(nd, s)


def parse(ports, s, stim):
    r = vcd.VcdReader(stim)
    required = sorted({name for name, _ in ports.input_pins})
    _, sc = vcd.auto_detect_vcd_scope(r.scopes, required)
    m = vcd.match_vcd_inputs(sc, ports.input_pins)
    snaps, ots = vcd.parse_input_vcd(r, m, ports.input_pos, ports.clock_pins, s.reg_io_state_size)
    return r, snaps, ots


def write(ports, s, r, ots, states):
    out = io.StringIO()
    w = vcd.VcdWriter(out)
    w.timescale(*r.timescale)
    w.add_module("gem_top_module")
    out2vcd = ports.out2vcd(w, s)
    w.upscope()
    w.enddefinitions()
    w.begin_dumpvars()
    vcd.write_output_vcd(w, out2vcd, ots, states)
    return out.getvalue()


@pytest.mark.parametrize("gv,stim,want", CASES)
def test_reference_fixture_output_vcd(gv, stim, want):
    nd, s, ports = build(gv)
    r, snaps, ots = parse(ports, s, read(stim))
    st = np.ascontiguousarray(snaps).reshape(-1).copy()
    oracle_lib.simulate(s, st, snaps.shape[0] - 1, s.reg_io_state_size)
    got = write(ports, s, r, ots, st)
    assert got.strip() == read(want).strip()


def test_netlist_cells_and_ports():
    nd, s, ports = build("assert_synth.gv")
    kinds = nd.design.kind
    assert int(nd.design.num_dffs) == 9
    assert sorted(k for k, _ in nd.input_pins) == sorted(["clk", "rst"] + ["data_in"] * 4)
    assert len(nd.clock_flags) == 1 and len(nd.assertions) == 1
    assert [lab for _, lab in ports.outputs] == ["data_out[3]", "data_out[2]", "data_out[1]",
                                                 "data_out[0]", "overflow_flag"]
    assert (kinds == 1).sum() == nd.design.num_and
