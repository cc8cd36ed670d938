"""Device-side output transitions (jq_output_transitions) against the host
walk of the reference's writer, and the VCD-in / VCD-out flow on the plain
interpreter against the oracle's snapshots written by the host walk."""
import io

import numpy as np
import pytest
import torch

import cases
import oracle_lib
from jacquard_b200 import sim, state, vcd

pytestmark = pytest.mark.gpu


def host_transitions(snaps, first, num, xoff, aoff, pos, const):
    counts, outs, codes, arrs = [], [], [], []
    prev = [2] * len(pos)
    for s in range(first, first + num):
        n = 0
        for j, p in enumerate(pos):
            if p == vcd.U32_MAX:
                c = const[j]
            else:
                w = p >> 5
                c = int(snaps[s, w] >> (p & 31)) & 1
                if xoff and (int(snaps[s, xoff + w] >> (p & 31)) & 1):
                    c = 3
            if c != prev[j]:
                outs.append(j)
                codes.append(c)
                arrs.append(0 if (p == vcd.U32_MAX or not aoff) else int(snaps[s, aoff + (p >> 5)]) & 0xFFFF)
                n += 1
            prev[j] = c
        counts.append(n)
    return np.array(counts), np.array(outs), np.array(codes), np.array(arrs)


@pytest.mark.parametrize("n_out,words", [(5, 3), (300, 40), (1000, 64)])
def test_device_transitions_match_host_walk(n_out, words):
    rng = np.random.default_rng(n_out)
    nsnap, first, num = 50, 3, 40
    stride = 3 * words  # values | X | arrivals
    snaps = rng.integers(0, 1 << 32, size=(nsnap, stride), dtype=np.uint64).astype(np.uint32)
    # sparse X and slowly changing values so that both kinds of transitions occur
    snaps[:, words:2 * words] &= rng.integers(0, 1 << 32, size=(nsnap, words), dtype=np.uint64).astype(np.uint32)
    for s in range(1, nsnap):
        keep = rng.random(words) < 0.7
        snaps[s, :words][keep] = snaps[s - 1, :words][keep]
    pos = rng.integers(0, 32 * words, size=n_out).astype(np.uint32)
    pos[::7] = vcd.U32_MAX
    const = (rng.random(n_out) < 0.5).astype(np.uint32)
    dev = torch.from_numpy(snaps.reshape(-1).view(np.int32)).cuda()
    tr = vcd.device_transitions(dev, first, num, stride, pos, out_const=const, xmask_offset=words,
                                arrival_offset=2 * words)
    counts, outs, codes, arrs = host_transitions(snaps, first, num, words, 2 * words, pos.tolist(),
                                                 const.tolist())
    assert np.array_equal(tr["counts"], counts)
    assert np.array_equal(tr["offsets"], np.concatenate([[0], np.cumsum(counts)]))
    assert np.array_equal(tr["outputs"], outs)
    assert np.array_equal(tr["codes"], codes)
    assert np.array_equal(tr["arrivals"], arrs)


@pytest.mark.parametrize("kind,nb,split,xprop", [("tiny", 8, (5,), False), ("sram", 16, (8,), True)])
def test_vcd_in_simulate_vcd_out_matches_oracle(kind, nb, split, xprop):
    d = cases.design(kind)
    s = cases.script(kind, nb, split, xprop=xprop)
    ports = vcd.DesignPorts(d, s)
    vals = state.stimulus_inputs(s, d, 40, seed=9, p_toggle=0.3, reset_cycles=3)
    buf = io.StringIO()
    vcd.write_stimulus_vcd(buf, ports, vals, s.input_layout, d.clock_flag_pin, period=10)
    text = buf.getvalue()
    got_text, dev_states = vcd.simulate_vcd(s, ports, text, xprop_all_x=xprop)

    # the same flow with the oracle and the reference writer's host walk
    r = vcd.VcdReader(text)
    _, sc = vcd.auto_detect_vcd_scope(r.scopes, ["clk"])
    snaps, ots = vcd.parse_input_vcd(r, vcd.match_vcd_inputs(sc, ports.input_pins), ports.input_pos,
                                     ports.clock_pins, s.reg_io_state_size)
    rio = s.reg_io_state_size
    host = snaps
    if xprop:
        host = state.expand_states_for_xprop(snaps, s)
        host[0, rio:] = state.xmask_all_state_x(s)
    eff = host.shape[1]
    st = np.ascontiguousarray(host).reshape(-1).copy()
    n_sram = max(1, s.sram_storage_size)
    oracle_lib.simulate(s, st, host.shape[0] - 1, eff, sram=np.zeros(n_sram, np.uint32),
                        sram_x=np.full(n_sram, 0xFFFFFFFF, np.uint32))
    assert np.array_equal(sim.dev_to_u32(dev_states), st)
    if xprop:
        values, xmask = state.split_xprop_states(st, rio)
        values, xmask = values.reshape(-1), xmask.reshape(-1)
    else:
        values, xmask = st, None
    out = io.StringIO()
    w = vcd.VcdWriter(out)
    w.timescale(*r.timescale)
    w.add_module("gem_top_module")
    out2vcd = ports.out2vcd(w, s)
    w.upscope()
    w.enddefinitions()
    w.begin_dumpvars()
    vcd.write_output_vcd(w, out2vcd, ots, values, xmask)
    assert got_text == out.getvalue()
    assert sum(line.startswith("#") for line in got_text.splitlines()) == len(ots) - 1


@pytest.mark.parametrize("gv,stim,want", [("dff_test_synth.gv", "dff_test.vcd", "dff_test_output.vcd"),
                                          ("assert_synth.gv", "assert_test.vcd", "assert_test_output.vcd")])
def test_reference_fixtures_on_the_gpu(gv, stim, want):
    """The reference's netlist + stimulus fixtures through the plain
    interpreter and the device transition walk: the reference's output VCD."""
    import test_netlist_golden as golden
    from jacquard_b200 import netlist, observe
    nd = netlist.read_netlist(golden.read(gv))
    s = nd.design.build_script(num_blocks=1)
    ports = netlist.NetlistPorts(nd, s)
    text, dev = vcd.simulate_vcd(s, ports, golden.read(stim))
    assert text.strip() == golden.read(want).strip()
    # assertion post-scan: device probe == host probe over the same snapshots
    rio = s.reg_io_state_size
    cycles = dev.numel() // rio - 1
    host = sim.dev_to_u32(dev)
    asserts = ports.assertion_positions(s)
    if asserts:
        assert observe.device_post_scan(dev, cycles, rio, assertions=asserts) == \
            observe.post_scan(host, cycles, rio, assertions=asserts)


def test_display_post_scan_on_the_gpu():
    import os
    import test_observe
    from jacquard_b200 import netlist, observe
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "display_counter.gv")) as f:
        nd = netlist.read_netlist(f.read())
    s = nd.design.build_script(num_blocks=1)
    ports = netlist.NetlistPorts(nd, s)
    _, dev = vcd.simulate_vcd(s, ports, test_observe.stimulus(30))
    rio = s.reg_io_state_size
    cycles = dev.numel() // rio - 1
    disp = ports.display_positions(s)
    got = observe.device_post_scan(dev, cycles, rio, displays=disp)
    want = observe.post_scan(sim.dev_to_u32(dev), cycles, rio, displays=disp)
    assert got == want and len(got[0]) >= 5
