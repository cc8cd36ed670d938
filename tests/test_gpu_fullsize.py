"""Parity at the benchmark's full size: the 2M-gate SoC design (2^21 clustered
ANDs + reset gates, depth 80, 200k DFFs, 16 SRAMs 1024x32, X-propagation,
every DFF and SRAM bit X at start), scripted as the benchmark scripts it
(148 blocks, level split every 4 levels, 6000-gate partitions).

- The batched interpreter over 256 streams against the plain interpreter run
  stream by stream, every snapshot and the SRAM contents of every stream; two
  of the streams also against the oracle.
- The timed path on the same netlist with per-pin delays U[20,200] ps, setup
  30 ps / hold 10 ps, a 10 ns clock and per-DFF clock arrival U[0,300] ps:
  snapshots (values, X, arrivals) and the violation multiset against the
  oracle, window by window.
"""
import os

import numpy as np
import pytest
import torch

import cases
import oracle_lib
from jacquard_b200 import batched, frontend, sim, state

pytestmark = pytest.mark.gpu

SPLIT = tuple(range(4, 80, 4))
CYCLES = 12
LANES = 8
THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def soc():
    d = frontend.Design(frontend.soc_params(seed=2, n_clusters=512, n_dff=200_000, n_sram=16))
    s = d.build_script(num_blocks=148, level_split=SPLIT, xprop=True, target_cone=6000)
    return d, s


def stream_inputs(s, d, k, cycles):
    vals = state.stimulus_inputs(s, d, cycles, seed=500 + k, p_toggle=0.25, reset_cycles=2)
    return state.pack_inputs(s, vals)  # (cycles+1, rio)


def stream_snapshots(s, packed, tmpl, x0):
    rio = s.reg_io_state_size
    v = np.empty((packed.shape[0], 2 * rio), np.uint32)
    v[:, :rio] = packed
    v[:, rio:] = tmpl
    v[0, rio:] = x0
    return v


def stream_of(rec, k):
    """Per-stream words (C, sig/32) of lane-major records (C, lanes, sig), on the device."""
    lane, bit = divmod(k, 32)
    c, _, sig = rec.shape
    bits = ((rec[:, lane, :] >> bit) & 1).to(torch.int64).view(c, sig // 32, 32)
    return (bits << torch.arange(32, device=rec.device)).sum(-1)


def check_256_streams(d, s, packed, cycles, po_sig=None, per_item=0):
    """The batched interpreter over 256 streams (per-stream packed inputs
    `packed[k]`, (cycles+1, rio)) against the plain interpreter stream by
    stream: every snapshot (values and X) and the SRAM contents of every
    stream, the recorded outputs when `po_sig` is given; the first and last
    streams also against the oracle."""
    rio = s.reg_io_state_size
    eff = 2 * rio
    streams = 32 * LANES
    tmpl = state.xmask_template(s)
    x0 = state.xmask_all_state_x(s)
    B = batched.BatchedSim(s, LANES, record=True, po_signals=po_sig, lanes_per_item=per_item)
    words = batched.input_words(s)
    stim = batched.to_batched(np.stack([p[:, :words] for p in packed]))  # (C+1, lanes, in_sigs)
    snap0 = np.zeros((LANES, B.sig), np.uint32)
    xbits = ((x0[:, None] >> np.arange(32, dtype=np.uint32)) & 1).reshape(-1).astype(bool)
    snap0[:, rio * 32:] = np.where(xbits, np.uint32(0xFFFFFFFF), np.uint32(0))[None, :]
    snap0[:, :B.in_sigs] = stim[0]
    B.load_state(snap0)
    B.reset_sram(x=True)
    dstim = torch.from_numpy(np.ascontiguousarray(stim).reshape(-1).view(np.int32)).cuda()
    rec = torch.zeros((cycles + 1, LANES, B.sig), dtype=torch.int32, device="cuda")
    rec[0].copy_(torch.from_numpy(snap0.view(np.int32)))
    wave = None
    if po_sig is not None:
        wave = torch.zeros(cycles * len(po_sig) * LANES, dtype=torch.int32, device="cuda")
    B.run(dstim, cycles, record_buf=rec, wave=wave)
    assert B.status() == 0
    bsram = B.sram.view(streams, -1)
    bsram_x = B.sram_x.view(streams, -1)
    if wave is not None:  # recorded outputs = the output signals of each snapshot
        w = wave.view(cycles, len(po_sig), LANES)
        po = torch.tensor(np.asarray(po_sig, np.int64), device="cuda")
        assert torch.equal(w, rec[1:].index_select(2, po).transpose(1, 2))

    ds = sim.DeviceScript(s)
    n_sram = max(1, s.sram_storage_size)
    mask = torch.tensor(0xFFFFFFFF, dtype=torch.int64, device="cuda")
    oracle_streams = {0, streams - 1}
    for k in range(streams):
        host = stream_snapshots(s, packed[k], tmpl, x0)
        st = sim.u32_to_dev(host.reshape(-1))
        sram = torch.zeros(n_sram, dtype=torch.int32, device="cuda")
        sram_x = torch.full((n_sram,), -1, dtype=torch.int32, device="cuda")
        sim.simulate(ds, st, cycles, eff, sram, sram_x)
        assert sim.status() == 0
        got = stream_of(rec, k)
        want = st.view(cycles + 1, eff).to(torch.int64) & mask
        assert torch.equal(got, want), f"stream {k}: batched != plain"
        assert torch.equal(bsram[k, :n_sram], sram), f"stream {k}: SRAM"
        assert torch.equal(bsram_x[k, :n_sram], sram_x), f"stream {k}: SRAM X"
        if k in oracle_streams:
            ost = host.reshape(-1).copy()
            osram = np.zeros(n_sram, np.uint32)
            osram_x = np.full(n_sram, 0xFFFFFFFF, np.uint32)
            oracle_lib.simulate(s, ost, cycles, eff, sram=osram, sram_x=osram_x, threads=THREADS)
            assert np.array_equal(sim.dev_to_u32(st), ost), f"stream {k}: plain != oracle"
            assert np.array_equal(sim.dev_to_u32(sram), osram)
            assert np.array_equal(sim.dev_to_u32(sram_x), osram_x)
    # the run did real work: DFF values known after reset and changing afterwards
    last = sim.dev_to_u32(st).reshape(cycles + 1, eff)
    assert np.count_nonzero(last[-1, :rio] != last[-2, :rio]) > 0


def test_batched_256_streams_match_plain_and_oracle(soc):
    d, s = soc
    packed = [stream_inputs(s, d, k, CYCLES) for k in range(32 * LANES)]
    check_256_streams(d, s, packed, CYCLES)


def test_benchmark_script_and_stimulus_256_streams_64_cycles():
    """The exact configuration bench.py times: its design, its script
    (148 blocks, balanced partitions, at most 148 per major stage, flat
    stages in the compact form, the cut bench.py picks), octet work items,
    its stimulus (16 reset cycles, then p_toggle 0.25, stream k seeded
    1000 + k) and one of its 64-cycle windows with the output waveform, 256
    streams: every snapshot of every stream against the plain interpreter,
    two streams against the oracle."""
    import bench
    d = bench.build_design()
    s, per_item = bench.default_batched_script(d)  # as bench.py builds it
    assert per_item == 8 and s.num_partitions <= 148 * s.num_major_stages
    assert int(s.features[:, 14].max()) <= 1  # flat stages: the compact form
    cycles = 64
    packed = []
    for k in range(32 * LANES):
        vals = state.stimulus_inputs(s, d, cycles, 1000 + k, bench.P_TOGGLE, bench.RESET_CYCLES)
        packed.append(state.pack_inputs(s, vals))
    check_256_streams(d, s, packed, cycles, po_sig=state.po_positions(s, d), per_item=per_item)


def test_timed_path_full_size_matches_oracle(soc):
    d, _ = soc
    from jacquard_b200 import timing
    rng = np.random.default_rng(3)
    n = d.num_pins + 1
    r = rng.integers(20, 201, size=n).astype(np.uint32)
    r[d.kind != 1] = 0
    d.set_delays(r, r)
    try:
        s = d.build_script(num_blocks=148, level_split=SPLIT, xprop=True, target_cone=6000)
    finally:
        zero = np.zeros(n, np.uint32)
        d.set_delays(zero, zero)
    s.enable_timing_arrivals()
    rio = s.reg_io_state_size
    cycles, window, cap = 16, 8, 1 << 18
    vals = state.stimulus_inputs(s, d, cycles, seed=77, p_toggle=0.25, reset_cycles=2)
    states = state.expand_states_for_arrivals(state.expand_states_for_xprop(state.pack_inputs(s, vals), s), s)
    states[0, rio:2 * rio] = state.xmask_all_state_x(s)
    states = np.ascontiguousarray(states)
    eff = states.shape[1]
    cons = cases.constraint_buffer_for(d, s)

    st = states.reshape(-1).copy()
    n_sram = max(1, s.sram_storage_size)
    osram = np.zeros(n_sram, np.uint32)
    osram_x = np.full(n_sram, 0xFFFFFFFF, np.uint32)
    want_stats = timing.new_stats()
    want = []
    for c0 in range(0, cycles, window):
        k = min(window, cycles - c0)
        ev, cnt = oracle_lib.simulate(s, st[c0 * eff:], k, eff, sram=osram, sram_x=osram_x,
                                      constraints=cons, event_cap=cap,
                                      arrival_state_offset=s.arrival_state_offset, threads=THREADS)
        recs = ev.view(np.uint32).reshape(-1, 8).copy()
        recs[:, 2] += c0
        want.append(recs)
        timing.process_events(recs, cnt, cap, want_stats)

    ds = sim.DeviceScript(s)
    dst = sim.u32_to_dev(states.reshape(-1))
    gs = sim.u32_to_dev(np.zeros(n_sram, np.uint32))
    gsx = sim.u32_to_dev(np.full(n_sram, 0xFFFFFFFF, np.uint32))
    b = timing.ReportBuilder({"clock_period_ps": 10_000}, max_violations=None)
    got_stats = timing.run_timed(ds, dst, cycles, eff, gs, gsx, sim.u32_to_dev(cons), window, cap,
                                 s.arrival_state_offset, builder=b)
    assert np.array_equal(sim.dev_to_u32(dst), st)
    assert np.array_equal(sim.dev_to_u32(gs), osram) and np.array_equal(sim.dev_to_u32(gsx), osram_x)
    assert got_stats == want_stats
    assert got_stats["hold_violations"] > 0 and got_stats["events_dropped"] == 0
    rep = b.finalize(cycles, got_stats)
    got_ms = sorted((v["cycle"], v["kind"], v["word_id"], v["slack_ps"], v["arrival_ps"])
                    for v in rep["violations"])
    want_ms = sorted((int(x[2]), "setup" if x[0] == 4 else "hold", int(x[4]), timing._s32(x[5]), int(x[6]))
                     for x in np.concatenate(want))
    assert got_ms == want_ms

