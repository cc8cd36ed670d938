"""Batched (bit-lane) interpreter vs the CPU oracle run stream by stream."""
import os

import numpy as np
import pytest
import torch

import cases
import oracle_lib
from jacquard_b200 import batched, state

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


@pytest.mark.parametrize("kind,nb,split,xprop,lanes,wo_slots,per_item,grid", [
    ("tiny", 8, (5,), False, 1, None, 0, 0),
    ("sram", 16, (8,), True, 2, None, 0, 0),     # lane pairs
    ("sram", 16, (8,), True, 2, None, 1, 0),     # single lanes, double-buffered tree
    ("sram", 16, (8,), True, 1, 256, 0, 0),      # single-buffered tree state
    ("sram", 16, (8,), True, 2, 256, 0, 0),      # lane pairs do not fit: single lanes
    ("tiny", 8, (5,), False, 4, None, 2, 0),
    ("soc_mini", 148, (20, 40, 60), True, 1, None, 0, 0),
    ("soc_mini", 148, (20, 40, 60), True, 2, None, 0, 0),
    # fewer CTAs than items: work tickets instead of one item per CTA
    ("soc_mini", 148, (20, 40, 60), True, 2, None, 0, 5),
    ("sram", 16, (8,), True, 2, None, 1, 3),
])
def test_batched_matches_oracle_per_stream(kind, nb, split, xprop, lanes, wo_slots, per_item,
                                           grid):
    check_batched(kind, cases.script(kind, nb, split, xprop=xprop), lanes, wo_slots, per_item, grid)


@pytest.mark.parametrize("kind,nb,split,parts,lanes,grid", [
    ("soc_mini", 148, (20, 40, 60), 37, 2, 0),   # one item per CTA per stage
    ("soc_mini", 148, (20, 40, 60), 37, 2, 5),   # tickets
    ("sram", 16, (8,), 4, 2, 0),
    # lane-pair barrier groups: 3 groups of uneven size (idle CTAs included)
    ("soc_mini", 148, (20, 40, 60), 37, 6, 0),
    ("soc_mini", 148, (20, 40, 60), 37, 8, 0),   # 4 groups of 37, as the benchmark
    ("soc_mini", 148, (20, 40, 60), 37, 8, 100),  # tickets: one barrier for all
])
def test_batched_balanced_partitions_match_oracle(kind, nb, split, parts, lanes, grid):
    """Balanced, flat partitions (every gate at tree level 1, the batched
    workload's script form) in lane-pair items."""
    s = cases.script(kind, nb, split, xprop=True, target_parts=parts)
    assert int(s.features[:, 14].max()) <= 1  # deepest tree level with a gate
    check_batched(kind, s, lanes, None, 2, grid)


SPLIT4 = tuple(range(4, 80, 4))  # the benchmark's level split (20 major stages)


@pytest.mark.parametrize("kind,nb,split,parts,lanes,grid", [
    ("soc_mini", 148, SPLIT4, 37, 8, 0),     # one octet item per CTA per stage
    ("soc_mini", 148, SPLIT4, 37, 16, 0),    # two octet groups, own barriers
    ("soc_mini", 148, SPLIT4, 37, 8, 7),     # tickets
    ("sram", 16, (8,), 16, 8, 0),            # SRAM ports and duplicates
])
def test_batched_octet_items_match_oracle(kind, nb, split, parts, lanes, grid):
    """Octet work items (8 lane words, the octet state layout, writeouts
    named in the tree slots) on balanced flat partitions, every stream
    against the oracle."""
    s = cases.script(kind, nb, split, xprop=True, target_parts=parts)
    check_batched(kind, s, lanes, None, 8, grid)


def test_octet_items_refuse_a_script_they_cannot_run():
    """Octet items need the compact form: a script in the tree form (deep
    boomerang stages) is refused on the host, before any launch."""
    s = cases.script("sram", 16, (8,), xprop=True)
    with pytest.raises(ValueError):
        batched.BatchedSim(s, 8, lanes_per_item=8)


class BatchedCase:
    """A batched run prepared on the device with its per-stream oracle
    results: launch() issues it (on any stream), verify() checks every
    snapshot and SRAM word of every stream."""

    def __init__(self, kind, s, lanes, wo_slots=None, per_item=0, grid=0, cycles=10, seed0=1000):
        xprop = s.xprop_enabled
        self.cycles, self.lanes, self.S = cycles, lanes, 32 * lanes
        snaps = np.stack([cases.stimulus(kind, s, cycles, seed=seed0 + k, x_init=xprop)
                          for k in range(self.S)])  # (S, cycles+1, eff)
        self.eff = snaps.shape[-1]
        self.want = snaps.copy()
        self.wsram = []
        for k in range(self.S):  # oracle, stream by stream
            st = self.want[k].reshape(-1).copy()
            sram = np.zeros(max(1, s.sram_storage_size), np.uint32)
            sram_x = np.full_like(sram, 0xFFFFFFFF)
            oracle_lib.simulate(s, st, cycles, self.eff, sram=sram, sram_x=sram_x, threads=THREADS)
            self.want[k] = st.reshape(cycles + 1, self.eff)
            self.wsram.append(sram)
        self.B = batched.BatchedSim(s, lanes, record=True, wo_slots=wo_slots,
                                    lanes_per_item=per_item, grid=grid)
        self.bt = batched.to_batched(snaps)  # (cycles+1, lanes, sig)
        B = self.B
        self.stim = torch.from_numpy(
            np.ascontiguousarray(self.bt[:, :, :B.in_sigs]).reshape(-1).view(np.int32)).cuda()
        self.rec = torch.zeros((cycles + 1) * B.sig * lanes, dtype=torch.int32, device="cuda")
        self.reset()

    def reset(self):
        B = self.B
        B.load_state(self.bt[0])
        B.reset_sram()
        self.rec.zero_()
        self.rec[: B.sig * self.lanes].copy_(
            torch.from_numpy(np.ascontiguousarray(self.bt[0]).reshape(-1).view(np.int32)))

    def launch(self, stream=None, barrier_timeout_cycles=0):
        self.B.run(self.stim, self.cycles, record_buf=self.rec, stream=stream,
                   barrier_timeout_cycles=barrier_timeout_cycles)

    def verify(self):
        B = self.B
        got = batched.from_batched(
            self.rec.cpu().numpy().view(np.uint32).reshape(self.cycles + 1, self.lanes, B.sig), self.eff)
        assert got.shape == self.want.shape
        for k in range(self.S):
            assert np.array_equal(got[k], self.want[k]), f"stream {k}"
        gs = B.sram.cpu().numpy().view(np.uint32).reshape(self.S, -1)
        for k in range(self.S):
            assert np.array_equal(gs[k][: self.wsram[k].size], self.wsram[k])


def check_batched(kind, s, lanes, wo_slots, per_item, grid):
    c = BatchedCase(kind, s, lanes, wo_slots, per_item, grid)
    c.launch()
    assert c.B.status() == 0
    c.verify()


def test_batched_launches_on_two_streams_overlap_safely():
    """Two batched launches on different streams, each on a few CTAs so both
    are resident at once: each takes its own barrier/ticket/status slot, and
    both match the oracle stream by stream."""
    a = BatchedCase("soc_mini", cases.script("soc_mini", 148, (20, 40, 60), xprop=True,
                                             target_parts=37), 2, per_item=2, grid=5)
    b = BatchedCase("sram", cases.script("sram", 16, (8,), xprop=True), 2, per_item=2, grid=4,
                    seed0=3000)
    torch.cuda.synchronize()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    a.launch(stream=s1)
    b.launch(stream=s2)
    assert a.B.status(s1) == 0 and b.B.status(s2) == 0
    a.verify()
    b.verify()


def test_batched_barrier_wait_that_runs_out_is_reported():
    """A grid-barrier wait limited to one SM clock runs out: the launch ends
    with JQ_ERR_BARRIER_TIMEOUT (script-chunk copies keep their own fixed
    limit, so no CTA leaves with a copy in flight), and a normal launch
    afterwards on the same context matches the oracle."""
    c = BatchedCase("soc_mini", cases.script("soc_mini", 148, (20, 40, 60), xprop=True,
                                             target_parts=37), 2, per_item=2)
    c.launch(barrier_timeout_cycles=1)
    assert c.B.status() == -3  # JQ_ERR_BARRIER_TIMEOUT
    c.reset()
    c.launch()
    assert c.B.status() == 0
    c.verify()


def test_lane_pairs_rejected_for_odd_lanes():
    s = cases.script("tiny", 8, (5,), xprop=False)
    B = batched.BatchedSim(s, 1, lanes_per_item=2)
    stim = None
    with pytest.raises(RuntimeError):
        B.run(stim, 1)


def test_layout_roundtrip():
    rng = np.random.default_rng(0)
    a = rng.integers(0, 2**32, size=(64, 3, 5), dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(batched.from_batched(batched.to_batched(a), 5), a)


@pytest.mark.parametrize("per_item", [0, 8])
def test_multi_design_single_launch_matches_oracle(per_item):
    """Designs of uneven size relocated into one script share one persistent
    launch, captured in a CUDA graph and replayed; every snapshot of every
    checked stream of every design equals the oracle's run of that design
    and stream alone, and so do the SRAM contents.  per_item 0: three
    designs on one lane word (every stream checked); 8: octet items on
    balanced partitions of two designs, 256 streams (every 17th checked)."""
    if per_item == 8:
        specs = [("sram", 16, (8,), 16), ("soc_mini", 148, SPLIT4, 37)]
        lanes, step = 8, 17
    else:
        specs = [("tiny", 8, (5,), 0), ("sram", 16, (8,), 0), ("soc_mini", 148, (20, 40, 60), 0)]
        lanes, step = 1, 1
    scripts = [cases.script(k, nb, sp, xprop=True, target_parts=tp) for k, nb, sp, tp in specs]
    cycles = 8
    S = 32 * lanes
    snaps = [np.stack([cases.stimulus(k, s, cycles, seed=500 + 37 * i + j, x_init=True)
                       for j in range(S)]) for i, ((k, _, _, _), s) in enumerate(zip(specs, scripts))]
    C = batched.CombinedScript(scripts)
    BC = batched.BatchedSim(C, lanes, record=True, lanes_per_item=per_item)
    bts = [batched.to_batched(sn) for sn in snaps]  # (cycles+1, lanes, sig_d)
    snap0 = C.combine_states([bt[0] for bt in bts])
    assert snap0.shape == (lanes, BC.sig)
    BC.load_state(snap0)
    BC.reset_sram()
    stim = np.concatenate([bt[:, :, :batched.input_words(s) * 32] for s, bt in zip(scripts, bts)], axis=-1)
    stim_d = torch.from_numpy(np.ascontiguousarray(stim).reshape(-1).view(np.int32)).cuda()
    rec = torch.zeros((cycles + 1) * lanes * BC.sig, dtype=torch.int32, device="cuda")
    rec[:lanes * BC.sig].copy_(torch.from_numpy(np.ascontiguousarray(snap0).reshape(-1).view(np.int32)))
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        BC.run(stim_d, cycles, record_buf=rec)
    g.replay()
    torch.cuda.synchronize()
    assert BC.status() == 0
    got_all = rec.cpu().numpy().view(np.uint32).reshape(cycles + 1, lanes, BC.sig)
    sram = BC.sram.cpu().numpy().view(np.uint32).reshape(S, -1)
    for d, s in enumerate(scripts):
        eff = snaps[d].shape[-1]
        got = batched.from_batched(C.design_state(d, got_all), eff)  # (S, cycles+1, eff)
        n_sram = max(1, s.sram_storage_size)
        for k in range(0, S, step):
            want = snaps[d][k].reshape(-1).copy()
            osram = np.zeros(n_sram, np.uint32)
            osram_x = np.full(n_sram, 0xFFFFFFFF, np.uint32)
            oracle_lib.simulate(s, want, cycles, eff, sram=osram, sram_x=osram_x, threads=THREADS)
            assert np.array_equal(got[k].reshape(-1), want), f"design {d} stream {k}"
            if s.sram_storage_size:
                b = C.sram_base[d]
                assert np.array_equal(sram[k, b:b + s.sram_storage_size], osram[:s.sram_storage_size])


@pytest.mark.parametrize("xprop,lanes,per_item,parts", [(False, 2, 2, 0), (True, 2, 2, 0),
                                                         (True, 1, 1, 0), (True, 2, 2, 4),
                                                         (True, 4, 2, 4), (True, 8, 8, 16)])
def test_batched_setup_hold_events_match_oracle_per_stream(xprop, lanes, per_item, parts):
    """Setup/hold checks in the batched interpreter, two launch windows of 12
    cycles: every stream's snapshots, and the multiset of (stream, event)
    records over all streams, equal the oracle's run of each stream with the
    same windows (per-block writeout arrivals restart with each launch)."""
    s = cases.script("sram", 16, (8,), xprop=xprop, timing_seed=9, target_parts=parts)
    cons = cases.constraint_buffer("sram", s, clock_ps=120, setup=30, hold=150)
    S, win, nwin = 32 * lanes, 12, 2
    cycles = win * nwin
    snaps = np.stack([cases.stimulus("sram", s, cycles, seed=700 + k, x_init=xprop)
                      for k in range(S)])
    eff = snaps.shape[-1]
    want_ev = []
    want = snaps.copy()
    for k in range(S):
        st = want[k].reshape(-1)
        sram = np.zeros(max(1, s.sram_storage_size), np.uint32)
        sram_x = np.full_like(sram, 0xFFFFFFFF)
        for w in range(nwin):
            ev, cnt = oracle_lib.simulate(s, st[w * win * eff:], win, eff, sram=sram, sram_x=sram_x,
                                          constraints=cons, event_cap=1 << 14)
            r = ev.view(np.uint32).reshape(-1, 8).copy()
            assert cnt == r.shape[0]
            r[:, 2] += w * win
            r[:, 3] = k
            want_ev.append(r)
    want_ev = np.concatenate(want_ev)
    assert set(want_ev[:, 0].tolist()) == {4, 5}

    B = batched.BatchedSim(s, lanes, record=True, lanes_per_item=per_item)
    tm = batched.Timing(s, cons, capacity=want_ev.shape[0] + 1024)
    bt = batched.to_batched(snaps)  # (cycles+1, lanes, sig)
    B.load_state(bt[0])
    B.reset_sram()
    got = []
    for w in range(nwin):
        rows = bt[w * win:(w + 1) * win + 1, :, :B.in_sigs]
        stim = torch.from_numpy(np.ascontiguousarray(rows).reshape(-1).view(np.int32)).cuda()
        rec = torch.zeros((win + 1) * B.sig * lanes, dtype=torch.int32, device="cuda")
        B.run(stim, win, record_buf=rec, timing=tm, first_cycle=w * win)
        assert B.status() == 0
        g = batched.from_batched(rec.cpu().numpy().view(np.uint32).reshape(win + 1, lanes, B.sig), eff)
        for k in range(S):
            assert np.array_equal(g[k][1:], want[k][w * win + 1:(w + 1) * win + 1]), f"window {w} stream {k}"
    recs, count, overflow = tm.read()
    assert overflow == 0 and count == want_ev.shape[0]
    assert sorted(map(tuple, recs.tolist())) == sorted(map(tuple, want_ev.tolist()))
