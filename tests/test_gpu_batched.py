"""Batched (bit-lane) interpreter vs the CPU oracle run stream by stream."""
import numpy as np
import pytest
import torch

import cases
import oracle_lib
from jacquard_b200 import batched, state

pytestmark = pytest.mark.gpu


def per_stream_states(kind, s, cycles, streams, x_init):
    out = []
    for k in range(streams):
        out.append(cases.stimulus(kind, s, cycles, seed=1000 + k, x_init=x_init))
    return np.stack(out)  # (S, cycles+1, eff)


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
])
def test_batched_balanced_partitions_match_oracle(kind, nb, split, parts, lanes, grid):
    """Balanced, flat partitions (every gate at tree level 1, the batched
    workload's script form) in lane-pair items."""
    s = cases.script(kind, nb, split, xprop=True, target_parts=parts)
    assert int(s.features[:, 14].max()) <= 1  # deepest tree level with a gate
    check_batched(kind, s, lanes, None, 2, grid)


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
            oracle_lib.simulate(s, st, cycles, self.eff, sram=sram, sram_x=sram_x)
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


def _batched_inputs(kind, s, cycles, lanes, seed0):
    S = 32 * lanes
    snaps = np.stack([cases.stimulus(kind, s, cycles, seed=seed0 + k, x_init=True) for k in range(S)])
    return batched.to_batched(snaps)  # (cycles+1, lanes, sig)


def test_multi_design_single_launch_matches_separate_runs():
    """Three designs of uneven size relocated into one script share one
    persistent launch; each design's state equals its own separate run."""
    specs = [("tiny", 8, (5,)), ("sram", 16, (8,)), ("soc_mini", 148, (20, 40, 60))]
    scripts = [cases.script(k, nb, sp, xprop=True) for k, nb, sp in specs]
    lanes, cycles = 1, 8
    bts = [_batched_inputs(k, s, cycles, lanes, 500 + 37 * i)
           for i, ((k, _, _), s) in enumerate(zip(specs, scripts))]
    finals = []
    for s, bt in zip(scripts, bts):
        B = batched.BatchedSim(s, lanes)
        B.load_state(bt[0])
        B.reset_sram()
        stim = torch.from_numpy(np.ascontiguousarray(bt[:, :, :B.in_sigs]).reshape(-1).view(np.int32)).cuda()
        B.run(stim, cycles)
        assert B.status() == 0
        finals.append(B.final_state(cycles).cpu().numpy().view(np.uint32).reshape(lanes, -1))
    C = batched.CombinedScript(scripts)
    BC = batched.BatchedSim(C, lanes)
    snap0 = C.combine_states([bt[0] for bt in bts])
    assert snap0.shape == (lanes, BC.sig)
    BC.load_state(snap0)
    BC.reset_sram()
    stim = np.concatenate([bt[:, :, :batched.input_words(s) * 32] for s, bt in zip(scripts, bts)], axis=-1)
    stim_d = torch.from_numpy(np.ascontiguousarray(stim).reshape(-1).view(np.int32)).cuda()
    # capture the launch in a CUDA graph and replay it
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        BC.run(stim_d, cycles)
    g.replay()
    torch.cuda.synchronize()
    assert BC.status() == 0
    got = BC.final_state(cycles).cpu().numpy().view(np.uint32).reshape(lanes, -1)
    for d, s in enumerate(scripts):
        assert np.array_equal(C.design_state(d, got), finals[d]), f"design {d}"
