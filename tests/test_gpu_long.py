"""Runs of the full length the workloads name, bit-exact.

- The small CPU-runnable design (16,384 ANDs, depth 32, 1,024 DFFs, 32
  inputs / 32 outputs, no X) for its whole 4,096 cycles: the plain
  interpreter against the oracle on every snapshot; the batched interpreter
  over 64 streams against the plain interpreter on every snapshot of every
  stream, four streams also against the oracle.
- The 2M-gate SoC design as the benchmark scripts it, 256 streams, for
  100,000 cycles after a 16-cycle reset, in launch windows of 2,000 cycles:
  the last stream (lane word 7, bit 31) against the plain interpreter window
  by window (final state, every cycle's outputs, SRAM contents), and three
  16-cycle windows of the plain run against the oracle started from the
  plain run's own checkpoint (snapshot and SRAM contents at the window's
  start).
"""
import os

import numpy as np
import pytest
import torch

import cases
import oracle_lib
from jacquard_b200 import batched, sim, state

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def test_small_design_4096_cycles_plain_and_batched():
    cycles = 4096
    s = cases.script("small", 64, (8, 16, 24))
    states = cases.stimulus("small", s, cycles, seed=1)
    want = states.reshape(-1).copy()
    oracle_lib.simulate(s, want, cycles, states.shape[1], threads=THREADS)
    ds = sim.DeviceScript(s)
    st = sim.u32_to_dev(states.reshape(-1))
    sram = torch.zeros(1, dtype=torch.int32, device="cuda")
    sim.simulate(ds, st, cycles, states.shape[1], sram, sram)
    assert sim.status() == 0
    assert np.array_equal(sim.dev_to_u32(st), want)

    # batched: balanced flat partitions in lane-pair items, 64 streams
    sb = cases.script("small", 148, (8, 16, 24), target_parts=37)
    lanes = 2
    S = 32 * lanes
    snaps = np.stack([cases.stimulus("small", sb, cycles, seed=100 + k) for k in range(S)])
    eff = snaps.shape[-1]
    B = batched.BatchedSim(sb, lanes, record=True, lanes_per_item=2)
    bt = batched.to_batched(snaps)  # (cycles+1, lanes, sig)
    B.load_state(bt[0])
    B.reset_sram()
    stim = torch.from_numpy(np.ascontiguousarray(bt[:, :, :B.in_sigs]).reshape(-1).view(np.int32)).cuda()
    rec = torch.zeros((cycles + 1) * lanes * B.sig, dtype=torch.int32, device="cuda")
    rec[:lanes * B.sig].copy_(torch.from_numpy(np.ascontiguousarray(bt[0]).reshape(-1).view(np.int32)))
    B.run(stim, cycles, record_buf=rec)
    assert B.status() == 0
    got = batched.from_batched(rec.cpu().numpy().view(np.uint32).reshape(cycles + 1, lanes, B.sig), eff)
    dsb = sim.DeviceScript(sb)
    for k in range(S):
        pst = sim.u32_to_dev(snaps[k].reshape(-1))
        sim.simulate(dsb, pst, cycles, eff, sram, sram)
        assert sim.status() == 0
        plain = sim.dev_to_u32(pst).reshape(cycles + 1, eff)
        assert np.array_equal(got[k], plain), f"stream {k}: batched != plain"
        if k % 21 == 0:  # streams 0, 21, 42, 63
            o = snaps[k].reshape(-1).copy()
            oracle_lib.simulate(sb, o, cycles, eff, threads=THREADS)
            assert np.array_equal(plain.reshape(-1), o), f"stream {k}: plain != oracle"


class LaneStimulus:
    """Seeded stimulus generated window by window directly as lane words:
    every primary input toggles with probability 1/4 per cycle (the AND of
    two uniform random bits) in each stream, the clock posedge flag is 1,
    the reset input is 1 for the first `reset` snapshots, then 0."""

    def __init__(self, s, d, lanes, seed, reset):
        self.lay = np.asarray(s.input_layout)
        self.pos = state.input_positions(s)
        self.lanes, self.reset = lanes, reset
        self.rng = np.random.default_rng(seed)
        n = self.lay.size
        self.cur = self.rng.integers(0, 2**32, size=(n, lanes), dtype=np.uint32)
        self.fixed = {}
        self.fixed_cols = np.flatnonzero(self.lay == d.clock_flag_pin)
        self.reset_cols = np.flatnonzero(self.lay == d.reset_pin) if d.reset_pin else np.zeros(0, int)
        self.c = 0  # snapshot index of self.cur

    def _fix(self, v, c):
        v[self.fixed_cols] = 0xFFFFFFFF
        v[self.reset_cols] = 0xFFFFFFFF if c < self.reset else 0
        return v

    def window(self, cycles):
        """(cycles+1, n_in, lanes) input lane words of snapshots c .. c+cycles
        (the first row is the last row of the previous window)."""
        n = self.lay.size
        out = np.empty((cycles + 1, n, self.lanes), np.uint32)
        out[0] = self._fix(self.cur.copy(), self.c)
        for i in range(1, cycles + 1):
            t = (self.rng.integers(0, 2**32, size=(n, self.lanes), dtype=np.uint32)
                 & self.rng.integers(0, 2**32, size=(n, self.lanes), dtype=np.uint32))
            self.cur ^= t
            out[i] = self._fix(self.cur.copy(), self.c + i)
        self.c += cycles
        return out

    def batched_rows(self, w, in_sigs):
        """(rows, lanes, in_sigs) batched stimulus of a window."""
        rows = np.zeros((w.shape[0], self.lanes, in_sigs), np.uint32)
        rows[:, :, self.pos] = np.swapaxes(w, 1, 2)
        return rows

    @staticmethod
    def stream_values(w, k):
        """(rows, n_in) 0/1 inputs of stream k."""
        lane, bit = divmod(k, 32)
        return ((w[:, :, lane] >> np.uint32(bit)) & 1).astype(np.uint32)


def test_soc_100k_cycles_256_streams_windowed():
    import bench
    d = bench.build_design()
    s, per_item = bench.default_batched_script(d)  # as bench.py builds it
    lanes, W, total = 8, 2000, 100_000 + bench.RESET_CYCLES
    total -= total % W  # whole windows: 100,000 cycles
    streams = 32 * lanes
    rio = s.reg_io_state_size
    eff = 2 * rio
    tmpl = state.xmask_template(s)
    x0 = state.xmask_all_state_x(s)
    po = state.po_positions(s, d)
    gen = LaneStimulus(s, d, lanes, seed=2024, reset=bench.RESET_CYCLES)
    B = batched.BatchedSim(s, lanes, po_signals=po, lanes_per_item=per_item)
    checked = (streams - 1,)
    oracle_windows = {0, total // W // 2, total // W - 1}
    # snapshot 0 of the batched state and of the checked plain streams
    w = gen.window(W)
    snap0 = np.zeros((lanes, B.sig), np.uint32)
    xbits = ((x0[:, None] >> np.arange(32, dtype=np.uint32)) & 1).reshape(-1).astype(bool)
    snap0[:, rio * 32:] = np.where(xbits, np.uint32(0xFFFFFFFF), np.uint32(0))[None, :]
    snap0[:, :B.in_sigs] = gen.batched_rows(w[:1], B.in_sigs)[0]
    B.load_state(snap0)
    B.reset_sram(x=True)
    ds = sim.DeviceScript(s)
    n_sram = max(1, s.sram_storage_size)
    plain = {}
    for k in checked:
        v0 = np.empty(eff, np.uint32)
        v0[:rio] = state.pack_inputs(s, LaneStimulus.stream_values(w[:1], k))[0]
        v0[rio:] = x0
        plain[k] = dict(last=v0, sram=torch.zeros(n_sram, dtype=torch.int32, device="cuda"),
                        sram_x=torch.full((n_sram,), -1, dtype=torch.int32, device="cuda"))
    wave = torch.zeros(W * len(po) * lanes, dtype=torch.int32, device="cuda")
    po_t = torch.tensor(po, dtype=torch.int64, device="cuda")
    for wi in range(total // W):
        if wi:
            w = gen.window(W)
        rows = gen.batched_rows(w, B.in_sigs)
        dstim = torch.from_numpy(np.ascontiguousarray(rows).reshape(-1).view(np.int32)).cuda()
        B.run(dstim, W, wave=wave)
        assert B.status() == 0, f"window {wi}"
        final = B.final_state(W).view(lanes, B.sig)  # lane-major, on the device
        waves = wave.view(W, len(po), lanes)
        for k in checked:
            p = plain[k]
            host = np.empty((W + 1, eff), np.uint32)
            host[0] = p["last"]
            host[1:, :rio] = state.pack_inputs(s, LaneStimulus.stream_values(w[1:], k))
            host[1:, rio:] = tmpl
            if wi in oracle_windows:  # checkpoint for the oracle
                ck = (host.copy(), sim.dev_to_u32(p["sram"]), sim.dev_to_u32(p["sram_x"]))
            st = sim.u32_to_dev(host.reshape(-1))
            sim.simulate(ds, st, W, eff, p["sram"], p["sram_x"])
            assert sim.status() == 0
            snaps = st.view(W + 1, eff)
            p["last"] = sim.dev_to_u32(snaps[W])
            lane, bit = divmod(k, 32)
            fk = ((final[lane] >> bit) & 1).to(torch.int64).view(eff, 32)
            fk = (fk << torch.arange(32, device=fk.device)).sum(-1)
            assert torch.equal(fk, snaps[W].to(torch.int64) & 0xFFFFFFFF), \
                f"window {wi} stream {k}: final state"
            got_po = ((waves[:, :, lane] >> bit) & 1).to(torch.int64)
            sn = snaps[1:].to(torch.int64) & 0xFFFFFFFF
            want_po = (sn.index_select(1, po_t >> 5) >> (po_t & 31)) & 1
            assert torch.equal(got_po, want_po), f"window {wi} stream {k}: outputs"
            if wi in oracle_windows:
                oh, osram, osx = ck
                o = oh[:17].reshape(-1).copy()
                oracle_lib.simulate(s, o, 16, eff, sram=osram, sram_x=osx, threads=THREADS)
                assert np.array_equal(o.reshape(17, eff), sim.dev_to_u32(snaps[:17])), \
                    f"window {wi} stream {k}: plain != oracle"
    bs = B.sram.view(streams, -1)
    bsx = B.sram_x.view(streams, -1)
    for k in checked:
        assert torch.equal(bs[k, :n_sram], plain[k]["sram"])
        assert torch.equal(bsx[k, :n_sram], plain[k]["sram_x"])
