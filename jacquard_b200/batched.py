"""Bit-lane batched interpreter: 32*lanes stimulus streams per launch.

Streams are bit-sliced: a lane word holds one signal of 32 streams.  Helpers
convert between per-stream snapshots (the reference layout) and the
signal-major batched layout; the kernel itself is jq_simulate_batched in
libjacquard_b200.so.
"""
import ctypes

import numpy as np
import torch

from . import sim
from ._native import load

vp = ctypes.c_void_p


class BatchArgs(ctypes.Structure):
    _fields_ = [("num_blocks", ctypes.c_size_t), ("num_major_stages", ctypes.c_size_t),
                ("blocks_start", vp), ("blocks_data", vp), ("lanes", ctypes.c_uint32),
                ("sram_data", vp), ("sram_xmask", vp), ("sram_words_per_stream", ctypes.c_size_t),
                ("num_cycles", ctypes.c_size_t), ("signals_per_snapshot", ctypes.c_size_t),
                ("state_a", vp), ("state_b", vp), ("stimulus", vp), ("input_signals", ctypes.c_size_t),
                ("input_regions", vp), ("n_input_regions", ctypes.c_uint32),
                ("po_signals", vp), ("n_po", ctypes.c_uint32), ("wave", vp), ("record", vp),
                ("wo_slots", ctypes.c_uint32), ("block_list", vp), ("block_list_start", vp),
                ("part_cycles", vp), ("part_base", vp), ("gr_sources", vp),
                ("grid", ctypes.c_size_t),
                ("barrier_timeout_cycles", ctypes.c_uint64), ("stream", vp),
                ("lanes_per_item", ctypes.c_uint32), ("x_interleaved", ctypes.c_int32),
                ("timing_constraints", vp), ("arrival_first", vp), ("arrival_steady", vp),
                ("events", vp), ("event_capacity", ctypes.c_uint32), ("first_cycle", ctypes.c_uint32)]


def lib():
    L = load("libjacquard_b200.so")
    if not getattr(L, "_jq_batched_typed", False):
        L.jq_simulate_batched.restype = ctypes.c_int
        L.jq_simulate_batched.argtypes = [ctypes.POINTER(BatchArgs)]
        L.jq_batched_status.restype = ctypes.c_int
        L.jq_batched_status.argtypes = [vp]
        L.jq_batched_max_blocks.restype = ctypes.c_int
        L.jq_batched_max_blocks.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(ctypes.c_size_t)]
        L.jq_batched_gr_words.restype = ctypes.c_size_t
        L.jq_batched_gr_words.argtypes = [ctypes.c_size_t]
        L.jq_batched_prepare.restype = ctypes.c_int
        L.jq_batched_prepare.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                                         ctypes.c_size_t, vp, vp, vp, vp]
        L.jq_batched_state_words.restype = ctypes.c_size_t
        L.jq_batched_state_words.argtypes = [ctypes.c_uint32, ctypes.c_size_t]
        for fn in (L.jq_batched_pack_state, L.jq_batched_unpack_state):
            fn.restype = ctypes.c_int
            fn.argtypes = [vp, ctypes.c_uint32, ctypes.c_size_t, ctypes.c_int32, vp, vp]
        L.jq_batched_oct_capacity.restype = ctypes.c_int
        L.jq_batched_oct_capacity.argtypes = [ctypes.POINTER(ctypes.c_uint32)]
        L.jq_batched_slot_need.restype = ctypes.c_int
        L.jq_batched_slot_need.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_size_t, vp, vp]
        L._jq_batched_typed = True
    return L


# (shift, mask) rounds of a 32x32 bit-matrix transpose by block swaps: the
# off-diagonal 16x16 blocks, then within each the 8x8 ones, down to single
# bits.
_T32_ROUNDS = ((16, 0x0000FFFF), (8, 0x00FF00FF), (4, 0x0F0F0F0F), (2, 0x33333333),
               (1, 0x55555555))


def _transpose32(x):
    """(..., 32) u32 -> (..., 32) u32 with bit i of out[..., b] = bit b of
    x[..., i] (a copy)."""
    x = np.array(x, dtype=np.uint32, copy=True)
    for j, m in _T32_ROUNDS:
        xr = x.reshape(x.shape[:-1] + (32 // (2 * j), 2, j))
        a, b = xr[..., 0, :], xr[..., 1, :]
        t = ((a >> np.uint32(j)) ^ b) & np.uint32(m)
        b ^= t
        a ^= t << np.uint32(j)
    return x


def octet_capacity():
    """64-byte tree slots an octet work item holds on the current device."""
    n = ctypes.c_uint32()
    rc = lib().jq_batched_oct_capacity(ctypes.byref(n))
    if rc:
        raise RuntimeError("jq_batched_oct_capacity: " + sim.lib().jq_strerror(rc).decode())
    return n.value


def to_batched(per_stream):
    """(streams, ..., words) u32 per-stream layout -> (..., lanes, words*32)
    lane-major lane words: word [l, signal] holds `signal` of streams
    32l..32l+31 (bit i = stream 32l+i).  streams must be a multiple of 32."""
    a = np.asarray(per_stream, dtype=np.uint32)
    S, W = a.shape[0], a.shape[-1]
    assert S % 32 == 0
    x = np.moveaxis(a.reshape((S // 32, 32) + a.shape[1:]), (0, 1), (-3, -1))  # (..., lanes, W, 32)
    y = _transpose32(x)
    return np.ascontiguousarray(y.reshape(y.shape[:-2] + (W * 32,)))


def from_batched(batched, words):
    """Inverse of to_batched: (..., lanes, sig) -> (streams, ..., words)."""
    b = np.asarray(batched, dtype=np.uint32)
    lanes = b.shape[-2]
    y = _transpose32(b.reshape(b.shape[:-1] + (words, 32)))         # (..., lanes, W, 32)
    y = np.moveaxis(y, (-3, -1), (0, 1))                            # (lanes, 32, ..., W)
    return np.ascontiguousarray(y.reshape((lanes * 32,) + y.shape[2:]))


def input_words(script):
    """Words of the input region (src/flatten.rs:1159-1166)."""
    n = len(script.input_layout)
    w = (n + 31) // 32
    if n == w * 32:
        w += 1
    return w


def block_work(script):
    """Per (major stage, block): (boomerang stages + 2 per partition, max num_ios)."""
    bd = script.blocks_data
    nb, nms = script.num_blocks, script.num_major_stages
    work = np.zeros((nms, nb), np.int64)
    mio = 0
    for ms in range(nms):
        for b in range(nb):
            off = int(script.blocks_start[ms * nb + b])
            while True:
                ns = int(bd[off])
                if ns == 0:
                    break
                mio = max(mio, int(bd[off + 2]))
                work[ms, b] += ns + 2
                R, last = int(bd[off + 6]), int(bd[off + 1])
                off += 256 + 512 * R + 5120 * (ns + 2)
                if last:
                    break
    return work, mio


def max_num_ios(script):
    return block_work(script)[1]


def block_lists(script):
    """Non-empty blocks of each major stage, heaviest first, and offsets."""
    work, _ = block_work(script)
    lst, start = [], [0]
    for ms in range(work.shape[0]):
        nz = np.nonzero(work[ms])[0]
        nz = nz[np.argsort(-work[ms][nz], kind="stable")]
        lst.extend(nz.tolist())
        start.append(len(lst))
    return np.asarray(lst if lst else [0], np.uint32), np.asarray(start, np.uint32)


def check_x_offsets(script, value_words):
    """Every X-capable partition's X offset (metadata word 9) must be
    value_words: the batched kernel takes a signal's X plane from the quad
    layout, not from the offset."""
    bd = np.asarray(script.blocks_data, dtype=np.uint32)
    starts = np.asarray(script.blocks_start, dtype=np.int64)
    for off in starts[:-1].tolist():
        while True:
            ns = int(bd[off])
            if ns == 0:
                break
            if bd[off + 8] and int(bd[off + 9]) != value_words:
                raise ValueError(f"X offset {int(bd[off + 9])} != {value_words} value words")
            if bd[off + 1]:
                break
            off += 256 + 512 * int(bd[off + 6]) + 5120 * (ns + 2)


class BatchedSim:
    """Script + buffers on the device for `lanes` lane words (32*lanes streams)."""

    def __init__(self, script, lanes, device="cuda", record=False, po_signals=None, grid=0,
                 wo_slots=None, lanes_per_item=0):
        self.script = script
        self.lanes = lanes
        self.device = torch.device(device)
        self.ds = sim.DeviceScript(script, self.device)
        # the kernel reads the script in its own prepared layout, with the
        # global-read sources resolved once
        L = lib()
        n_parts = getattr(script, "num_partitions", None)
        if n_parts is None:
            n_parts = len(script.stage_block_part)
        self.num_partitions = int(n_parts)
        self.prepared = torch.empty_like(self.ds.blocks_data)
        self.part_base_dev = torch.empty(self.ds.num_blocks * self.ds.num_major_stages,
                                         dtype=torch.int32, device=self.device)
        self.gr_sources = torch.empty(L.jq_batched_gr_words(self.num_partitions), dtype=torch.int32,
                                      device=self.device)
        rc = L.jq_batched_prepare(self.ds.blocks_start.data_ptr(), self.ds.blocks_data.data_ptr(),
                                  self.ds.blocks_data.numel(), self.ds.num_blocks,
                                  self.ds.num_major_stages, self.num_partitions,
                                  self.prepared.data_ptr(), self.part_base_dev.data_ptr(),
                                  self.gr_sources.data_ptr(),
                                  torch.cuda.current_stream(self.device).cuda_stream)
        if rc:
            raise RuntimeError("jq_batched_prepare: " + sim.lib().jq_strerror(rc).decode())
        self.eff = getattr(script, "effective_words", None) or \
            script.reg_io_state_size * (2 if script.xprop_enabled else 1)
        self.sig = self.eff * 32
        # X-capable scripts run in the quad layout (lane pairs) or the octet
        # layout (octet items): signals [sig/2, sig) are the X planes of
        # [0, sig/2), which every X partition's offset must say
        self.x_interleaved = 1 if script.xprop_enabled else 0
        if self.x_interleaved:
            check_x_offsets(script, self.eff // 2)
        if lanes_per_item == 8:
            need, cap = self.octet_need(), octet_capacity()
            if not script.xprop_enabled or lanes % 8 or need > cap:
                raise ValueError(f"octet items need an X-propagating script, lanes divisible by 8 "
                                 f"and every partition within {cap} slots (needs {need:#x})")
            self.x_interleaved = 2
        regions = getattr(script, "input_regions", None)
        if regions is None:
            self.in_sigs = input_words(script) * 32
            self.regions = None
        else:
            r = np.asarray(regions, np.uint32).reshape(-1, 3)
            self.in_sigs = int(r[:, 2].sum())
            self.regions = torch.from_numpy(r.reshape(-1).view(np.int32)).to(self.device)
        # writeout capacity: the largest num_ios, or more (256 selects the
        # single-buffered tree state, whose shared memory fits any script)
        self.wo_slots = max(1, max_num_ios(script)) if wo_slots is None else wo_slots
        bl, bls = block_lists(script)
        self.block_list = torch.from_numpy(bl.view(np.int32)).to(self.device)
        self.block_list_start = torch.from_numpy(bls.view(np.int32)).to(self.device)
        self.sram_words = max(1, script.sram_storage_size)
        n_streams = 32 * lanes
        self.state_a = torch.zeros(L.jq_batched_state_words(lanes, self.sig), dtype=torch.int32,
                                   device=self.device)
        self.state_b = torch.zeros_like(self.state_a)
        self.sram = torch.zeros(n_streams * self.sram_words, dtype=torch.int32, device=self.device)
        self.sram_x = torch.full_like(self.sram, -1)
        self.po = torch.from_numpy(np.asarray(po_signals if po_signals is not None else [0],
                                              dtype=np.int64).astype(np.int32)).to(self.device)
        self.n_po = 0 if po_signals is None else len(po_signals)
        self.record = record
        self.grid = grid
        # lane words per work item: 0 lets the library pick (lane pairs when
        # lanes is even and they fit), 1, 2 or 8 (octets) forces one
        self.lanes_per_item = lanes_per_item

    def octet_need(self):
        """The most 64-byte tree slots an octet item needs for any partition
        of the prepared script (0xffffffff: some partition cannot run as one)."""
        need = torch.zeros(1, dtype=torch.int32, device=self.device)
        st = torch.cuda.current_stream(self.device).cuda_stream
        rc = lib().jq_batched_slot_need(self.ds.blocks_start.data_ptr(), self.prepared.data_ptr(),
                                        self.ds.num_blocks, self.ds.num_major_stages,
                                        need.data_ptr(), st)
        if rc:
            raise RuntimeError("jq_batched_slot_need: " + sim.lib().jq_strerror(rc).decode())
        return int(need.cpu().numpy().view(np.uint32)[0])

    def _convert(self, fn, src, dst):
        st = torch.cuda.current_stream(self.device).cuda_stream
        rc = fn(src.data_ptr(), self.lanes, self.sig, self.x_interleaved, dst.data_ptr(), st)
        if rc:
            raise RuntimeError("batched state conversion: " + sim.lib().jq_strerror(rc).decode())

    def load_state(self, snap0):
        """snap0: (lanes, sig) u32 lane-major snapshot 0 (values + X template)."""
        t = torch.from_numpy(np.ascontiguousarray(snap0, np.uint32).reshape(-1).view(np.int32)).to(self.device)
        assert t.numel() == self.lanes * self.sig
        self._convert(lib().jq_batched_pack_state, t, self.state_a)
        self.state_b.copy_(self.state_a)

    def reset_sram(self, x=True):
        self.sram.zero_()
        self.sram_x.fill_(-1 if x else 0)

    def part_base(self):
        """Index of the first partition of each (major stage, block)."""
        sbp = self.script.stage_block_part
        nb = self.script.num_blocks
        base = np.zeros(self.script.num_major_stages * nb, np.uint32)
        seen = {}
        for i, (ms, b, _) in enumerate(sbp.tolist()):
            seen.setdefault(ms * nb + b, i)
        nxt = len(sbp)
        for k in range(base.size - 1, -1, -1):
            nxt = seen.get(k, nxt)
            base[k] = nxt
        return base

    def run(self, stim, cycles, wave=None, record_buf=None, stream=None, part_cycles=None,
            barrier_timeout_cycles=0, timing=None, first_cycle=0):
        """stim: device tensor [(cycles+1) * lanes * in_sigs] int32 or None.
        barrier_timeout_cycles: grid-barrier wait limit in SM clocks (0 = the
        library's default of about a second).  timing: a Timing (setup/hold
        checks per stream into its event buffer), or None."""
        L = lib()
        wave_ptr = wave.data_ptr() if wave is not None else None
        a = BatchArgs(self.ds.num_blocks, self.ds.num_major_stages, self.ds.blocks_start.data_ptr(),
                      self.prepared.data_ptr(), self.lanes, self.sram.data_ptr(),
                      self.sram_x.data_ptr(), self.sram_words, cycles, self.sig,
                      self.state_a.data_ptr(), self.state_b.data_ptr(),
                      stim.data_ptr() if stim is not None else None, self.in_sigs,
                      self.regions.data_ptr() if self.regions is not None else None,
                      0 if self.regions is None else self.regions.numel() // 3,
                      self.po.data_ptr(), self.n_po, wave_ptr,
                      record_buf.data_ptr() if record_buf is not None else None,
                      self.wo_slots, self.block_list.data_ptr(), self.block_list_start.data_ptr(),
                      part_cycles.data_ptr() if part_cycles is not None else None,
                      self.part_base_dev.data_ptr(), self.gr_sources.data_ptr(),
                      self.grid, barrier_timeout_cycles,
                      stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream,
                      self.lanes_per_item, self.x_interleaved)
        if timing is not None:
            a.timing_constraints = timing.constraints.data_ptr()
            a.arrival_first = timing.arrival_first.data_ptr()
            a.arrival_steady = timing.arrival_steady.data_ptr()
            a.events = timing.events.data_ptr()
            a.event_capacity = timing.capacity
            a.first_cycle = first_cycle
        rc = L.jq_simulate_batched(ctypes.byref(a))
        if rc:
            raise RuntimeError("jq_simulate_batched: " + sim.lib().jq_strerror(rc).decode())

    def status(self, stream=None):
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        return lib().jq_batched_status(s)

    def final_state(self, cycles):
        """Lane-major (lanes * sig) copy of the state after `cycles` cycles."""
        src = self.state_a if cycles % 2 == 0 else self.state_b
        out = torch.empty(self.lanes * self.sig, dtype=torch.int32, device=self.device)
        self._convert(lib().jq_batched_unpack_state, src, out)
        return out


def arrival_tables(script, device="cuda", stream=None):
    """The u16 arrival of every state word in the first cycle of a launch
    and in later cycles (int32 device tensors of reg_io_state_size words):
    the arrival sections of snapshots 1 and 2 of a two-cycle run of the
    plain interpreter on the same script.  Arrivals follow from the script's
    delays and each block's execution order, not from the stimulus, so an
    all-zero state serves."""
    rio = script.reg_io_state_size
    eff = rio * (2 if script.xprop_enabled else 1) + rio  # + arrival section
    ds = sim.DeviceScript(script, device)
    st = torch.zeros(3 * eff, dtype=torch.int32, device=device)
    n_sram = max(1, script.sram_storage_size)
    sram = torch.zeros(n_sram, dtype=torch.int32, device=device)
    sram_x = torch.zeros(n_sram, dtype=torch.int32, device=device)
    off = eff - rio
    sim.simulate(ds, st, 2, eff, sram, sram_x, arrival_state_offset=off, stream=stream)
    rc = sim.status(stream)
    if rc:
        raise RuntimeError("arrival tables: " + sim.lib().jq_strerror(rc).decode())
    snaps = st.view(3, eff)
    return snaps[1, off:].clone(), snaps[2, off:].clone()


class Timing:
    """Setup/hold checking for batched runs: the constraint buffer
    ([clock_ps, setup << 16 | hold per state word]), the script's arrival
    tables and an event buffer of `capacity` records (sim.new_event_buffer)."""

    def __init__(self, script, constraints, capacity, device="cuda"):
        self.constraints = sim.u32_to_dev(np.asarray(constraints, np.uint32), device)
        self.arrival_first, self.arrival_steady = arrival_tables(script, device)
        self.capacity = capacity
        self.events = sim.new_event_buffer(capacity, device)

    def reset_events(self):
        self.events[:2].zero_()

    def read(self):
        """(records (n, 8) u32, count, overflow) of the events so far."""
        return sim.read_events(self.events)


class CombinedScript:
    """Several designs' scripts relocated into one script and one state so a
    single persistent launch runs them all (work items of every design share
    the CTAs; designs with fewer major stages leave empty blocks).

    The combined state holds every design's value words, then every design's
    X words in the same order (the batched quad layout needs one X offset).
    Relocation only shifts absolute offsets: IO offset (metadata word 3), SRAM
    offset (word 5) and global-read word indices move by the design's value /
    SRAM base, and the X offset (word 9) becomes the total value words."""

    def __init__(self, scripts):
        self.parts = scripts
        self.xprop_enabled = True
        nms = max(s.num_major_stages for s in scripts)
        self.num_major_stages = nms
        self.num_blocks = sum(s.num_blocks for s in scripts)
        self.state_base, self.sram_base, self.block_base = [], [], []
        sb = srb = bb = 0
        for s in scripts:
            assert s.xprop_enabled, "designs are combined with X-propagation on"
            self.state_base.append(sb)
            self.sram_base.append(srb)
            self.block_base.append(bb)
            sb += s.reg_io_state_size
            srb += s.sram_storage_size
            bb += s.num_blocks
        self.value_words = sb
        self.effective_words = 2 * sb
        self.sram_storage_size = srb
        self.reg_io_state_size = sb
        data, starts, sbp = [], [], []
        pos = 0
        dummy = np.zeros(256, np.uint32)
        dummy[1] = 1
        pidx = 0
        for ms in range(nms):
            for d, s in enumerate(scripts):
                for b in range(s.num_blocks):
                    starts.append(pos)
                    if ms >= s.num_major_stages:
                        data.append(dummy)
                        pos += 256
                        continue
                    lo = int(s.blocks_start[ms * s.num_blocks + b])
                    hi = int(s.blocks_start[ms * s.num_blocks + b + 1])
                    blk = s.blocks_data[lo:hi].copy()
                    off = 0
                    while True:
                        ns = int(blk[off])
                        if ns == 0:
                            break
                        R = int(blk[off + 6])
                        blk[off + 3] += self.state_base[d]
                        blk[off + 5] += self.sram_base[d]
                        if blk[off + 8]:
                            blk[off + 9] = self.value_words
                        g = blk[off + 256: off + 256 + 512 * R].reshape(-1, 2)
                        nz = g[:, 1] != 0
                        hi_bit = g[:, 0] & np.uint32(0x80000000)
                        g[:, 0] = np.where(nz, hi_bit | ((g[:, 0] & np.uint32(0x7FFFFFFF)) +
                                                         np.uint32(self.state_base[d])), g[:, 0])
                        sbp.append((ms, self.block_base[d] + b, pidx))
                        pidx += 1
                        last = int(blk[off + 1])
                        off += 256 + 512 * R + 5120 * (ns + 2)
                        if last:
                            break
                    data.append(blk)
                    pos += blk.size
        starts.append(pos)
        data.append(np.zeros(8 * 256, np.uint32))
        self.blocks_data = np.concatenate(data).astype(np.uint32)
        self.blocks_start = np.asarray(starts, np.uint64)
        self.stage_block_part = np.asarray(sbp, np.uint32).reshape(-1, 3)
        # stimulus: each design's input signals, concatenated per lane
        regions, src = [], 0
        for d, s in enumerate(scripts):
            n = input_words(s) * 32
            regions.append((self.state_base[d] * 32, src, n))
            src += n
        self.input_regions = regions

    def script_words_per_cycle(self):
        return int(self.blocks_start[-1])

    def signal(self, d, sig):
        """Combined signal index of design d's signal `sig` (its own layout:
        values, then X at reg_io_state_size * 32)."""
        n = self.parts[d].reg_io_state_size * 32
        if sig < n:
            return self.state_base[d] * 32 + sig
        return (self.value_words + self.state_base[d]) * 32 + sig - n

    def combine_states(self, states):
        """Per-design lane-major states (..., 2 * rio_d * 32) -> the combined
        lane-major state (..., 2 * value_words * 32)."""
        vals = [st[..., :s.reg_io_state_size * 32] for st, s in zip(states, self.parts)]
        xs = [st[..., s.reg_io_state_size * 32:] for st, s in zip(states, self.parts)]
        return np.concatenate(vals + xs, axis=-1)

    def design_state(self, d, state):
        """Design d's lane-major state (values, then X) out of a combined one."""
        n = self.parts[d].reg_io_state_size * 32
        lo = self.state_base[d] * 32
        xlo = (self.value_words + self.state_base[d]) * 32
        return np.concatenate([state[..., lo:lo + n], state[..., xlo:xlo + n]], axis=-1)
