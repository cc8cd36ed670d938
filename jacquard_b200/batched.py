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
                ("po_signals", vp), ("n_po", ctypes.c_uint32), ("wave", vp), ("record", vp),
                ("wo_slots", ctypes.c_uint32), ("grid", ctypes.c_size_t),
                ("barrier_timeout_cycles", ctypes.c_uint64), ("stream", vp)]


def lib():
    L = load("libjacquard_b200.so")
    if not getattr(L, "_jq_batched_typed", False):
        L.jq_simulate_batched.restype = ctypes.c_int
        L.jq_simulate_batched.argtypes = [ctypes.POINTER(BatchArgs)]
        L.jq_batched_status.restype = ctypes.c_int
        L.jq_batched_status.argtypes = [vp]
        L.jq_batched_max_blocks.restype = ctypes.c_int
        L.jq_batched_max_blocks.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(ctypes.c_size_t)]
        L._jq_batched_typed = True
    return L


def to_batched(per_stream):
    """(streams, ..., words) u32 per-stream layout -> (..., words*32, lanes)
    signal-major lane words (streams must be a multiple of 32)."""
    a = np.asarray(per_stream, dtype=np.uint32)
    S = a.shape[0]
    assert S % 32 == 0
    bits = ((a[..., None] >> np.arange(32, dtype=np.uint32)) & 1).astype(np.uint8)
    bits = bits.reshape(a.shape[:-1] + (a.shape[-1] * 32,))       # (S, ..., sig)
    bits = np.moveaxis(bits, 0, -1)                                # (..., sig, S)
    packed = np.packbits(bits, axis=-1, bitorder="little")        # (..., sig, S/8)
    return np.ascontiguousarray(packed).view(np.uint32)           # (..., sig, lanes)


def from_batched(batched, words):
    """Inverse of to_batched: (..., sig, lanes) -> (streams, ..., words)."""
    b = np.ascontiguousarray(batched, dtype=np.uint32)
    lanes = b.shape[-1]
    bits = np.unpackbits(b.view(np.uint8), axis=-1, bitorder="little")  # (..., sig, S)
    bits = np.moveaxis(bits, -1, 0).astype(np.uint32)              # (S, ..., sig)
    bits = bits.reshape(bits.shape[:-1] + (words, 32))
    return (bits << np.arange(32, dtype=np.uint32)).sum(axis=-1, dtype=np.uint64).astype(np.uint32)


def input_words(script):
    """Words of the input region (src/flatten.rs:1159-1166)."""
    n = len(script.input_layout)
    w = (n + 31) // 32
    if n == w * 32:
        w += 1
    return w


def max_num_ios(script):
    bd, m = script.blocks_data, 0
    for b in range(script.num_blocks * script.num_major_stages):
        off = int(script.blocks_start[b])
        while True:
            ns = int(bd[off])
            if ns == 0:
                break
            m = max(m, int(bd[off + 2]))
            R, last = int(bd[off + 6]), int(bd[off + 1])
            off += 256 + 512 * R + 5120 * (ns + 2)
            if last:
                break
    return m


class BatchedSim:
    """Script + buffers on the device for `lanes` lane words (32*lanes streams)."""

    def __init__(self, script, lanes, device="cuda", record=False, po_signals=None, grid=0):
        self.script = script
        self.lanes = lanes
        self.device = torch.device(device)
        self.ds = sim.DeviceScript(script, self.device)
        self.eff = script.reg_io_state_size * (2 if script.xprop_enabled else 1)
        self.sig = self.eff * 32
        self.in_sigs = input_words(script) * 32
        self.wo_slots = max(1, max_num_ios(script))
        self.sram_words = max(1, script.sram_storage_size)
        n_streams = 32 * lanes
        self.state_a = torch.zeros(self.sig * lanes, dtype=torch.int32, device=self.device)
        self.state_b = torch.zeros_like(self.state_a)
        self.sram = torch.zeros(n_streams * self.sram_words, dtype=torch.int32, device=self.device)
        self.sram_x = torch.full_like(self.sram, -1)
        self.po = torch.from_numpy(np.asarray(po_signals if po_signals is not None else [0],
                                              dtype=np.int64).astype(np.int32)).to(self.device)
        self.n_po = 0 if po_signals is None else len(po_signals)
        self.record = record
        self.grid = grid

    def load_state(self, snap0):
        """snap0: (sig, lanes) u32 batched snapshot 0 (values + X template)."""
        t = torch.from_numpy(np.ascontiguousarray(snap0, np.uint32).reshape(-1).view(np.int32)).to(self.device)
        self.state_a.copy_(t)
        self.state_b.copy_(t)

    def reset_sram(self, x=True):
        self.sram.zero_()
        self.sram_x.fill_(-1 if x else 0)

    def run(self, stim, cycles, wave=None, record_buf=None, stream=None):
        """stim: device tensor [(cycles+1) * in_sigs * lanes] int32 or None."""
        L = lib()
        wave_ptr = wave.data_ptr() if wave is not None else None
        a = BatchArgs(self.ds.num_blocks, self.ds.num_major_stages, self.ds.blocks_start.data_ptr(),
                      self.ds.blocks_data.data_ptr(), self.lanes, self.sram.data_ptr(),
                      self.sram_x.data_ptr(), self.sram_words, cycles, self.sig,
                      self.state_a.data_ptr(), self.state_b.data_ptr(),
                      stim.data_ptr() if stim is not None else None, self.in_sigs,
                      self.po.data_ptr(), self.n_po, wave_ptr,
                      record_buf.data_ptr() if record_buf is not None else None,
                      self.wo_slots, self.grid, 0,
                      stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
        rc = L.jq_simulate_batched(ctypes.byref(a))
        if rc:
            raise RuntimeError("jq_simulate_batched: " + sim.lib().jq_strerror(rc).decode())

    def status(self, stream=None):
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        return lib().jq_batched_status(s)

    def final_state(self, cycles):
        return self.state_a if cycles % 2 == 0 else self.state_b
