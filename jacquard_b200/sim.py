"""Host driver of the interpreter: the `sim_cuda` step of the reference
(src/bin/jacquard.rs:1089-1256) over this library's C ABI.

Device buffers are torch tensors (int32 storage for u32 words); every kernel
call goes through libjacquard_b200.so -- there is no other execution path.
"""
import ctypes

import numpy as np
import torch

from ._native import load

vp = ctypes.c_void_p


class SimArgs(ctypes.Structure):
    _fields_ = [("num_blocks", ctypes.c_size_t), ("num_major_stages", ctypes.c_size_t),
                ("blocks_start", vp), ("blocks_data", vp), ("sram_data", vp),
                ("sram_xmask", vp), ("num_cycles", ctypes.c_size_t),
                ("state_size", ctypes.c_size_t), ("states", vp), ("timing_constraints", vp),
                ("events", vp), ("event_capacity", ctypes.c_uint32),
                ("arrival_state_offset", ctypes.c_int32), ("first_cycle", ctypes.c_uint32),
                ("barrier_timeout_cycles", ctypes.c_uint64), ("stream", vp),
                ("stage_depth", vp), ("stage_depth_base", vp)]


EVENT_WORDS = 8
EVENT_HEADER_WORDS = 4


def lib():
    L = load("libjacquard_b200.so")
    if not getattr(L, "_jq_typed", False):
        L.jq_simulate.restype = ctypes.c_int
        L.jq_simulate.argtypes = [ctypes.POINTER(SimArgs)]
        L.jq_sim_status.restype = ctypes.c_int
        L.jq_sim_status.argtypes = [vp]
        L.jq_max_blocks.restype = ctypes.c_int
        L.jq_max_blocks.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
        L.jq_plain_prepare.restype = ctypes.c_int
        L.jq_plain_prepare.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_size_t, vp, vp,
                                       ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), vp]
        L.jq_strerror.restype = ctypes.c_char_p
        L.jq_strerror.argtypes = [ctypes.c_int]
        sz, u32p, i32 = ctypes.c_size_t, vp, ctypes.c_int32
        L.simulate_v1_noninteractive_simple_scan_cuda.restype = None
        L.simulate_v1_noninteractive_simple_scan_cuda.argtypes = [sz, sz, vp, vp, vp, vp, sz, sz, vp, i32]
        L.simulate_v1_noninteractive_timed_cuda.restype = None
        L.simulate_v1_noninteractive_timed_cuda.argtypes = [sz, sz, vp, vp, vp, vp, sz, sz, vp, vp, vp, i32]
        L._jq_typed = True
    return L


def u32_to_dev(a, device="cuda"):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32)).to(device)


def dev_to_u32(t):
    return t.cpu().numpy().view(np.uint32)


class DeviceScript:
    """Script arrays resident on the device."""

    def __init__(self, script, device="cuda"):
        self.script = script
        self.num_blocks = script.num_blocks
        self.num_major_stages = script.num_major_stages
        self.blocks_start = torch.from_numpy(
            np.ascontiguousarray(script.blocks_start, dtype=np.uint64).view(np.int64)).to(device)
        self.blocks_data = u32_to_dev(script.blocks_data, device)
        self._depth = None

    def depth(self, stream=None):
        """(stage depth codes, per-entry base) on the device
        (jq_plain_prepare), computed on first use."""
        if self._depth is None:
            L = lib()
            st = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
            entries = self.num_blocks * self.num_major_stages
            base = torch.empty(entries, dtype=torch.int32, device=self.blocks_data.device)
            n = ctypes.c_size_t()
            rc = L.jq_plain_prepare(self.blocks_start.data_ptr(), self.blocks_data.data_ptr(),
                                    self.num_blocks, self.num_major_stages, base.data_ptr(),
                                    None, 0, ctypes.byref(n), st)
            if rc:
                raise RuntimeError("jq_plain_prepare: " + lib().jq_strerror(rc).decode())
            depth = torch.empty(max(1, n.value), dtype=torch.uint8, device=self.blocks_data.device)
            rc = L.jq_plain_prepare(self.blocks_start.data_ptr(), self.blocks_data.data_ptr(),
                                    self.num_blocks, self.num_major_stages, base.data_ptr(),
                                    depth.data_ptr(), depth.numel(), None, st)
            if rc:
                raise RuntimeError("jq_plain_prepare: " + lib().jq_strerror(rc).decode())
            self._depth = (depth, base)
        return self._depth


def max_blocks(device=0):
    n = ctypes.c_size_t()
    rc = lib().jq_max_blocks(device, ctypes.byref(n))
    if rc:
        raise RuntimeError(lib().jq_strerror(rc).decode())
    return n.value


def simulate(ds, states, num_cycles, state_size, sram, sram_x=None, constraints=None,
             events=None, event_capacity=0, arrival_state_offset=0, first_cycle=0,
             stream=None, barrier_timeout_cycles=0, skip_dead_levels=True):
    """Launch the plain interpreter (asynchronous).  All tensors on device.
    skip_dead_levels: pass the script's stage-depth tables, so tree levels
    whose outputs nothing reads are skipped (False runs every level)."""
    a = SimArgs(ds.num_blocks, ds.num_major_stages, ds.blocks_start.data_ptr(),
                ds.blocks_data.data_ptr(), sram.data_ptr(),
                sram_x.data_ptr() if sram_x is not None else None, num_cycles, state_size,
                states.data_ptr(), constraints.data_ptr() if constraints is not None else None,
                events.data_ptr() if events is not None else None, event_capacity,
                arrival_state_offset, first_cycle, barrier_timeout_cycles,
                stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    if skip_dead_levels:
        depth, base = ds.depth(stream)
        a.stage_depth = depth.data_ptr()
        a.stage_depth_base = base.data_ptr()
    rc = lib().jq_simulate(ctypes.byref(a))
    if rc:
        raise RuntimeError("jq_simulate: " + lib().jq_strerror(rc).decode())


def status(stream=None):
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    return lib().jq_sim_status(s)


def new_event_buffer(capacity, device="cuda"):
    buf = torch.zeros(EVENT_HEADER_WORDS + EVENT_WORDS * capacity, dtype=torch.int32, device=device)
    buf[2] = capacity
    return buf


def read_events(buf):
    h = dev_to_u32(buf[:EVENT_HEADER_WORDS])
    count, overflow, cap = int(h[0]), int(h[1]), int(h[2])
    n = min(count, cap)
    ev = dev_to_u32(buf[EVENT_HEADER_WORDS:EVENT_HEADER_WORDS + EVENT_WORDS * n]).reshape(n, EVENT_WORDS)
    return ev, count, overflow
