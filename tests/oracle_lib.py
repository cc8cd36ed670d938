"""ctypes binding of the CPU oracle (oracle/libjq_oracle.so).

Test infrastructure: used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline only, never by the product path.
"""
import ctypes
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(REPO, "oracle", "libjq_oracle.so")

_lib = None

vp = ctypes.c_void_p


class Event(ctypes.Structure):
    _fields_ = [("event_type", ctypes.c_uint32), ("message_id", ctypes.c_uint32),
                ("cycle", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("data", ctypes.c_uint32 * 4)]


EVENT_DTYPE = np.dtype([("event_type", "<u4"), ("message_id", "<u4"), ("cycle", "<u4"),
                        ("reserved", "<u4"), ("data", "<u4", (4,))])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(ORACLE_SO)
        L.jqo_simulate.restype = ctypes.c_int
        L.jqo_simulate.argtypes = [ctypes.c_size_t, ctypes.c_size_t, vp, vp, vp, vp,
                                   ctypes.c_size_t, ctypes.c_size_t, vp, vp, vp,
                                   ctypes.c_size_t, vp, ctypes.c_int32, ctypes.c_uint32,
                                   ctypes.c_int]
        L.jqo_simulate_block.restype = ctypes.c_long
        L.jqo_simulate_block.argtypes = [vp, ctypes.c_size_t, vp, vp, vp, vp, ctypes.c_uint32]
        u = ctypes.c_uint32
        L.jqo_xprop_and.argtypes = [u, u, u, u, u, u, u, ctypes.POINTER(u), ctypes.POINTER(u)]
        L.jqo_dff_commit.argtypes = [u, u, u, u, u, u, ctypes.POINTER(u), ctypes.POINTER(u)]
        L.jqo_setup_violation.argtypes = [ctypes.c_uint16, ctypes.c_uint16, u,
                                          ctypes.POINTER(ctypes.c_int32)]
        L.jqo_hold_violation.argtypes = [ctypes.c_uint16, ctypes.c_uint16,
                                         ctypes.POINTER(ctypes.c_int32)]
        L.jqo_aig_simulate.restype = ctypes.c_int
        L.jqo_aig_simulate.argtypes = [ctypes.c_uint32, vp, vp, vp, ctypes.c_size_t, vp, vp, vp,
                                       ctypes.c_size_t, vp, ctypes.c_size_t, vp, ctypes.c_size_t,
                                       vp, vp, ctypes.c_size_t, vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def simulate(script, states, num_cycles, state_size, sram=None, sram_x=None,
             constraints=None, arrival_state_offset=0, event_cap=0, flags=0, threads=1):
    """Run the oracle over `states` (modified in place).  Returns
    (events structured array, total event count)."""
    L = lib()
    bs = np.ascontiguousarray(script.blocks_start, dtype=np.uint64)
    bd = np.ascontiguousarray(script.blocks_data, dtype=np.uint32)
    assert states.dtype == np.uint32 and states.flags.c_contiguous
    assert states.size >= (num_cycles + 1) * state_size
    if sram is None:
        sram = np.zeros(max(1, script.sram_storage_size), dtype=np.uint32)
    ev = np.zeros(max(1, event_cap), dtype=EVENT_DTYPE)
    cnt = ctypes.c_uint64(0)
    cons = None if constraints is None else np.ascontiguousarray(constraints, dtype=np.uint32)
    r = L.jqo_simulate(script.num_blocks, script.num_major_stages, _p(bs), _p(bd), _p(sram),
                       _p(sram_x), num_cycles, state_size, _p(states), _p(cons),
                       _p(ev) if event_cap else None, event_cap, ctypes.addressof(cnt),
                       arrival_state_offset, flags, threads)
    if r != 0:
        raise RuntimeError(f"oracle rejected the script (code {r})")
    n = min(int(cnt.value), event_cap)
    return ev[:n], int(cnt.value)


def aig_simulate(design, input_layout, in_vals, dff_init, num_cycles):
    """Netlist-level two-state simulation; returns (dff_state, po_vals)."""
    L = lib()
    kind = design.kind
    fa = design.fanin_a
    fb = design.fanin_b
    d, en, q = design.dff_d, design.dff_en, design.dff_q
    po = design.primary_outputs
    sr = np.ascontiguousarray(design.sram_records.reshape(-1)) if design.num_srams else np.zeros(1, np.uint32)
    n_dff, n_po, n_in = d.size, po.size, input_layout.size
    dff = np.zeros((num_cycles + 1, n_dff), dtype=np.uint8)
    dff[0] = dff_init
    pov = np.zeros((num_cycles + 1, n_po), dtype=np.uint8)
    sram_words = np.zeros(max(1, design.num_srams) * 8192, dtype=np.uint32)
    sram_rd = np.zeros((num_cycles + 1, max(1, design.num_srams), 32), dtype=np.uint8)
    inv = np.ascontiguousarray(in_vals, dtype=np.uint8)
    lay = np.ascontiguousarray(input_layout, dtype=np.uint32)
    L.jqo_aig_simulate(int(design.num_pins), _p(kind), _p(fa), _p(fb), n_dff, _p(d), _p(en),
                       _p(q), int(design.num_srams), _p(sr), n_in, _p(lay), num_cycles, _p(inv),
                       _p(dff), n_po, _p(po), _p(pov), _p(sram_words), _p(sram_rd))
    return dff, pov


def repcut(inp):
    """jqo_repcut on the arrays of jacquard_b200.repcut.slice_inputs:
    (class of each pin or -1, cluster first pins, cluster sizes, endpoint
    weights)."""
    L = lib()
    if not getattr(L, "_jq_repcut_typed", False):
        vp = ctypes.c_void_p
        L.jqo_repcut.restype = ctypes.c_int
        L.jqo_repcut.argtypes = [ctypes.c_uint32, vp, vp, vp, vp, vp, vp, ctypes.c_uint32, vp, vp,
                                 vp, vp, vp, vp]
        L._jq_repcut_typed = True
    N, E = inp["num_pins"], inp["num_endpoints"]
    cls = np.zeros(N + 1, np.int32)
    first = np.zeros(N + 1, np.uint32)
    count = np.zeros(N + 1, np.uint32)
    ew = np.zeros(max(1, E), np.uint64)
    arrs = [np.ascontiguousarray(inp[k]) for k in ("kind", "fa", "fb", "fanout_start", "fanouts", "staged")]
    n = L.jqo_repcut(N, *(a.ctypes.data for a in arrs), E, inp["ep_start"].ctypes.data,
                     inp["ep_pins"].ctypes.data, cls.ctypes.data, first.ctypes.data, count.ctypes.data,
                     ew.ctypes.data)
    if n < 0:
        raise MemoryError("repcut oracle")
    return cls.astype(np.int64), first[:n].astype(np.int64), count[:n].astype(np.int64), ew[:E]
