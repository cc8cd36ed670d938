"""The reference's own known-answer tests, run against the CPU oracle and the
host helpers that restate reference code (numbers copied from the reference
test files cited per test)."""
import ctypes

import numpy as np
import pytest

import oracle_lib
from minimal_script import build_minimal_xprop_script
from jacquard_b200 import state
from jacquard_b200._native import load


def xand(a_v, a_x, b_v, b_x, xora, xorb, orb):
    r, rx = ctypes.c_uint32(), ctypes.c_uint32()
    oracle_lib.lib().jqo_xprop_and(a_v, a_x, b_v, b_x, xora, xorb, orb, ctypes.byref(r), ctypes.byref(rx))
    return r.value, rx.value


# ---- src/sim/cpu_reference.rs:816-903
def test_xprop_and_absorbs_zero():
    assert xand(0, 0, 0, 0xFFFFFFFF, 0, 0, 0) == (0, 0)


def test_xprop_and_propagates_x():
    assert xand(0xFFFFFFFF, 0, 0, 0xFFFFFFFF, 0, 0, 0) == (0, 0xFFFFFFFF)


def test_xprop_and_x_and_x():
    assert xand(0, 0xFFFFFFFF, 0, 0xFFFFFFFF, 0, 0, 0)[1] == 0xFFFFFFFF


def test_xprop_and_known_values():
    assert xand(0xFFFFFFFF, 0, 0xFFFFFFFF, 0, 0, 0, 0) == (0xFFFFFFFF, 0)
    assert xand(0xFFFFFFFF, 0, 0, 0, 0, 0, 0) == (0, 0)


def test_xprop_passthrough_orb():
    assert xand(0, 0xFFFFFFFF, 0, 0xFFFFFFFF, 0, 0, 0xFFFFFFFF)[1] == 0xFFFFFFFF
    assert xand(0xAAAAAAAA, 0, 0, 0xFFFFFFFF, 0, 0, 0xFFFFFFFF) == (0xAAAAAAAA, 0)


def test_xprop_inversion_xora():
    assert xand(0, 0, 0, 0xFFFF, 0xFFFF, 0, 0)[1] & 0xFFFF == 0xFFFF


def test_xprop_mixed_bits():
    v, x = xand(0b1010, 0b0100, 0b1000, 0b0011, 0, 0, 0)
    assert x & 1 == 0 and x & 2 == 2 and x & 4 == 0
    assert v & 8 == 8 and x & 8 == 0


# ---- src/sim/cpu_reference.rs:906-942
def commit(old_v, old_x, new_v, new_x, clken, clken_x):
    a, b = ctypes.c_uint32(), ctypes.c_uint32()
    oracle_lib.lib().jqo_dff_commit(old_v, old_x, new_v, new_x, clken, clken_x, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def test_xprop_dff_writeout_clken():
    old_v, old_x, new_v, new_x = 0xAAAAAAAA, 0, 0x55555555, 0xFF00FF00
    assert commit(old_v, old_x, new_v, new_x, 0xFFFFFFFF, 0) == (new_v, new_x)
    assert commit(old_v, old_x, new_v, new_x, 0, 0) == (old_v, old_x)
    assert commit(old_v, old_x, new_v, new_x, 0, 0xFFFFFFFF)[1] == 0xFFFFFFFF


# ---- src/sim/cpu_reference.rs:1093-1206 (minimal one-partition script)
def run_block(script, inp, sram=None, sram_x=None, flags=0):
    out = np.zeros_like(inp)
    r = oracle_lib.lib().jqo_simulate_block(script.ctypes.data, script.size, inp.ctypes.data,
                                            out.ctypes.data,
                                            None if sram is None else sram.ctypes.data,
                                            None if sram_x is None else sram_x.ctypes.data, flags)
    assert r == script.size
    return out


def test_xprop_kernel_known_value_passthrough():
    n = 4
    sc = build_minimal_xprop_script(True, n)
    inp = np.zeros(2 * n, np.uint32)
    inp[0] = 1
    out = run_block(sc, inp)
    assert out[n + 0] & 1 == 0


def test_xprop_kernel_x_input_propagates():
    n = 4
    sc = build_minimal_xprop_script(True, n)
    inp = np.zeros(2 * n, np.uint32)
    inp[n + 0] = 1
    out = run_block(sc, inp)
    assert out[n + 0] != 0


def test_xprop_kernel_non_xcapable_delegates():
    n = 4
    sc = build_minimal_xprop_script(False, n)
    inp = np.zeros(2 * n, np.uint32)
    inp[0] = 0xAB
    a = run_block(sc, inp)
    b = run_block(sc, inp, flags=1)  # the CPU reference's delegate path
    assert np.array_equal(a[:n], b[:n])
    assert not a[n:].any()


# ---- src/flatten.rs:3076-3245 (violation predicates)
def setup(arr, su, clk):
    s = ctypes.c_int32()
    return s.value if oracle_lib.lib().jqo_setup_violation(arr, su, clk, ctypes.byref(s)) else None


def hold(arr, ho):
    s = ctypes.c_int32()
    return s.value if oracle_lib.lib().jqo_hold_violation(arr, ho, ctypes.byref(s)) else None


def test_setup_violation_detection():
    assert setup(900, 200, 1000) == -100
    assert setup(800, 200, 1000) is None


def test_setup_violation_with_realistic_inv_chain():
    assert setup(1323, 85, 1200) == -208
    assert setup(1323, 85, 1500) is None
    assert setup(1323, 85, 1400) == -8


def test_hold_violation_detection():
    assert hold(10, 50) == -40
    assert hold(50, 50) is None
    assert hold(0, 50) == -50


def test_no_violation_with_zero_constraint():
    assert hold(0, 0) is None and hold(500, 0) is None


def test_setup_skips_zero_arrival():
    assert setup(0, 200, 100) is None
    assert setup(1, 200, 100) is not None
    assert setup(0, 65535, 1) is None


def test_setup_u16_max_arrival():
    assert setup(65000, 1000, 60000) == -6000
    assert setup(65000, 1000, 70000) is None
    assert setup(65535, 65535, 131069) == -1
    assert setup(65535, 65535, 131070) is None


# ---- src/flatten.rs:2969-3365 (constraint buffer)
def cbuf(words, clock, dffs):
    from jacquard_b200.frontend import _lib
    L = _lib()
    n = len(dffs)
    su = np.array([d[0] for d in dffs], np.uint16)
    ho = np.array([d[1] for d in dffs], np.uint16)
    ca = np.array([d[2] for d in dffs], np.int16)
    pos = np.array([d[3] for d in dffs], np.uint32)
    out = np.zeros(max(1, words), np.uint32)
    clk = ctypes.c_uint32()
    vp = ctypes.c_void_p
    L.jqf_constraint_buffer(ctypes.c_uint32(words), ctypes.c_uint64(clock), ctypes.c_size_t(n),
                            vp(su.ctypes.data), vp(ho.ctypes.data), vp(ca.ctypes.data),
                            vp(pos.ctypes.data), ctypes.byref(clk), vp(out.ctypes.data))
    return clk.value, out[:words]


def test_empty_constraints():
    c, b = cbuf(4, 10000, [])
    assert c == 10000 and b.tolist() == [0, 0, 0, 0]


def test_single_dff_constraint():
    c, b = cbuf(4, 25000, [(200, 50, 0, 35)])
    assert c == 25000 and b.tolist() == [0, (200 << 16) | 50, 0, 0]


def test_multiple_dffs_same_word_takes_min():
    _, b = cbuf(2, 10000, [(300, 100, 0, 5), (150, 200, 0, 10)])
    assert b[0] == (150 << 16) | 100


def test_skip_invalid_and_out_of_range():
    assert not cbuf(2, 10000, [(200, 50, 0, 0xFFFFFFFF)])[1].any()
    assert not cbuf(2, 10000, [(200, 50, 0, 100)])[1].any()


def test_clock_period_saturation():
    assert cbuf(1, 2**64 - 1, [])[0] == 0xFFFFFFFF


def test_constraint_buffer_with_tight_clock():
    c, b = cbuf(8, 1000, [(200, 50, 0, 160)])
    assert b[5] == (200 << 16) | 50 and np.count_nonzero(b) == 1
    assert setup(850, b[5] >> 16, c) == -50


def test_clock_arrival_fold():
    _, b = cbuf(2, 10000, [(200, 50, 80, 0)])
    assert (b[0] >> 16, b[0] & 0xFFFF) == (120, 130)
    _, b = cbuf(1, 10000, [(100, 65535 - 10, 500, 0)])
    assert (b[0] >> 16, b[0] & 0xFFFF) == (0, 65535)
    _, b = cbuf(1, 10000, [(1234, 567, 0, 0)])
    assert b[0] == (1234 << 16) | 567


# ---- src/flatten.rs:2868-2929 (delay injection)
def inject(delays, patches, size):
    from jacquard_b200.frontend import _lib
    L = _lib()
    bd = np.zeros(size, np.uint32)
    offs = np.array([p[0] for p in patches], np.uint64)
    starts = np.zeros(len(patches) + 1, np.uint32)
    pins = []
    for i, p in enumerate(patches):
        pins += p[1]
        starts[i + 1] = len(pins)
    pins = np.array(pins or [0], np.uint32)
    r = np.array([d[0] for d in delays], np.uint16)
    f = np.array([d[1] for d in delays], np.uint16)
    vp = ctypes.c_void_p
    L.jqf_inject_delays(vp(bd.ctypes.data), ctypes.c_size_t(size), ctypes.c_size_t(len(patches)),
                        vp(offs.ctypes.data), vp(starts.ctypes.data), vp(pins.ctypes.data),
                        vp(r.ctypes.data), vp(f.ctypes.data), ctypes.c_size_t(len(delays)))
    return bd


def test_delay_injection_kats():
    assert inject([(0, 0), (100, 100)], [(0, [1])], 1)[0] == 100
    assert inject([(0, 0), (350, 350), (0, 0)], [(0, [1, 2])], 1)[0] == 350
    assert inject([(0, 0), (0, 0)], [(0, [1])], 1)[0] == 0
    bd = inject([(0, 0), (5, 5), (15, 15)], [(0, [1]), (1, [2])], 2)
    assert bd.tolist() == [5, 15]


# ---- src/flatten.rs:3403-3512 (state sizes) and src/sim/vcd_io.rs:1075-1334
class Layout:
    def __init__(self, rio, xprop, inputs=(), arrivals=False):
        self.reg_io_state_size = rio
        self.xprop_enabled = xprop
        self.xprop_state_offset = rio if xprop else 0
        self.input_map = {100 + 2 * i: p for i, p in enumerate(inputs)}
        self.timing_arrivals_enabled = False
        self.arrival_state_offset = 0
        if arrivals:
            self.timing_arrivals_enabled = True
            self.arrival_state_offset = rio * (1 + int(xprop))

    def effective_state_size(self):
        return state.effective_state_size(self)


def test_effective_state_sizes():
    assert Layout(42, False).effective_state_size() == 42
    assert Layout(42, True).effective_state_size() == 84
    assert Layout(0, True).effective_state_size() == 0
    assert Layout(42, False, arrivals=True).effective_state_size() == 84
    lay = Layout(42, True, arrivals=True)
    assert lay.effective_state_size() == 126 and lay.arrival_state_offset == 84


def test_expand_split_roundtrip():
    lay = Layout(2, True, inputs=[0])
    vals = np.array([1, 0, 1, 1, 0, 1], np.uint32)
    ex = state.expand_states_for_xprop(vals, lay)
    assert ex.size == 12
    v, x = state.split_xprop_states(ex, 2)
    assert v.reshape(-1).tolist() == vals.tolist()
    assert x[:, 0].tolist() == [0xFFFFFFFE] * 3 and x[:, 1].tolist() == [0xFFFFFFFF] * 3


def test_split_preserves_cycle_structure():
    rio, n = 3, 4
    buf = []
    for snap in range(n):
        buf += [snap * 100 + w for w in range(rio)] + [snap * 100 + w + 1000 for w in range(rio)]
    v, x = state.split_xprop_states(np.array(buf, np.uint32), rio)
    for snap in range(n):
        assert v[snap].tolist() == [snap * 100 + w for w in range(rio)]
        assert x[snap].tolist() == [snap * 100 + w + 1000 for w in range(rio)]


def test_expand_xmask_template():
    lay = Layout(4, True, inputs=[0, 5, 64])
    ex = state.expand_states_for_xprop(np.zeros(4, np.uint32), lay).reshape(-1)
    xm = ex[4:]
    assert xm[0] == 0xFFFFFFFF & ~1 & ~(1 << 5)
    assert xm[1] == 0xFFFFFFFF and xm[2] == 0xFFFFFFFE and xm[3] == 0xFFFFFFFF


def test_expand_split_arrivals():
    lay = Layout(3, False, arrivals=True)
    ex = state.expand_states_for_arrivals(np.array([10, 20, 30, 40, 50, 60], np.uint32), lay)
    assert ex.reshape(-1).tolist() == [10, 20, 30, 0, 0, 0, 40, 50, 60, 0, 0, 0]
    lay = Layout(2, True, arrivals=True)
    ex = state.expand_states_for_arrivals(np.array([1, 2, 0xFF, 0xFF, 3, 4, 0xAA, 0xBB], np.uint32), lay)
    assert ex.reshape(-1).tolist() == [1, 2, 0xFF, 0xFF, 0, 0, 3, 4, 0xAA, 0xBB, 0, 0]
    lay = Layout(2, False, arrivals=True)
    a = state.split_arrival_states(np.array([10, 20, 350, 0, 30, 40, 500, 100], np.uint32), lay)
    assert a.reshape(-1).tolist() == [350, 0, 500, 100]
    lay = Layout(2, True, arrivals=True)
    a = state.split_arrival_states(np.array([10, 20, 0xFF, 0xFF, 350, 885], np.uint32), lay)
    assert a.reshape(-1).tolist() == [350, 885]
