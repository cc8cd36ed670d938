"""State-snapshot layout helpers.

A snapshot is `effective_state_size` u32 words: [values | X-mask | arrivals]
(src/flatten.rs:1581-1603).  The helpers below restate the reference's
host-side buffer preparation (src/sim/vcd_io.rs:465-550) and generate the
seeded synthetic stimulus that stands in for input VCDs (one snapshot per
active clock edge, clock posedge flag set in every snapshot).
"""
import numpy as np


def effective_state_size(script):
    """src/flatten.rs:682-691: [values | X-mask if X-prop | arrivals if on]."""
    n = script.reg_io_state_size
    if script.xprop_enabled:
        n += script.reg_io_state_size
    if script.timing_arrivals_enabled:
        n += script.reg_io_state_size
    return n


def input_positions(script):
    """State bit positions of the input_layout pins (inputs + clock flags)."""
    return np.array([script.input_map[int(p)] for p in script.input_layout], dtype=np.int64)


def pack_inputs(script, in_vals):
    """(rows, n_in) 0/1 -> (rows, reg_io_state_size) u32 with only input bits set."""
    in_vals = np.asarray(in_vals, dtype=np.uint32)
    rows = in_vals.shape[0]
    out = np.zeros((rows, script.reg_io_state_size), dtype=np.uint32)
    pos = input_positions(script)
    for i, p in enumerate(pos):
        out[:, p >> 5] |= in_vals[:, i] << np.uint32(p & 31)
    return out


def stimulus_inputs(script, design, cycles, seed, p_toggle=0.5, reset_cycles=0):
    """(cycles+1, n_in) input values: each primary input toggles with
    probability p_toggle per cycle, the clock posedge flag is 1 on every
    snapshot, and the reset input (if any) is held at 1 for the first
    reset_cycles snapshots and 0 afterwards."""
    rng = np.random.default_rng(seed)
    lay = np.asarray(script.input_layout)
    n = lay.size
    vals = np.zeros((cycles + 1, n), dtype=np.uint8)
    cur = rng.integers(0, 2, size=n, dtype=np.uint8)
    for c in range(cycles + 1):
        if c:
            cur ^= (rng.random(n) < p_toggle).astype(np.uint8)
        vals[c] = cur
    vals[:, lay == design.clock_flag_pin] = 1
    if design.reset_pin:
        col = lay == design.reset_pin
        vals[:, col] = 0
        vals[:reset_cycles, col] = 1
    return vals


def random_stimulus_states(script, design, cycles, seed, p_toggle=0.5, reset_cycles=0):
    """Value-only snapshots (cycles+1, reg_io_state_size): inputs filled,
    DFF / output words 0 (the reference's pre-fill, src/sim/vcd_io.rs:347-455)."""
    return pack_inputs(script, stimulus_inputs(script, design, cycles, seed, p_toggle, reset_cycles))


def xmask_template(script):
    """X-mask words of a snapshot: all X except input_map positions
    (src/sim/vcd_io.rs:465-484)."""
    rio = script.reg_io_state_size
    t = np.full(rio, 0xFFFFFFFF, dtype=np.uint32)
    for pos in script.input_map.values():
        t[pos >> 5] &= np.uint32(~(1 << (pos & 31)) & 0xFFFFFFFF)
    return t


def xmask_all_state_x(script):
    """X-mask words of an initial snapshot with every DFF and SRAM-read bit X:
    only the input_layout pins (primary inputs, clock flags) are known.  The
    reference CLI clears X on DFF-Q positions (the template above); a run that
    starts from an unknown register state sets this mask in snapshot 0."""
    rio = script.reg_io_state_size
    t = np.full(rio, 0xFFFFFFFF, dtype=np.uint32)
    for p in input_positions(script).tolist():
        t[p >> 5] &= np.uint32(~(1 << (p & 31)) & 0xFFFFFFFF)
    return t


def expand_states_for_xprop(value_states, script):
    """[values | xmask template] per snapshot (src/sim/vcd_io.rs:465-484)."""
    rio = script.reg_io_state_size
    v = np.asarray(value_states, dtype=np.uint32).reshape(-1, rio)
    out = np.empty((v.shape[0], 2 * rio), dtype=np.uint32)
    out[:, :rio] = v
    out[:, rio:] = xmask_template(script)
    return out


def split_xprop_states(states, rio):
    """src/sim/vcd_io.rs:491-504."""
    s = np.asarray(states, dtype=np.uint32).reshape(-1, 2 * rio)
    return s[:, :rio].copy(), s[:, rio:].copy()


def expand_states_for_arrivals(states, script):
    """Append a zeroed arrival section per snapshot (src/sim/vcd_io.rs:511-530)."""
    rio = script.reg_io_state_size
    old = rio * (2 if script.xprop_enabled else 1)
    s = np.asarray(states, dtype=np.uint32).reshape(-1, old)
    out = np.zeros((s.shape[0], old + rio), dtype=np.uint32)
    out[:, :old] = s
    return out


def split_arrival_states(states, script):
    """src/sim/vcd_io.rs:537-550."""
    eff = effective_state_size(script)
    rio = script.reg_io_state_size
    s = np.asarray(states, dtype=np.uint32).reshape(-1, eff)
    a = script.arrival_state_offset
    return s[:, a:a + rio].copy()


def dff_positions(script, design):
    return np.array([script.input_map[int(q)] for q in design.dff_q], dtype=np.int64)


def po_positions(script, design):
    return np.array([script.output_map[int(p)] for p in design.primary_outputs], dtype=np.int64)


def bits_at(states, pos):
    """Extract bits at state positions: states (rows, words) -> (rows, len(pos))."""
    s = np.asarray(states, dtype=np.uint32)
    return ((s[:, pos >> 5] >> (pos & 31).astype(np.uint32)) & 1).astype(np.uint8)
